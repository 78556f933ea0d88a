"""Zhang-Shu positivity limiter (PositivityPreservingLimiterZhangShu as TrixiLW applies it after a step,
src/callbacks/callbacks_stage/positivity_zhang_shu_dg2d.jl:8-176): the oracle's properties on the CPU
(thresholds met, element means kept, untouched elements unchanged, the mortar pass), the Python interface,
and libtlw's fused limiter kernel against the oracle on the GPU: one application, and whole runs of LW and
MDRK steps with the limiter active every step (1e-12 relative L2 per variable)."""
import os

import numpy as np
import pytest

NTH = os.cpu_count() or 1
GAMMA = 1.4


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def pressure(u):
    u = u.reshape(-1, 4)
    return (GAMMA - 1.0) * (u[:, 3] - 0.5 * (u[:, 1] ** 2 + u[:, 2] ** 2) / u[:, 0])


def noisy_state(mesh, N, seed, amp=0.35):
    """rho = 1 + noise, v = (0.3, -0.2) + noise, p = 1 + noise per node, the noise amplitude amp in even
    elements and amp / 4 in odd ones: nodes of the even elements dip below rho 0.75 / p 0.75 while every
    element mean stays near 1 (the limiter's working regime) and the odd elements stay above."""
    rng = np.random.default_rng(seed)
    nn = (N + 1) ** 2
    nodes = mesh.n_elements * nn
    a = np.where(np.arange(mesh.n_elements) % 2 == 0, amp, 0.25 * amp).repeat(nn)
    rho = 1.0 + a * rng.uniform(-1, 1, nodes)
    v1 = 0.3 + 0.1 * rng.uniform(-1, 1, nodes)
    v2 = -0.2 + 0.1 * rng.uniform(-1, 1, nodes)
    p = 1.0 + a * rng.uniform(-1, 1, nodes)
    u = np.stack([rho, rho * v1, rho * v2, p / (GAMMA - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2)], axis=1)
    return np.ascontiguousarray(u.reshape(-1))


def element_means(u, N):
    from trixilw.basis import gauss_lobatto
    _, w = gauss_lobatto(N)
    return np.einsum("ejiv,j,i->ev", u.reshape(-1, N + 1, N + 1, 4), w, w) / 4.0


def tree(tl, level=3):
    return tl.TreeMesh((-1.0, -1.0), (1.0, 1.0), level)


def refined(tl):
    return tl.RefinedTreeMesh((-10.0, -10.0), (10.0, 10.0), 3, ((-4.0, -4.0), (4.0, 4.0)))


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("N", [2, 3, 4, 5])
def test_oracle_limiter_element_pass(oracle_mod, tl, N):
    m = tree(tl)
    o = oracle_mod.Oracle(m, N)
    thr = (0.75, 0.75)
    o.set_positivity_limiter(thr, (0, 1))
    u = noisy_state(m, N, seed=N)
    lim = o.apply_positivity_limiter(u)
    nn = (N + 1) ** 2
    rho0 = u.reshape(-1, nn, 4)[:, :, 0]
    p0 = pressure(u).reshape(-1, nn)
    touched = (rho0.min(axis=1) < thr[0]) | (p0.min(axis=1) < thr[1])
    assert touched.any() and (~touched).any()
    # elements above both thresholds are left bit for bit; the others keep their mean and meet the thresholds
    ue, le = u.reshape(-1, nn * 4), lim.reshape(-1, nn * 4)
    assert np.array_equal(ue[~touched], le[~touched])
    np.testing.assert_allclose(element_means(lim, N), element_means(u, N), rtol=1e-13, atol=1e-14)
    assert lim.reshape(-1, 4)[:, 0].min() >= thr[0] * (1 - 1e-12)
    assert pressure(lim).min() >= thr[1] * (1 - 1e-12)
    # the minimum sits on the threshold in the elements the density pass limited (linear in theta)
    rho1 = lim.reshape(-1, nn, 4)[:, :, 0]
    dens = rho0.min(axis=1) < thr[0]
    np.testing.assert_allclose(rho1[dens].min(axis=1)[p0[dens].min(axis=1) >= thr[1]], thr[0], rtol=1e-12)


def test_oracle_limiter_nan_element_left_alone(oracle_mod, tl):
    # Julia's min propagates NaN and NaN < threshold is false: such an element is not limited
    m = tree(tl, 2)
    N = 3
    o = oracle_mod.Oracle(m, N)
    o.set_positivity_limiter((0.75,), (0,))
    u = noisy_state(m, N, seed=1)
    nn = (N + 1) ** 2
    u.reshape(-1, nn, 4)[0, 0, 0] = np.nan
    u.reshape(-1, nn, 4)[0, 1, 0] = 0.1
    lim = o.apply_positivity_limiter(u)
    np.testing.assert_array_equal(lim.reshape(-1, nn * 4)[0], u.reshape(-1, nn * 4)[0])


def spike_mortar_faces(mesh, N, u, rho_face=3.0):
    """Density rho_face on every large element's mortar face (velocity and pressure kept): an admissible
    state whose face traces lie far above the element mean, where limit_mortars!'s theta = min(|(value_mean -
    threshold) / (value_mean - value_min)|, 1) drops below 1 although no node is below the threshold."""
    u = u.reshape(-1, N + 1, N + 1, 4).copy()     # [e, j, i, v]
    ids = mesh.mortar_neighbor_ids.reshape(-1, 3) - 1
    for k in range(len(ids)):
        lg, side, ori = ids[k, 2], mesh.mortar_large_sides[k], mesh.mortar_orientations[k]
        fi = N if side == 1 else 0
        sl = (lg, slice(None), fi) if ori == 1 else (lg, fi, slice(None))
        x = u[sl]
        rho, v1, v2 = x[:, 0], x[:, 1] / x[:, 0], x[:, 2] / x[:, 0]
        p = (GAMMA - 1.0) * (x[:, 3] - 0.5 * rho * (v1 * v1 + v2 * v2))
        r = np.full_like(rho, rho_face)
        u[sl] = np.stack([r, r * v1, r * v2, p / (GAMMA - 1.0) + 0.5 * r * (v1 * v1 + v2 * v2)], axis=1)
    return np.ascontiguousarray(u.reshape(-1))


def test_oracle_limiter_mortar_pass(oracle_mod, tl):
    """limit_mortars!: every mortar blends its large element towards its mean with theta = min(|(value_mean -
    threshold) / (value_mean - value_min)|, 1), value_min over the large face trace interpolated onto both
    halves. Large elements keep their means; elements in no mortar's large side are left to the element pass,
    which has nothing to do here."""
    m = refined(tl)
    N = 3
    o = oracle_mod.Oracle(m, N)
    u = spike_mortar_faces(m, N, noisy_state(m, N, seed=7, amp=0.05))
    thr = 0.5
    assert u.reshape(-1, 4)[:, 0].min() > thr
    o.set_positivity_limiter((thr,), (0,))
    lim = o.apply_positivity_limiter(u)
    nn = (N + 1) ** 2
    ids = m.mortar_neighbor_ids.reshape(-1, 3) - 1
    large = set(ids[:, 2].tolist())
    ue, le = u.reshape(-1, nn * 4), lim.reshape(-1, nn * 4)
    others = np.array([e not in large for e in range(m.n_elements)])
    assert np.array_equal(ue[others], le[others])
    np.testing.assert_allclose(element_means(lim, N), element_means(u, N), rtol=1e-13, atol=1e-14)
    # theta of every large element with a single mortar, recomputed here from the forward operators
    fu, fl, _, _ = oracle_mod.mortar_operators(N)
    means = element_means(u, N)
    changed = 0
    for k in range(len(ids)):
        lg = ids[k, 2]
        if np.count_nonzero(ids[:, 2] == lg) != 1:
            continue
        side, ori = m.mortar_large_sides[k], m.mortar_orientations[k]
        ul = u.reshape(-1, N + 1, N + 1, 4)[lg]        # [j, i, v]
        fi = N if side == 1 else 0
        face = ul[:, fi, :] if ori == 1 else ul[fi, :, :]
        vals = np.concatenate([(fu @ face)[:, 0], (fl @ face)[:, 0]])
        theta = min(abs((means[lg, 0] - thr) / (means[lg, 0] - vals.min())), 1.0)
        changed += theta < 1.0
        expect = theta * ul + (1 - theta) * means[lg]
        np.testing.assert_allclose(lim.reshape(-1, N + 1, N + 1, 4)[lg], expect, rtol=1e-13, atol=1e-14)
    assert changed > 0


def test_limiter_python_interface(tl):
    from trixilw import limiters
    lim = tl.PositivityPreservingLimiterZhangShu(thresholds=(5.0e-6, 5.0e-6), variables=(tl.density, tl.pressure))
    assert lim.codes == (0, 1)
    thr, var = limiters.pairs((lim, tl.PositivityPreservingLimiterZhangShu((1e-6,), (tl.density_pressure,))))
    assert thr == (5.0e-6, 5.0e-6, 1e-6) and var == (0, 1, 2)
    with pytest.raises(ValueError):
        tl.PositivityPreservingLimiterZhangShu((1e-6,), (tl.density, tl.pressure))
    with pytest.raises(ValueError):
        tl.PositivityPreservingLimiterZhangShu((1e-6,), (len,))
    with pytest.raises(ValueError):
        limiters.pairs((lim, lim, lim))
    u = np.array([[2.0, 1.0, -0.5, 3.0]])
    assert tl.pressure(u)[0] == pytest.approx(0.4 * (3.0 - 0.5 * 1.25 / 2.0))
    assert tl.density_pressure(u)[0] == pytest.approx(2.0 * tl.pressure(u)[0])


# ---------------------------------------------------------------------------------------------- GPU
def make_semi(tl, mesh, N, td="lw"):
    eq = tl.CompressibleEulerEquations2D(GAMMA)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tdo))
    return tl.SemidiscretizationHyperbolic(mesh, tdo, eq, tl.ConstantState(), solver)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 7])
@pytest.mark.parametrize("meshkind", ["tree", "refined"])
def test_gpu_limiter_application_matches_oracle(oracle_mod, tl, N, meshkind):
    from trixilw import limiters
    m = tree(tl) if meshkind == "tree" else refined(tl)
    semi = make_semi(tl, m, N)
    u = noisy_state(m, N, seed=10 + N, amp=0.3)
    if meshkind == "refined":   # the element pass and the mortar pass both act
        u = spike_mortar_faces(m, N, u)
    thr = (0.75, 0.75)
    lim = tl.PositivityPreservingLimiterZhangShu(thr, (tl.density, tl.pressure))
    o = oracle_mod.Oracle(m, N)
    o.set_positivity_limiter(thr, (0, 1))
    expect = o.apply_positivity_limiter(u)
    assert not np.array_equal(expect, u)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1.0)))
    integ.set_state(u, 0.0)
    limiters.install(semi, (lim,))
    lim(None, integ, semi, 0.0)
    got = integ.get_state()
    assert np.all(rel_l2(got, expect) < 1e-13)
    nn = (N + 1) ** 2
    same = np.all(u.reshape(-1, nn * 4) == expect.reshape(-1, nn * 4), axis=1)
    assert np.array_equal(got.reshape(-1, nn * 4)[same], u.reshape(-1, nn * 4)[same])


@pytest.mark.gpu
@pytest.mark.parametrize("td,N,meshkind", [("lw", 4, "tree"), ("lw", 3, "tree"), ("mdrk", 4, "tree"),
                                           ("lw", 4, "refined"), ("lw", 5, "tree")])
def test_gpu_limited_steps_match_oracle(oracle_mod, tl, td, N, meshkind):
    """Steps with the limiter active after every step (LW: twice, MDRK: once, as solve_lwfr), graph-captured,
    CFL from the limited state (the CFL slots rewritten by the limiter on the plain LW path)."""
    from trixilw import limiters
    m = tree(tl, 4) if meshkind == "tree" else refined(tl)
    semi = make_semi(tl, m, N, td)
    u0 = noisy_state(m, N, seed=3, amp=0.3)
    thr = (0.8, 0.8)
    o = oracle_mod.Oracle(m, N)
    o.set_positivity_limiter(thr, (0, 1))
    u_cpu = o.apply_positivity_limiter(u0)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    limiters.install(semi, (tl.PositivityPreservingLimiterZhangShu(thr, (tl.density, tl.pressure)),))
    tl._lib.check(semi.handle, tl._lib.lib().tlw_apply_positivity_limiter(semi.handle))
    integ.step(6, 0.25, use_graph=True)
    integ.sync_time()
    u_gpu = integ.get_state()
    s, t = o.steps(u_cpu, 6, 0.25, 0.0, 1e9, kind=0 if td == "lw" else 1, nthreads=NTH)
    assert s == integ.iter == 6 and integ.t == pytest.approx(t, rel=1e-12)
    assert np.all(rel_l2(u_gpu, u_cpu) < 1e-12)
    # the limiter acted during the run: without it the oracle's run differs
    o.set_positivity_limiter((), ())
    u_free = o.apply_positivity_limiter(u0)
    o.steps(u_free, 6, 0.25, 0.0, 1e9, kind=0 if td == "lw" else 1, nthreads=NTH)
    assert np.max(rel_l2(u_free, u_cpu)) > 1e-6


@pytest.mark.gpu
def test_gpu_solve_lwfr_with_limiter_stays_positive(tl):
    """solve_lwfr(...; limiters) end to end: a near-vacuum density wave (rho down to 1e-3) at N = 4 keeps
    rho and p at or above the thresholds after every callback interval."""
    m = tree(tl, 4)
    N = 4
    eq = tl.CompressibleEulerEquations2D(GAMMA)
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    semi = tl.SemidiscretizationHyperbolic(m, tl.LW(), eq, tl.DensityWave(amplitude=0.999, k=1.0), solver)
    ode = tl.semidiscretize(semi, tl.LW(), (0.0, 0.5))
    thr = (1e-4, 1e-4)
    mins = []

    class Probe:
        interval = 5

        def __call__(self, integ, u):
            mins.append((u.reshape(-1, 4)[:, 0].min(), pressure(u).min()))

    lim = tl.PositivityPreservingLimiterZhangShu(thresholds=thr, variables=(tl.density, tl.pressure))
    sol = tl.solve_lwfr(ode, (Probe(),), 0.0, None, time_step_computation=tl.CFLBased(0.98 * 5 * 0.103),
                        limiters=(lim,))
    assert sol.t[-1] == pytest.approx(0.5)
    assert mins and all(r >= thr[0] * (1 - 1e-9) and p >= thr[1] * (1 - 1e-9) for r, p in mins)
