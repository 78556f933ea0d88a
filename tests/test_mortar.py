"""L2 mortars of a non-conforming TreeMesh{2} (a refined patch, as after one AMR step): the mortar
operators and the oracle's properties on the CPU, libtlw's mortar kernel against the oracle on the GPU
(1e-12 relative L2 per variable of the state after one step)."""
import os

import numpy as np
import pytest

NTH = os.cpu_count() or 1


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def refined(tl, level=3):
    return tl.RefinedTreeMesh((-10.0, -10.0), (10.0, 10.0), level, ((-4.0, -4.0), (4.0, 4.0)))


def vortex(tl, mesh, N, beta=5.0):
    eq = tl.CompressibleEulerEquations2D(1.4)
    xy = mesh.node_coordinates(N)
    v = tl.IsentropicVortex(beta, center=(0.7, -0.4))(xy[0], xy[1], 0.0, eq)
    return np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 7])
def test_mortar_operators(oracle_mod, tl, N):
    from trixilw.basis import gauss_lobatto
    fu, fl, ru, rl = oracle_mod.mortar_operators(N)
    x, w = gauss_lobatto(N)
    rng = np.random.default_rng(N)
    c = rng.standard_normal(N + 1)
    p = np.polynomial.polynomial.polyval(x, c)
    # forward: exact interpolation onto the halves
    np.testing.assert_allclose(fu @ p, np.polynomial.polynomial.polyval(0.5 * (x + 1), c), atol=1e-13)
    np.testing.assert_allclose(fl @ p, np.polynomial.polynomial.polyval(0.5 * (x - 1), c), atol=1e-13)
    # reverse: the L2 projection returns a large-face polynomial unchanged and keeps integrals
    np.testing.assert_allclose(ru @ (fu @ p) + rl @ (fl @ p), p, atol=1e-13)
    f_u, f_l = rng.standard_normal(N + 1), rng.standard_normal(N + 1)
    assert w @ (ru @ f_u + rl @ f_l) == pytest.approx(0.5 * (w @ f_u + w @ f_l), rel=1e-13, abs=1e-14)


def test_refined_mesh_connectivity(tl):
    m = refined(tl)
    assert (m.n_elements, m.n_interfaces, m.n_mortars) == (112, 200, 16)
    # every element face is covered exactly once by an interface or a mortar
    cover = np.zeros((m.n_elements, 4), dtype=int)
    ids = m.interface_neighbor_ids.reshape(-1, 2) - 1
    for (l, r), o in zip(ids, m.interface_orientations):
        cover[l, 1 if o == 1 else 3] += 1
        cover[r, 0 if o == 1 else 2] += 1
    mids = m.mortar_neighbor_ids.reshape(-1, 3) - 1
    for (lo, up, lg), side, o in zip(mids, m.mortar_large_sides, m.mortar_orientations):
        small_face = (0 if o == 1 else 2) if side == 1 else (1 if o == 1 else 3)
        large_face = (1 if o == 1 else 3) if side == 1 else (0 if o == 1 else 2)
        cover[lo, small_face] += 1
        cover[up, small_face] += 1
        cover[lg, large_face] += 1
    assert np.all(cover == 1)


@pytest.mark.parametrize("N", [2, 3, 4])
def test_oracle_mortar_free_stream_and_conservation(oracle_mod, tl, N):
    from trixilw.basis import gauss_lobatto
    m = refined(tl)
    o = oracle_mod.Oracle(m, N)
    u = np.tile(np.array([1.0, 0.3, -0.2, 2.5]), m.n_elements * (N + 1) ** 2)
    assert np.abs(o.rhs(u, 0.0, 0.05)).max() < 1e-12
    u = vortex(tl, m, N)
    du = o.rhs(u, 0.0, o.max_dt(u, 0.4))
    _, w = gauss_lobatto(N)
    tot = np.einsum("ejiv,e,j,i->v", du.reshape(-1, N + 1, N + 1, 4), (1.0 / m.inverse_jacobian) ** 2, w, w)
    assert np.all(np.abs(tot) < 1e-11)


# ---------------------------------------------------------------------------------------------- GPU
def make_semi(tl, mesh, N, td="lw", flux=None):
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    solver = tl.DGSEM(N, flux or tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tdo))
    return tl.SemidiscretizationHyperbolic(mesh, tdo, eq, tl.IsentropicVortex(5.0), solver)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_gpu_mortar_rhs_matches_oracle(oracle_mod, tl, N):
    m = refined(tl)
    semi = make_semi(tl, m, N)
    u = vortex(tl, m, N)
    o = oracle_mod.Oracle(m, N)
    dt = o.max_dt(u, 0.3)
    du_cpu = o.rhs(u, 0.0, dt)
    semi.cache["dt"][0] = dt
    du_gpu = np.empty_like(u)
    tl.rhs(du_gpu, u, semi, 0.0)
    assert np.all(rel_l2(u + dt * du_gpu, u + dt * du_cpu) < 1e-12)
    assert np.all(rel_l2(du_gpu, du_cpu) < 1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("td,flux,speed", [("lw", "hll", "naive"), ("lw", "rusanov", "davis"), ("mdrk", "rusanov", "naive")])
def test_gpu_mortar_steps_match_oracle(oracle_mod, tl, td, flux, speed):
    m = refined(tl)
    f = tl.FluxLaxFriedrichs(max_abs_speed=speed) if flux == "rusanov" else tl.FluxHLL()
    semi = make_semi(tl, m, 4, td, f)
    u0 = vortex(tl, m, 4)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(7, 0.3, use_graph=True)
    integ.sync_time()
    u_gpu = integ.get_state()
    o = oracle_mod.Oracle(m, 4, flux_kind=0 if flux == "rusanov" else 1, speed_kind=1 if speed == "davis" else 0)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 7, 0.3, 0.0, 1e9, kind=0 if td == "lw" else 1, nthreads=NTH)
    assert s == integ.iter == 7 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(u_gpu, u_cpu) < 1e-12)


# ------------------------------------------------------------------ shock capturing across mortars (TreeMesh)
def blast(tl, mesh, N):
    """A circular blast at rest around (-3, -3), across the refined patch's corner: (rho, p) = (1, 3) inside
    radius 3, (0.5, 1) outside."""
    eq = tl.CompressibleEulerEquations2D(1.4)
    x, y = mesh.node_coordinates(N)
    inside = (x + 3.0) ** 2 + (y + 3.0) ** 2 < 9.0
    z = np.zeros(x.shape)
    v = eq.prim2cons(np.where(inside, 1.0, 0.5), z, z, np.where(inside, 3.0, 1.0))
    return np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)


def sc_semi(tl, mesh, N, td="lw"):
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5), tl.VolumeIntegralFR(tdo))
    return tl.SemidiscretizationHyperbolic(mesh, tdo, eq, tl.IsentropicVortex(5.0),
                                           tl.DGSEM(N, tl.flux_lax_friedrichs, vi))


@pytest.mark.parametrize("N", [3, 4])
def test_oracle_sc_across_mortars_conserves(oracle_mod, tl, N):
    """Shock capturing on the refined TreeMesh: the blending factors are smoothed across the mortars (a large
    element next to a blended small one gets half its factor), the mortars keep the plain LW flux, the rhs
    conserves."""
    m = refined(tl)
    o = oracle_mod.Oracle(m, N)
    o.set_shock_capturing(True, 0.5, 0.001, True)
    u = blast(tl, m, N)
    du = o.rhs(u, 0.0, o.max_dt(u, 0.15))
    alpha = o.get(6)
    assert alpha.max() > 0.1
    o2 = oracle_mod.Oracle(m, N)
    o2.set_shock_capturing(True, 0.5, 0.001, False)
    o2.rhs(u, 0.0, o.max_dt(u, 0.15))
    raw = o2.get(6)
    ids = np.asarray(m.mortar_neighbor_ids).reshape(-1, 3) - 1
    for lo, up, lg in ids:
        assert alpha[lg] >= 0.5 * max(raw[lo], raw[up]) and alpha[lo] >= 0.5 * raw[lg]
    x, y = m.node_coordinates(N)
    jac = (1.0 / m.inverse_jacobian) ** 2
    from trixilw.basis import gauss_lobatto
    _, w = gauss_lobatto(N)
    tot = np.einsum("ejiv,e,j,i->v", du.reshape(-1, N + 1, N + 1, 4), jac, w, w)
    assert np.all(np.abs(tot) < 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("N,td", [(3, "lw"), (4, "lw"), (4, "mdrk")])
def test_gpu_sc_across_mortars_matches_oracle(oracle_mod, tl, N, td):
    m = refined(tl)
    semi = sc_semi(tl, m, N, td)
    u0 = blast(tl, m, N)
    o = oracle_mod.Oracle(m, N)
    o.set_shock_capturing(True, 0.5, 0.001, True)
    dt = o.max_dt(u0, 0.15)
    if td == "lw":
        semi.cache["dt"][0] = dt
        du = np.empty_like(u0)
        tl.rhs(du, u0, semi, 0.0)
        assert np.all(rel_l2(u0 + dt * du, u0 + dt * o.rhs(u0, 0.0, dt)) < 1e-12)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(8, 0.15, use_graph=True)
    integ.sync_time()
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 8, 0.15, 0.0, 1e9, kind=0 if td == "lw" else 1, nthreads=NTH)
    assert s == integ.iter == 8 and integ.t == pytest.approx(t, rel=1e-12)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-11)
