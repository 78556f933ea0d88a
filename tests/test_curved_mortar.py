"""L2 mortars on curvilinear meshes (the reference's P4estMesh{2} path after an AMR step: a warped StructuredMesh
with some cells refined once): the oracle's properties on the CPU and libtlw's curvilinear mortar kernel against
the oracle on the GPU."""
import os

import numpy as np
import pytest

from test_curved import quad, rel_l2, vortex_state, warp

NTH = os.cpu_count() or 1
REFINED = [(1, 1), (2, 1), (4, 4), (5, 4), (4, 5), (0, 5)]


def affine(xi, eta):
    return 10.0 * xi, 10.0 * eta


def refined(tl, mapping=warp, cells=(6, 6), periodicity=True):
    from trixilw.curved_mesh import RefinedStructuredMesh
    return RefinedStructuredMesh(cells, mapping, REFINED, periodicity=periodicity)


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("N", [3, 4])
def test_oracle_curved_mortar_free_stream_affine_and_conservation(oracle_mod, tl, N):
    """A free stream stays one on the affinely mapped refined mesh (there -n_large / 2 is the small face's
    normal), and the rhs conserves every variable on the warped one (the large face takes the L2 projection of
    the small faces' fluxes)."""
    m = refined(tl, affine)
    cm = m.curved(N)
    assert cm.n_mortars > 0
    o = oracle_mod.Oracle(cm, N)
    u = np.tile(np.array([1.0, 0.3, -0.2, 2.5]), cm.n_elements * (N + 1) ** 2)
    assert np.abs(o.rhs(u, 0.0, 0.05)).max() < 1e-12
    cm = refined(tl).curved(N)
    o = oracle_mod.Oracle(cm, N)
    u = vortex_state(tl, cm)
    du = o.rhs(u, 0.0, o.max_dt(u, 0.4))
    assert np.all(np.abs(quad(cm, N, du)) < 1e-11)
    assert np.abs(du).max() > 1e-3


@pytest.mark.parametrize("kind", [0, 1])
def test_oracle_curved_mortar_vortex_runs(oracle_mod, tl, kind):
    """LW (kind 0) and MDRK (kind 1) steps of the vortex on the warped refined mesh stay close to the exact
    translation and conserve mass."""
    N = 4
    cm = refined(tl, cells=(8, 8)).curved(N)
    o = oracle_mod.Oracle(cm, N)
    u = vortex_state(tl, cm)
    m0 = quad(cm, N, u)
    s, t = o.steps(u, 40, 0.3, 0.0, 1e9, kind=kind, nthreads=NTH)
    assert s == 40 and np.all(np.isfinite(u))
    np.testing.assert_allclose(quad(cm, N, u), m0, rtol=1e-12, atol=1e-12)


# ---------------------------------------------------------------------------------------------- GPU
def make_semi(tl, mesh, N, td="lw", bc=None):
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tdo))
    kw = {} if bc is None else {"boundary_conditions": bc}
    return tl.SemidiscretizationHyperbolic(mesh, tdo, eq, tl.IsentropicVortex(5.0), solver, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [3, 4, 5])
def test_gpu_curved_mortar_rhs_matches_oracle(oracle_mod, tl, N):
    m = refined(tl)
    cm = m.curved(N)
    semi = make_semi(tl, m, N)
    u = vortex_state(tl, cm)
    o = oracle_mod.Oracle(cm, N)
    dt = o.max_dt(u, 0.3)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    du_cpu = o.rhs(u, 0.0, dt)
    assert np.all(rel_l2(u + dt * du, u + dt * du_cpu) < 1e-12)
    assert np.all(rel_l2(du, du_cpu) < 1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("td", ["lw", "mdrk"])
def test_gpu_curved_mortar_steps_match_oracle(oracle_mod, tl, td):
    N = 4
    m = refined(tl, cells=(8, 8))
    cm = m.curved(N)
    semi = make_semi(tl, m, N, td)
    u0 = vortex_state(tl, cm)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(12, 0.3, use_graph=True)
    integ.sync_time()
    o = oracle_mod.Oracle(cm, N)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 12, 0.3, 0.0, 1e9, kind=0 if td == "lw" else 1, nthreads=NTH)
    assert s == integ.iter == 12 and integ.t == pytest.approx(t, rel=1e-12)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-12)


@pytest.mark.gpu
def test_gpu_curved_mortar_with_walls_matches_oracle(oracle_mod, tl):
    """The refined mesh with slip walls on its four sides (mortars next to the walls too)."""
    N = 4
    m = refined(tl, periodicity=False)
    cm = m.curved(N)
    bc = {"x_neg": tl.boundary_condition_slip_wall_vertical, "x_pos": tl.boundary_condition_slip_wall_vertical,
          "y_neg": tl.boundary_condition_slip_wall_horizontal, "y_pos": tl.boundary_condition_slip_wall_horizontal}
    semi = make_semi(tl, m, N, bc=bc)
    eq = tl.CompressibleEulerEquations2D(1.4)
    v = tl.IsentropicVortex(3.0, center=(0.3, -0.2), velocity=(0.0, 0.0))(cm.xy[0], cm.xy[1], 0.0, eq)
    u0 = np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)
    o = oracle_mod.Oracle(cm, N)
    o.set_curved_boundaries(cm.boundary_elements, cm.boundary_faces,
                            np.repeat(np.array([1, 1, 2, 2], dtype=np.int32), cm.n_boundaries_per_direction))
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(8, 0.3, use_graph=True)
    integ.sync_time()
    u_cpu = u0.copy()
    s, _ = o.steps(u_cpu, 8, 0.3, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 8
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-12)


def noisy_constant(cm, N, seed=4):
    """rho = 1 (+-30 %), p = 1 (+-50 %) node noise at rest: nodes below the limiter's thresholds, element means
    above them."""
    rng = np.random.default_rng(seed)
    k = cm.n_elements * (N + 1) ** 2
    rho = 1.0 + 0.3 * rng.uniform(-1.0, 1.0, k)
    p = 1.0 + 0.5 * rng.uniform(-1.0, 1.0, k)
    return np.stack([rho, 0 * rho, 0 * rho, p / 0.4], axis=-1).reshape(-1)


@pytest.mark.parametrize("N", [3, 4])
def test_oracle_curved_mortar_limiter_acts_on_large_elements(oracle_mod, tl, N):
    """The P4estMesh limit_mortars! blends large elements whose mortar trace dips below the threshold."""
    cm = refined(tl).curved(N)
    o = oracle_mod.Oracle(cm, N)
    u = noisy_constant(cm, N)
    o.set_positivity_limiter((0.8, 0.6), (0, 1))
    lim = o.apply_positivity_limiter(u)
    nn = 4 * (N + 1) ** 2
    changed = np.any(lim.reshape(-1, nn) != u.reshape(-1, nn), axis=1)
    assert changed[cm.mortar_large - 1].any()


@pytest.mark.gpu
@pytest.mark.parametrize("N", [3, 4, 5])
def test_gpu_curved_mortar_limiter_matches_oracle(oracle_mod, tl, N):
    from trixilw import limiters
    m = refined(tl)
    cm = m.curved(N)
    semi = make_semi(tl, m, N)
    u = noisy_constant(cm, N)
    thr = (0.8, 0.6)
    o = oracle_mod.Oracle(cm, N)
    o.set_positivity_limiter(thr, (0, 1))
    expect = o.apply_positivity_limiter(u)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1.0)))
    integ.set_state(u, 0.0)
    limiters.install(semi, (tl.PositivityPreservingLimiterZhangShu(thr, (tl.density, tl.pressure)),))
    tl._lib.check(semi.handle, tl._lib.lib().tlw_apply_positivity_limiter(semi.handle))
    assert np.all(rel_l2(integ.get_state(), expect) < 1e-13)
    # and limited steps
    u_cpu = expect.copy()
    integ.step(6, 0.3, use_graph=True)
    integ.sync_time()
    s, _ = o.steps(u_cpu, 6, 0.3, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 6
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-12)
