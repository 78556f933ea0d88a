"""Shock capturing on curvilinear conforming meshes (the reference's P4estMesh{2} path: Hennemann-Gassner
blending with first-order or MUSCL subcells, the blended interface flux with the Zhang-Shu flux fix): the
oracle's properties on the CPU, and libtlw's kernels against the oracle on the GPU."""
import os

import numpy as np
import pytest

from test_curved import quad, rel_l2, warp

NTH = os.cpu_count() or 1
GAMMA = 1.4


def blast_state(cm, rho_in=1.0, p_in=10.0, rho_out=0.125, p_out=1.0, r0=3.0, center=(0.5, -0.7)):
    """A circular blast at rest: (rho_in, p_in) inside radius r0, (rho_out, p_out) outside."""
    x, y = cm.xy
    inside = (x - center[0]) ** 2 + (y - center[1]) ** 2 < r0 ** 2
    rho = np.where(inside, rho_in, rho_out)
    p = np.where(inside, p_in, p_out)
    v = np.stack([rho, 0.0 * rho, 0.0 * rho, p / (GAMMA - 1.0)], axis=-1)   # [i, j, e, v]
    return np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)


def make(oracle_mod, tl, N, cells=(6, 6), rec=0, alpha_max=0.5, rotate=False):
    m = tl.StructuredMesh(cells, warp)
    cm = m.curved(N)
    if rotate:
        turns = np.random.default_rng(N + 7).integers(0, 4, cm.n_elements)
        cm = tl.rotate_elements(cm, turns)
    o = oracle_mod.Oracle(cm if rotate else m, N)
    o.set_shock_capturing(True, alpha_max=alpha_max, alpha_min=0.001, alpha_smooth=True, reconstruction=rec)
    return m, cm, o


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("N", [3, 4])
def test_oracle_curved_sc_without_blending_is_the_fr_rhs(oracle_mod, tl, N):
    """alpha_max = 0: every element is pure DG and the blended interface flux is the LW flux, so the rhs is
    the FR one bit for bit (a smooth state keeps every subcell update admissible)."""
    m = tl.StructuredMesh((6, 6), warp)
    cm = m.curved(N)
    from test_curved import vortex_state
    u = vortex_state(tl, cm)
    plain = oracle_mod.Oracle(m, N)
    dt = plain.max_dt(u, 0.4)
    _, _, o = make(oracle_mod, tl, N, alpha_max=0.0)
    np.testing.assert_array_equal(o.rhs(u, 0.0, dt), plain.rhs(u, 0.0, dt))
    assert np.all(o.get(6) == 0.0)


@pytest.mark.parametrize("N,rec", [(3, 0), (4, 0), (4, 1), (5, 1), (3, 2), (4, 2)])
def test_oracle_curved_sc_blast_conservation(oracle_mod, tl, N, rec):
    """The blast: blending is active near the discontinuity, the rhs conserves every variable on the
    periodic mesh, and a few steps stay admissible."""
    _, cm, o = make(oracle_mod, tl, N, cells=(8, 8), rec=rec)
    u = blast_state(cm)
    dt = o.max_dt(u, 0.2)
    du = o.rhs(u, 0.0, dt)
    alpha = o.get(6)
    assert alpha.max() > 0.1 and (alpha == 0.0).sum() > 0
    assert np.all(np.abs(quad(cm, N, du)) < 1e-11 * np.abs(quad(cm, N, u)).max())
    mass0 = quad(cm, N, u)
    s, _ = o.steps(u, 20, 0.2, 0.0, 1e9, nthreads=NTH)
    assert s == 20 and np.all(np.isfinite(u))
    np.testing.assert_allclose(quad(cm, N, u), mass0, rtol=1e-12, atol=1e-12)
    uu = u.reshape(-1, 4)
    p = (GAMMA - 1.0) * (uu[:, 3] - 0.5 * (uu[:, 1] ** 2 + uu[:, 2] ** 2) / uu[:, 0])
    assert uu[:, 0].min() > 0.0 and p.min() > 0.0


def test_oracle_curved_muscl_differs_from_first_order(oracle_mod, tl):
    """MUSCL subcells change the blended elements' rhs once the state is no longer piecewise constant (on the
    initial blast every minmod slope is zero)."""
    N = 4
    _, cm, o1 = make(oracle_mod, tl, N, cells=(8, 8), rec=0)
    _, _, o2 = make(oracle_mod, tl, N, cells=(8, 8), rec=1)
    u = blast_state(cm)
    dt = o1.max_dt(u, 0.2)
    np.testing.assert_array_equal(o1.rhs(u, 0.0, dt), o2.rhs(u, 0.0, dt))
    o1.steps(u, 10, 0.2, 0.0, 1e9, nthreads=NTH)
    dt = o1.max_dt(u, 0.2)
    d1, d2 = o1.rhs(u, 0.0, dt).reshape(cm.n_elements, -1), o2.rhs(u, 0.0, dt).reshape(cm.n_elements, -1)
    alpha = o1.get(6)
    diff = np.abs(d1 - d2).max(axis=1)
    assert diff[alpha > 0].max() > 1e-3
    # MUSCL-Hancock (centred-difference slopes and the half-step update) differs from MUSCL as well
    _, _, o3 = make(oracle_mod, tl, N, cells=(8, 8), rec=2)
    d3 = o3.rhs(u, 0.0, dt).reshape(cm.n_elements, -1)
    assert np.abs(d3 - d2).max(axis=1)[alpha > 0].max() > 1e-3


# ---------------------------------------------------------------------------------------------- GPU
RECONSTRUCTIONS = {0: lambda tl: tl.FirstOrderReconstruction(), 1: lambda tl: tl.MUSCLReconstruction(),
                   2: lambda tl: tl.MUSCLHancockReconstruction()}


def sc_semi(tl, mesh, N, rec, bc=None):
    eq = tl.CompressibleEulerEquations2D(GAMMA)
    vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5, alpha_min=0.001),
                                           tl.VolumeIntegralFR(tl.LW()),
                                           reconstruction=RECONSTRUCTIONS[rec](tl))
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, vi)
    kw = {} if bc is None else {"boundary_conditions": bc}
    return tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, tl.ConstantState(), solver, **kw)


def gpu_rhs(tl, semi, u, dt):
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    return du


@pytest.mark.gpu
@pytest.mark.parametrize("N,rec,rotated", [(3, 0, False), (4, 0, True), (5, 0, False), (3, 1, True), (4, 1, False),
                                           (5, 1, True), (3, 2, False), (4, 2, True), (5, 2, False)])
def test_gpu_curved_sc_rhs_matches_oracle(oracle_mod, tl, N, rec, rotated):
    """One rhs of a blast that has run a few oracle steps (nonzero MUSCL slopes): blending factors, the
    face-adjacent subcell fluxes and du against the oracle."""
    from trixilw import _lib
    m, cm, o = make(oracle_mod, tl, N, cells=(8, 8), rec=rec, rotate=rotated)
    u = blast_state(cm)
    o.steps(u, 6, 0.2, 0.0, 1e9, nthreads=NTH)
    semi = sc_semi(tl, cm, N, rec)
    dt = o.max_dt(u, 0.2)
    assert semi.max_dt(u, 0.2) == pytest.approx(dt, rel=1e-13)
    du_cpu = o.rhs(u, 0.0, dt)
    du_gpu = gpu_rhs(tl, semi, u, dt)
    alpha = o.get(6)
    assert alpha.max() > 0.1
    np.testing.assert_allclose(semi.get_cache(_lib.TLW_CACHE_ALPHA), alpha, rtol=1e-12, atol=1e-15)
    fl_cpu, fl_gpu = o.get(7), semi.get_cache(_lib.TLW_CACHE_FN_LOW)
    assert np.all(rel_l2(fl_gpu, fl_cpu) < 1e-12)
    assert np.all(rel_l2(u + dt * du_gpu, u + dt * du_cpu) < 1e-12)
    assert np.all(rel_l2(du_gpu, du_cpu) < 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("rec", [0, 1, 2])
def test_gpu_curved_sc_steps_match_oracle(oracle_mod, tl, rec):
    """20 CFL steps of the blast (N = 4, rotated element frames) on the device against the oracle."""
    _, cm, o = make(oracle_mod, tl, 4, cells=(8, 8), rec=rec, rotate=True)
    semi = sc_semi(tl, cm, 4, rec)
    u0 = blast_state(cm)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(20, 0.2, use_graph=True)
    integ.sync_time()
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 20, 0.2, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 20 and integ.t == pytest.approx(t, rel=1e-12)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("rec", [0, 1, 2])
def test_gpu_curved_sc_walls_match_oracle(oracle_mod, tl, rec):
    """The blast in a warped box with slip walls: MUSCL falls back to first-order subcells on the elements
    next to the walls; 10 steps against the oracle."""
    N = 4
    m = tl.StructuredMesh((8, 8), warp, periodicity=False)
    cm = m.curved(N)
    bc = {"x_neg": tl.boundary_condition_slip_wall_vertical, "x_pos": tl.boundary_condition_slip_wall_vertical,
          "y_neg": tl.boundary_condition_slip_wall_horizontal, "y_pos": tl.boundary_condition_slip_wall_horizontal}
    semi = sc_semi(tl, cm, N, rec, bc)
    o = oracle_mod.Oracle(cm, N)
    o.set_curved_boundaries(cm.boundary_elements, cm.boundary_faces,
                            np.repeat(np.array([1, 1, 2, 2], dtype=np.int32), cm.n_boundaries_per_direction))
    o.set_shock_capturing(True, alpha_max=0.5, alpha_min=0.001, alpha_smooth=True, reconstruction=rec)
    u0 = blast_state(cm, center=(-5.0, 4.0))
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(10, 0.2, use_graph=False)
    integ.sync_time()
    u_cpu = u0.copy()
    s, _ = o.steps(u_cpu, 10, 0.2, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 10
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-11)


@pytest.mark.gpu
def test_gpu_curved_sc_with_positivity_limiter_matches_oracle(oracle_mod, tl):
    """MUSCL shock capturing with the Zhang-Shu limiter after every step (twice per LW step, as solve_lwfr), as
    the reference's curvilinear shock elixirs run. The blast's density and pressure carry node noise (30 %,
    50 %) so that some nodes fall below the thresholds while every element mean stays above them (the
    limiter's blend assumes an admissible mean; a threshold above a constant element's value divides by 0).
    8 steps."""
    from trixilw import limiters
    N = 4
    _, cm, o = make(oracle_mod, tl, N, cells=(8, 8), rec=1, rotate=True)
    semi = sc_semi(tl, cm, N, 1)
    u0 = blast_state(cm, p_in=100.0).reshape(-1, 4)
    rng = np.random.default_rng(5)
    p = (GAMMA - 1.0) * u0[:, 3] * (1.0 + 0.5 * rng.uniform(-1.0, 1.0, len(u0)))
    u0[:, 0] *= 1.0 + 0.3 * rng.uniform(-1.0, 1.0, len(u0))
    u0[:, 3] = p / (GAMMA - 1.0)
    u0 = u0.reshape(-1)
    thr = (0.1, 0.7)
    o.set_positivity_limiter(thr, (0, 1))
    u_cpu = o.apply_positivity_limiter(u0)
    assert not np.array_equal(u_cpu, u0)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    limiters.install(semi, (tl.PositivityPreservingLimiterZhangShu(thr, (tl.density, tl.pressure)),))
    tl._lib.check(semi.handle, tl._lib.lib().tlw_apply_positivity_limiter(semi.handle))
    integ.step(8, 0.2, use_graph=True)
    integ.sync_time()
    s, t = o.steps(u_cpu, 8, 0.2, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 8 and integ.t == pytest.approx(t, rel=1e-12)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-11)


# ---------------------------------------------------------------------------------------------- MDRK
@pytest.mark.parametrize("rec", [0, 1, 2])
def test_oracle_curved_sc_mdrk_conservation(oracle_mod, tl, rec):
    """MDRK with shock capturing on the curvilinear mesh (the reference's double Mach elixirs): both stages
    conserve on the periodic mesh and a few two-stage steps stay admissible."""
    N = 4
    _, cm, o = make(oracle_mod, tl, N, cells=(8, 8), rec=rec, rotate=True)
    u = blast_state(cm)
    dt = o.max_dt(u, 0.15)
    scale = np.abs(quad(cm, N, u)).max()
    d1 = o.rhs(u, 0.0, dt, kind=1)
    assert np.all(np.abs(quad(cm, N, d1)) < 1e-11 * scale)
    d2 = o.rhs(u, 0.0, dt, kind=2, us=u + dt * d1)
    assert np.all(np.abs(quad(cm, N, d2)) < 1e-11 * scale)
    mass0 = quad(cm, N, u)
    s, _ = o.steps(u, 10, 0.15, 0.0, 1e9, kind=1, nthreads=NTH)
    assert s == 10 and np.all(np.isfinite(u))
    np.testing.assert_allclose(quad(cm, N, u), mass0, rtol=1e-12, atol=1e-12)


def sc_semi_mdrk(tl, mesh, N, rec):
    eq = tl.CompressibleEulerEquations2D(GAMMA)
    vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5, alpha_min=0.001),
                                           tl.VolumeIntegralFR(tl.MDRK()),
                                           reconstruction=RECONSTRUCTIONS[rec](tl))
    return tl.SemidiscretizationHyperbolic(mesh, tl.MDRK(), eq, tl.ConstantState(),
                                           tl.DGSEM(N, tl.flux_lax_friedrichs, vi))


@pytest.mark.gpu
@pytest.mark.parametrize("N,rec", [(3, 1), (4, 0), (4, 1), (4, 2)])
def test_gpu_curved_sc_mdrk_stages_match_oracle(oracle_mod, tl, N, rec):
    """rhs_mdrk1 / rhs_mdrk2 with shock capturing on the rotated warped mesh against the oracle."""
    _, cm, o = make(oracle_mod, tl, N, cells=(8, 8), rec=rec, rotate=True)
    u = blast_state(cm)
    o.steps(u, 4, 0.15, 0.0, 1e9, kind=1, nthreads=NTH)
    semi = sc_semi_mdrk(tl, cm, N, rec)
    dt = o.max_dt(u, 0.15)
    semi.cache["dt"][0] = dt
    d1_gpu = np.empty_like(u)
    tl.rhs_mdrk1(d1_gpu, u, semi, 0.0)
    d1_cpu = o.rhs(u, 0.0, dt, kind=1)
    assert np.all(rel_l2(u + dt * d1_gpu, u + dt * d1_cpu) < 1e-12)
    us = u + dt * d1_cpu
    d2_gpu = np.empty_like(u)
    tl.rhs_mdrk2(d2_gpu, u, semi, 0.0, us)
    d2_cpu = o.rhs(u, 0.0, dt, kind=2, us=us)
    assert np.all(rel_l2(u + dt * d2_gpu, u + dt * d2_cpu) < 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("rec", [0, 1, 2])
def test_gpu_curved_sc_mdrk_steps_match_oracle(oracle_mod, tl, rec):
    _, cm, o = make(oracle_mod, tl, 4, cells=(8, 8), rec=rec, rotate=True)
    semi = sc_semi_mdrk(tl, cm, 4, rec)
    u0 = blast_state(cm)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.MDRK(), (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(12, 0.15, use_graph=True)
    integ.sync_time()
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 12, 0.15, 0.0, 1e9, kind=1, nthreads=NTH)
    assert s == integ.iter == 12 and integ.t == pytest.approx(t, rel=1e-12)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-11)
