"""GPU parity at the sizes the throughput numbers are quoted on: libtlw (through the C ABI) against the
multithreaded oracle on the full meshes, not on reduced ones.

* isentropic vortex, periodic TreeMesh 512 x 512, N = 3, 4, 5, LW: one rhs, then 3 device CFL steps;
* the same vortex with the two-stage MDRK step on 256 x 256 (N = 3, 4, 5) and 512 x 512 (N = 4): 3 device steps;
* four-quadrant Riemann problem on [0, 1]^2, TreeMesh 512 x 512, N = 4, Hennemann-Gassner blending
  (alpha_max = 0.5) with first-order subcells and Dirichlet(initial condition) boundaries: one rhs with the
  blending factors and the subcell fluxes next to the faces (fn_low), then 3 device steps;
* the curvilinear bench workloads on the warped 512 x 512 StructuredMesh, N = 4: the LW vortex and the
  shock-capturing blast with MUSCL subcells, 2 device steps;
* the warped 64 x 64 Navier-Stokes lid-driven cavity (Re = 1000, Ma = 0.1, Pr = 0.72, N = 4, slip walls for
  the advective part, no-slip adiabatic walls with the lid at v1 = 1): 20 steps at the workload's fixed dt.

Bar: 1e-12 relative L2 per variable of the state after the steps (the rhs of the 512^2 vortex: of u + dt du,
with du itself at 1e-11, where du is ~0 over the free stream and both sides leave roundoff of ~1e-13 J^-1).
"""
import os

import numpy as np
import pytest

import golden_cases

pytestmark = pytest.mark.gpu

NTH = os.cpu_count() or 1
RTOL = 1e-12


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def cfl_lw(N):
    """0.98 of the LW stability limit (trixi2lw, src/auxiliary/auxiliary.jl:14-23); N = 5: 0.98 * 6 * 0.07."""
    return 0.98 * (N + 1) * {3: 0.170, 4: 0.103}.get(N, 0.07)


def vortex_semi(tl, level, N, td):
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tdo))
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), level)
    return tl.SemidiscretizationHyperbolic(mesh, tdo, eq, tl.IsentropicVortex(5.0), solver)


def device_steps(tl, semi, u0, nsteps, cfl, **kw):
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(nsteps, cfl, use_graph=True, **kw)
    integ.sync_time()
    return integ.get_state(), integ


@pytest.mark.parametrize("N", [3, 4, 5])
def test_vortex_512_rhs_and_steps(tl, oracle_mod, N):
    semi = vortex_semi(tl, 9, N, "lw")
    u0 = semi.compute_coefficients(0.0)
    o = oracle_mod.Oracle(semi.mesh, N)
    cfl = cfl_lw(N)
    dt = o.max_dt(u0, cfl)
    assert semi.max_dt(u0, cfl) == pytest.approx(dt, rel=1e-14)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u0)
    tl.rhs(du, u0, semi, 0.0)
    ref = o.rhs(u0, 0.0, dt, nthreads=NTH)
    assert np.all(rel_l2(u0 + dt * du, u0 + dt * ref) < RTOL)
    assert np.all(rel_l2(du, ref) < 1e-11), rel_l2(du, ref)
    del du, ref
    u_gpu, integ = device_steps(tl, semi, u0, 3, cfl)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 3, cfl, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 3 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(u_gpu, u_cpu) < RTOL), rel_l2(u_gpu, u_cpu)


@pytest.mark.parametrize("level,N", [(8, 3), (8, 4), (8, 5), (9, 4)])
def test_vortex_mdrk_steps(tl, oracle_mod, level, N):
    semi = vortex_semi(tl, level, N, "mdrk")
    u0 = semi.compute_coefficients(0.0)
    cfl = cfl_lw(N)
    u_gpu, integ = device_steps(tl, semi, u0, 3, cfl)
    o = oracle_mod.Oracle(semi.mesh, N)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 3, cfl, 0.0, 1e9, kind=1, nthreads=NTH)
    assert s == integ.iter == 3 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(u_gpu, u_cpu) < RTOL), rel_l2(u_gpu, u_cpu)


def test_riemann_512_N4_shock_capturing(tl, oracle_mod):
    from trixilw import _lib
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((0.0, 0.0), (1.0, 1.0), 9, periodicity=False)
    ic = tl.FourQuadrantRiemann()
    vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5), tl.VolumeIntegralFR(tl.LW()))
    semi = tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, ic, tl.DGSEM(4, tl.flux_lax_friedrichs, vi),
                                           boundary_conditions=tl.BoundaryConditionDirichlet(ic))
    semi._prepare_boundaries(0.0, 0.0, 1.0)
    u0 = semi.compute_coefficients(0.0)
    o = oracle_mod.Oracle(mesh, 4)
    o.set_shock_capturing(True, 0.5, 0.001, True)
    lv, nw = golden_cases.boundary_data(mesh, 4, ic, eq)
    o.set_boundary_data(lv, nw)
    cfl = 0.15
    dt = o.max_dt(u0, cfl)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u0)
    tl.rhs(du, u0, semi, 0.0)
    ref = o.rhs(u0, 0.0, dt, nthreads=NTH)
    assert np.all(rel_l2(u0 + dt * du, u0 + dt * ref) < RTOL)
    alpha, alpha_ref = semi.get_cache(_lib.TLW_CACHE_ALPHA), o.get(6)
    assert alpha_ref.max() > 0.1 and np.count_nonzero(alpha_ref) > 1000     # the shocks are blended
    np.testing.assert_allclose(alpha, alpha_ref, rtol=1e-10, atol=1e-14)
    fnl, fnl_ref = semi.get_cache(_lib.TLW_CACHE_FN_LOW), o.get(7)
    np.testing.assert_allclose(fnl, fnl_ref, rtol=0, atol=1e-12 * np.abs(fnl_ref).max())
    del du, ref
    u_gpu, integ = device_steps(tl, semi, u0, 3, cfl)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 3, cfl, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 3 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(u_gpu, u_cpu) < RTOL), rel_l2(u_gpu, u_cpu)


def test_warped_cavity_64_N4_steps(tl, oracle_mod):
    """20 steps at the workload's fixed dt (5e-5) from a stirred state, so that every variable moves."""
    import test_curved_ns as ns
    N = 4
    mesh = ns.cavity_mesh(tl, 64)
    cm = mesh.curved(N)
    semi = ns.make_semi(tl, mesh, N, mu=0.001)
    u0 = ns.stirred(tl, cm)
    u_gpu, integ = device_steps(tl, semi, u0, 20, 0.98 * 5 * 0.103, fixed_dt=5e-5)
    assert integ.iter == 20 and integ.t == pytest.approx(20 * 5e-5, rel=1e-13)
    o = ns.oracle_for(oracle_mod, cm, N, mu=0.001)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 20, 0.98 * 5 * 0.103, 0.0, 1e9, fixed_dt=5e-5, nthreads=NTH)
    assert s == 20
    assert np.all(rel_l2(u_gpu, u_cpu) < RTOL), rel_l2(u_gpu, u_cpu)
    assert np.all(rel_l2(u_gpu, u0) > 1e-9)


def _bench():
    """bench.py's workload builders (the same meshes, initial conditions and CFL numbers as the timed runs)."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import bench
    return bench


@pytest.mark.parametrize("icname", ["warped", "blast"])
def test_curvilinear_512_bench_workloads_steps(tl, oracle_mod, icname):
    """The curvilinear throughput workloads at their own size (warped 512 x 512 StructuredMesh, N = 4): the LW
    vortex and the shock-capturing blast with MUSCL subcells, 2 device CFL steps against the oracle."""
    bench = _bench()
    semi = bench.build_semi(tl, 9, 4, "lw", icname, 0)
    u0 = semi.compute_coefficients(0.0)
    cfl = bench.RIEMANN_CFL if icname == "blast" else bench.cfl_for(4)
    u_gpu, integ = device_steps(tl, semi, u0, 2, cfl)
    o = oracle_mod.Oracle(bench.make_mesh(tl, 9, icname), 4)
    if icname == "blast":
        o.set_shock_capturing(True, 0.5, 0.001, True, reconstruction=1)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 2, cfl, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 2 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(u_gpu, u_cpu) < RTOL), rel_l2(u_gpu, u_cpu)
