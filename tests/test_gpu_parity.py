"""GPU parity tests: libtlw (CUDA, through the C ABI) against the oracle and the golden fixtures.

Tolerances. The bar is 1e-12 relative L2 per variable of the state after one step (u + dt du), which is
what "within 1e-12 relative L2 per step" measures. du itself is also compared, per variable, at 1e-12 on
small meshes; on large meshes du is ~0 over most of the free stream and both implementations leave
roundoff of ~1e-13 * J^-1 there, so the du bound is 1e-11 (it grows with the inverse Jacobian).
Multi-step runs: 1e-12 after ~10 steps, 1e-10 after a full t_end = 1 run.
"""
import os

import numpy as np
import pytest

import golden_cases

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def faces_from_full(X, n, E, F=None):
    """Face traces [e, face, l, v] of a full element array [e, j, i, v] (U) or of F [e, j, i, d, v]."""
    out = np.empty((E, 4, n, 4))
    if F is None:
        out[:, 0] = X[:, :, 0]
        out[:, 1] = X[:, :, n - 1]
        out[:, 2] = X[:, 0, :]
        out[:, 3] = X[:, n - 1, :]
    else:
        out[:, 0] = F[:, :, 0, 0]
        out[:, 1] = F[:, :, n - 1, 0]
        out[:, 2] = F[:, 0, :, 1]
        out[:, 3] = F[:, n - 1, :, 1]
    return out


def make_semi(tl, mesh, N, ic, td="lw", flux=None, bc=None, sc=False):
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    vi = tl.VolumeIntegralFR(tdo)
    if sc:
        vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5), vi)
    solver = tl.DGSEM(N, flux or tl.flux_lax_friedrichs, vi)
    kw = {}
    if mesh.n_boundaries:
        kw["boundary_conditions"] = bc or tl.BoundaryConditionDirichlet(ic)
    return tl.SemidiscretizationHyperbolic(mesh, tdo, eq, ic, solver, **kw)


@pytest.mark.parametrize("name", list(golden_cases.CASES))
def test_golden_cases(tl, name):
    from trixilw import _lib
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    td, N, eq, mesh, ic, u = golden_cases.setup(name, tl)
    n = N + 1
    E = mesh.n_elements
    sc = name in golden_cases.SHOCK_CAPTURING
    semi = make_semi(tl, mesh, N, ic, td, sc=sc)
    semi.cache["dt"][0] = float(ref["dt"][0])
    np.testing.assert_array_equal(u, ref["u"])
    du = np.empty_like(u)
    if td == "lw":
        tl.rhs(du, u, semi, 0.0)
        assert np.all(rel_l2(du, ref["du"]) < RTOL), rel_l2(du, ref["du"])
    else:
        tl.rhs_mdrk1(du, u, semi, 0.0)
        assert np.all(rel_l2(du, ref["du1"]) < RTOL)
        U2 = semi.get_cache(_lib.TLW_CACHE_U2)
        F2 = semi.get_cache(_lib.TLW_CACHE_F2)
        assert np.all(rel_l2(U2, ref["U2"]) < RTOL)
        assert np.all(rel_l2(F2, ref["F2"]) < RTOL)
        us = u + float(ref["dt"][0]) * du
        du2 = np.empty_like(u)
        tl.rhs_mdrk2(du2, u, semi, 0.0, us)
        assert np.all(rel_l2(du2, ref["du2"]) < RTOL), rel_l2(du2, ref["du2"])
    tU = semi.get_cache(_lib.TLW_CACHE_U_TRACES).reshape(E, 4, n, 4)
    tF = semi.get_cache(_lib.TLW_CACHE_F_TRACES).reshape(E, 4, n, 4)
    U = ref["U"].reshape(E, n, n, 4)
    F = ref["F"].reshape(E, n, n, 2, 4)
    np.testing.assert_allclose(tU, faces_from_full(U, n, E), rtol=0, atol=1e-13 * np.abs(U).max())
    np.testing.assert_allclose(tF, faces_from_full(None, n, E, F), rtol=0, atol=1e-12 * np.abs(F).max())
    if sc:
        alpha = semi.get_cache(_lib.TLW_CACHE_ALPHA)
        np.testing.assert_allclose(alpha, ref["alpha"], rtol=1e-10, atol=1e-14)
        fnl = semi.get_cache(_lib.TLW_CACHE_FN_LOW)
        np.testing.assert_allclose(fnl, ref["fn_low"], rtol=0, atol=1e-12 * np.abs(ref["fn_low"]).max())


@pytest.mark.parametrize("td,N", [("lw", 4), ("lw", 3), ("mdrk", 4)])
def test_shock_capturing_riemann_steps(tl, oracle_mod, td, N):
    """Four-quadrant Riemann problem with HG blending (alpha_max = 0.5) and first-order subcells,
    Dirichlet boundaries: 20 device steps (indicator fused into the CFL pass, CUDA graphs) vs the oracle."""
    mesh = tl.TreeMesh((0.0, 0.0), (1.0, 1.0), 4, periodicity=False)
    ic = tl.FourQuadrantRiemann()
    semi = make_semi(tl, mesh, N, ic, td, sc=True)
    u0 = semi.compute_coefficients(0.0)
    semi._prepare_boundaries(0.0, 0.0, 1.0)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(20, 0.15)
    u_gpu = integ.get_state()
    o = oracle_mod.Oracle(mesh, N)
    o.set_shock_capturing(True, 0.5, 0.001, True)
    lv, nw = golden_cases.boundary_data(mesh, N, ic, semi.equations)
    o.set_boundary_data(lv, nw)
    u_cpu = u0.copy()
    o.steps(u_cpu, 20, 0.15, 0.0, 1e9, kind=0 if td == "lw" else 1, nthreads=os.cpu_count() or 1)
    assert np.all(rel_l2(u_gpu, u_cpu) < 1e-11), rel_l2(u_gpu, u_cpu)


def test_shock_capturing_periodic_conservation(tl):
    """Periodic density square wave with shock capturing: alpha > 0 somewhere, discrete conservation holds."""
    from trixilw import _lib
    from trixilw.basis import gauss_lobatto
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((-1.0, -1.0), (1.0, 1.0), 5)

    def square(x, y, t, eq):
        rho = np.where((np.abs(x) < 0.4) & (np.abs(y) < 0.4), 2.0, 1.0)
        return eq.prim2cons(rho, 0.5, 0.3, 1.0)

    semi = make_semi(tl, mesh, 4, square, sc=True)
    u = semi.compute_coefficients(0.0)
    semi.cache["dt"][0] = semi.max_dt(u, 0.15)
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    assert semi.get_cache(_lib.TLW_CACHE_ALPHA).max() > 0.0
    _, w = gauss_lobatto(4)
    d = du.reshape(mesh.n_elements, 5, 5, 4)
    total = np.einsum("ejiv,j,i->v", d, w, w)
    scale = np.einsum("ejiv,j,i->v", np.abs(d), w, w)
    assert np.all(np.abs(total) <= 1e-12 * scale)


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_rhs_all_degrees(tl, oracle_mod, N):
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    ic = tl.IsentropicVortex(4.5, center=(-1.0, 2.0))
    semi = make_semi(tl, mesh, N, ic)
    u = semi.compute_coefficients(0.0)
    u = u * (1 + 1e-3 * np.random.default_rng(N).standard_normal(u.shape))
    o = oracle_mod.Oracle(mesh, N)
    dt = o.max_dt(u, 0.3)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    assert np.all(rel_l2(du, o.rhs(u, 0.0, dt)) < RTOL)


@pytest.mark.parametrize("flux,speed", [("rusanov", "davis"), ("hll", "naive")])
@pytest.mark.parametrize("N", [3, 4])
def test_rhs_flux_variants(tl, oracle_mod, flux, speed, N):
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    ic = tl.IsentropicVortex(5.0, center=(0.3, 0.2))
    f = tl.FluxLaxFriedrichs(speed) if flux == "rusanov" else tl.FluxHLL()
    semi = make_semi(tl, mesh, N, ic, flux=f)
    u = semi.compute_coefficients(0.0)
    o = oracle_mod.Oracle(mesh, N, flux_kind=0 if flux == "rusanov" else 1, speed_kind=1 if speed == "davis" else 0)
    dt = o.max_dt(u, 0.4)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    assert np.all(rel_l2(du, o.rhs(u, 0.0, dt)) < RTOL)


def test_max_dt_matches_oracle(tl, oracle_mod):
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 4)
    ic = tl.IsentropicVortex(5.0)
    semi = make_semi(tl, mesh, 4, ic)
    u = semi.compute_coefficients(0.0)
    o = oracle_mod.Oracle(mesh, 4)
    assert semi.max_dt(u, 0.5047) == pytest.approx(o.max_dt(u, 0.5047), rel=1e-15)


@pytest.mark.parametrize("td", ["lw", "mdrk"])
@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_device_steps_match_oracle(tl, oracle_mod, td, N):
    """Device CFL steps on a periodic mesh (the element-centric surface pass and the CFL slots, whose face-node
    maxima are reduced by shuffles for N = 1, 2, 4 and through shared memory otherwise) against the oracle."""
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 4)
    ic = tl.IsentropicVortex(5.0)
    semi = make_semi(tl, mesh, N, ic, td)
    u0 = semi.compute_coefficients(0.0)
    cfl = 0.98 * (N + 1) * 0.103 if 3 <= N <= 4 else 0.4 if N > 4 else 0.1
    upd = tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9))
    integ = tl.LWIntegrator(upd)
    integ.set_state(u0, 0.0)
    integ.step(7, cfl, use_graph=True)      # odd count: exercises the 2-step graph and a single step
    integ.step(6, cfl, use_graph=False)
    integ.sync_time()
    u_gpu = integ.get_state()
    o = oracle_mod.Oracle(mesh, N)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 13, cfl, 0.0, 1e9, kind=0 if td == "lw" else 1, nthreads=os.cpu_count() or 1)
    assert s == 13 and integ.iter == 13
    assert integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(u_gpu, u_cpu) < 1e-12)


def test_graph_and_stream_paths_bitwise_equal(tl):
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 4)
    semi = make_semi(tl, mesh, 4, tl.IsentropicVortex(5.0))
    u0 = semi.compute_coefficients(0.0)
    outs = []
    for g in (True, False):
        integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
        integ.set_state(u0, 0.0)
        integ.step(5, 0.5, use_graph=g)
        outs.append(integ.get_state())
    np.testing.assert_array_equal(outs[0], outs[1])


def test_config1_vortex_run(tl, oracle_mod):
    """Isentropic vortex, periodic [-10,10]^2, 16x16 elements, N=4, Rusanov, CFL 0.98 of the LW limit,
    t_end = 1: GPU state vs oracle state, and the discretisation error vs the exact solution."""
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 4)
    ic = tl.IsentropicVortex(5.0)
    semi = make_semi(tl, mesh, 4, ic)
    cfl = tl.trixi2lw(0.98, semi.solver)
    sol = tl.solve_lwfr(tl.semidiscretize(semi, tl.LW(), (0.0, 1.0)), (), 0.0, None, tl.CFLBased(cfl))
    assert sol.t[0] == pytest.approx(1.0, abs=1e-14)
    u_cpu = semi.compute_coefficients(0.0)
    o = oracle_mod.Oracle(mesh, 4)
    s, t = o.steps(u_cpu, 10 ** 6, cfl, 0.0, 1.0, nthreads=os.cpu_count() or 1)
    assert s == sol.stats.naccept
    assert np.all(rel_l2(sol.u[0], u_cpu) < 1e-10)
    l2_gpu, _ = tl.l2_linf_errors(semi, sol.u[0], 1.0)
    l2_cpu, _ = tl.l2_linf_errors(semi, u_cpu, 1.0)
    np.testing.assert_allclose(l2_gpu, l2_cpu, rtol=1e-8)
    assert l2_gpu[0] < 2e-3


def test_dirichlet_riemann_steps(tl, oracle_mod):
    mesh = tl.TreeMesh((0.0, 0.0), (1.0, 1.0), 4, periodicity=False)
    ic = tl.FourQuadrantRiemann()
    semi = make_semi(tl, mesh, 4, ic)
    u0 = semi.compute_coefficients(0.0)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    semi._prepare_boundaries(0.0, 0.0, 1.0)
    integ.set_state(u0, 0.0)
    integ.step(3, 0.2)
    u_gpu = integ.get_state()
    o = oracle_mod.Oracle(mesh, 4)
    lv, nw = golden_cases.boundary_data(mesh, 4, ic, semi.equations)
    o.set_boundary_data(lv, nw)
    u_cpu = u0.copy()
    o.steps(u_cpu, 3, 0.2, 0.0, 1e9)
    assert np.all(rel_l2(u_gpu, u_cpu) < 1e-12)


def test_domain_error_and_recovery(tl):
    mesh = tl.TreeMesh((-1.0, -1.0), (1.0, 1.0), 2)
    semi = make_semi(tl, mesh, 3, tl.ConstantState(1.0, 0.1, 0.1, 1.0))
    u = semi.compute_coefficients(0.0)
    semi.cache["dt"][0] = 1e-3
    bad = u.reshape(-1, 4).copy()
    bad[0, 3] = -1.0
    du = np.empty_like(u)
    with pytest.raises(tl.DomainError):
        tl.rhs(du, bad.reshape(-1), semi, 0.0)
    tl.rhs(du, u, semi, 0.0)    # the handle stays usable; the status was cleared
    assert np.abs(du).max() < 1e-13


@pytest.mark.parametrize("N", [3, 4, 5])
def test_large_mesh_rhs(tl, oracle_mod, N):
    """256^2 elements: one rhs against the (multithreaded) oracle."""
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 8)
    semi = make_semi(tl, mesh, N, tl.IsentropicVortex(5.0, center=(0.1, -0.2)))
    u = semi.compute_coefficients(0.0)
    o = oracle_mod.Oracle(mesh, N)
    dt = o.max_dt(u, 0.4)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    ref = o.rhs(u, 0.0, dt, nthreads=os.cpu_count() or 1)
    assert np.all(rel_l2(u + dt * du, u + dt * ref) < RTOL)
    assert np.all(rel_l2(du, ref) < 1e-11)


def test_full_size_properties(tl):
    """512^2 elements, N=4 (the throughput workload): size-independent properties of one rhs -
    free-stream preservation and discrete conservation on the periodic mesh."""
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 9)
    semi = make_semi(tl, mesh, 4, tl.ConstantState(1.2, 0.7, -0.3, 1.5))
    u = semi.compute_coefficients(0.0)
    semi.cache["dt"][0] = semi.max_dt(u, 0.5)
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    assert np.abs(du).max() < 1e-11
    semi2 = make_semi(tl, mesh, 4, tl.IsentropicVortex(5.0))
    u = semi2.compute_coefficients(0.0)
    semi2.cache["dt"][0] = semi2.max_dt(u, 0.5)
    tl.rhs(du, u, semi2, 0.0)
    from trixilw.basis import gauss_lobatto
    _, w = gauss_lobatto(4)
    d = du.reshape(mesh.n_elements, 5, 5, 4)
    total = np.einsum("ejiv,j,i->v", d, w, w)
    scale = np.einsum("ejiv,j,i->v", np.abs(d), w, w)
    # the sum runs over 6.5 M nodes: its own rounding is ~1e-13 of the absolute sum
    assert np.all(np.abs(total) <= 1e-10 * scale)


@pytest.mark.parametrize("offset", [0, 1, 2, 3])
def test_rhs_with_device_arrays_at_any_alignment(tl, offset):
    """tlw_rhs and tlw_max_dt on device arrays that start 8 offset bytes into an allocation: used in place when
    32-byte aligned, copied through the handle's buffers otherwise; the results equal the host-array call."""
    import ctypes

    import torch
    from trixilw import _lib
    L = _lib.lib()
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 4)
    semi = make_semi(tl, mesh, 4, tl.IsentropicVortex(5.0, center=(0.2, 0.1)), "mdrk")
    u = semi.compute_coefficients(0.0)
    dt = semi.max_dt(u, 0.4)
    semi.cache["dt"][0] = dt
    du_h = np.empty_like(u)
    tl.rhs_mdrk1(du_h, u, semi, 0.0)
    us = u + 0.5 * dt * du_h
    du2_h = np.empty_like(u)
    tl.rhs_mdrk2(du2_h, u, semi, 0.0, us)
    n = u.size
    bufs = [torch.zeros(n + 4, dtype=torch.float64, device="cuda") for _ in range(4)]
    d_u, d_us, d_du, d_du2 = (b[offset:offset + n] for b in bufs)
    d_u.copy_(torch.from_numpy(u))
    d_us.copy_(torch.from_numpy(us))
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    _lib.check(semi.handle, L.tlw_rhs(semi.handle, _lib.TLW_STAGE_MDRK1, p(d_du), p(d_u), None, 0.0, dt,
                                      _lib.TLW_WHERE_DEVICE))
    _lib.check(semi.handle, L.tlw_rhs(semi.handle, _lib.TLW_STAGE_MDRK2, p(d_du2), p(d_u), p(d_us), 0.0, dt,
                                      _lib.TLW_WHERE_DEVICE))
    dt_d = ctypes.c_double()
    _lib.check(semi.handle, L.tlw_max_dt(semi.handle, p(d_u), _lib.TLW_WHERE_DEVICE, 0.4, ctypes.byref(dt_d)))
    _lib.check(semi.handle, L.tlw_synchronize(semi.handle))
    np.testing.assert_array_equal(d_du.cpu().numpy(), du_h)
    np.testing.assert_array_equal(d_du2.cpu().numpy(), du2_h)
    assert dt_d.value == dt
