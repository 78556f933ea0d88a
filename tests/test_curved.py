"""Curvilinear conforming meshes (StructuredMesh{2} with a sinusoidal warp; the same mesh with element
frames turned as on a P4estMesh): the oracle's properties on the CPU, and libtlw's curvilinear volume and
interface kernels against the oracle on the GPU (1e-12 relative L2 per variable, as on TreeMesh)."""
import os

import numpy as np
import pytest

NTH = os.cpu_count() or 1


def warp(xi, eta):
    """[-1, 1]^2 -> [-10, 10]^2 with the interior warped by 5 % of the side, periodic-compatible."""
    X = 10.0 * xi
    Y = 10.0 * eta
    s = np.sin(np.pi * (X + 10.0) / 10.0) * np.sin(np.pi * (Y + 10.0) / 10.0)
    return X + 1.0 * s, Y + 1.0 * s


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def vortex_state(tl, cm, beta=5.0):
    eq = tl.CompressibleEulerEquations2D(1.4)
    v = tl.IsentropicVortex(beta, center=(0.7, -0.4))(cm.xy[0], cm.xy[1], 0.0, eq)
    return np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)


def quad(cm, N, du):
    from trixilw.basis import gauss_lobatto
    _, w = gauss_lobatto(N)
    return np.einsum("ejiv,eji,j,i->v", du.reshape(-1, N + 1, N + 1, 4), cm.jacobian_nodes(), w, w)


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("N", [3, 4, 5])
def test_oracle_curved_free_stream_and_conservation(oracle_mod, tl, N):
    m = tl.StructuredMesh((6, 6), warp)
    cm = m.curved(N)
    o = oracle_mod.Oracle(m, N)
    u = np.tile(np.array([1.0, 0.3, -0.2, 2.5]), cm.n_elements * (N + 1) ** 2)
    assert np.abs(o.rhs(u, 0.0, 0.05)).max() < 1e-12
    u = vortex_state(tl, cm)
    du = o.rhs(u, 0.0, o.max_dt(u, 0.4))
    assert np.all(np.abs(quad(cm, N, du)) < 1e-11)


@pytest.mark.parametrize("N", [3, 4])
def test_oracle_curved_invariant_under_element_rotations(oracle_mod, tl, N):
    m = tl.StructuredMesh((5, 4), warp)
    cm = m.curved(N)
    turns = np.random.default_rng(N).integers(0, 4, cm.n_elements)
    rm = tl.rotate_elements(cm, turns)
    u = vortex_state(tl, cm)
    o, o2 = oracle_mod.Oracle(m, N), oracle_mod.Oracle(rm, N)
    dt = o.max_dt(u, 0.4)
    ur = tl.rotate_state(u, N, turns)
    assert o2.max_dt(ur, 0.4) == pytest.approx(dt, rel=1e-13)
    du = o.rhs(u, 0.0, dt)
    assert np.all(rel_l2(o2.rhs(ur, 0.0, dt), tl.rotate_state(du, N, turns)) < 1e-12)


def test_oracle_curved_vortex_convergence(oracle_mod, tl):
    """Isentropic vortex on the warped mesh, N = 4, t = 1: the error falls at ~N+1 from 16^2 to 32^2."""
    errs = []
    for cells in (16, 32):
        m = tl.StructuredMesh((cells, cells), warp)
        cm = m.curved(4)
        eq = tl.CompressibleEulerEquations2D(1.4)
        ic = tl.IsentropicVortex(5.0)
        v = ic(cm.xy[0], cm.xy[1], 0.0, eq)
        u = np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)
        o = oracle_mod.Oracle(m, 4)
        s, t = o.steps(u, 10 ** 6, 0.4, 0.0, 1.0, nthreads=NTH)
        ve = ic(cm.xy[0], cm.xy[1], 1.0, eq)
        ue = np.ascontiguousarray(np.transpose(ve, (2, 1, 0, 3))).reshape(-1)
        d = (u - ue).reshape(-1, 5, 5, 4)
        from trixilw.basis import gauss_lobatto
        _, w = gauss_lobatto(4)
        errs.append(np.sqrt(np.einsum("ejiv,eji,j,i->v", d * d, cm.jacobian_nodes(), w, w)[0] / cm.area))
    assert np.log2(errs[0] / errs[1]) > 4.4


# ---------------------------------------------------------------------------------------------- GPU
def gpu_rhs(tl, semi, u, dt):
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, 0.0)
    return du


def make_semi(tl, mesh, N, flux=None):
    eq = tl.CompressibleEulerEquations2D(1.4)
    solver = tl.DGSEM(N, flux or tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    return tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, tl.IsentropicVortex(5.0), solver)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [3, 4, 5, 6, 7])
@pytest.mark.parametrize("rotated", [False, True])
def test_gpu_curved_rhs_matches_oracle(oracle_mod, tl, N, rotated):
    from trixilw import _lib
    m = tl.StructuredMesh((6, 5), warp)
    cm = m.curved(N)
    if rotated:
        cm = tl.rotate_elements(cm, np.random.default_rng(N).integers(0, 4, cm.n_elements))
    semi = make_semi(tl, cm, N)
    assert _lib.lib().tlw_curved_colors(semi.handle) >= 2
    u = vortex_state(tl, cm)
    o = oracle_mod.Oracle(cm, N)
    dt = o.max_dt(u, 0.3)
    assert semi.max_dt(u, 0.3) == pytest.approx(dt, rel=1e-13)
    du_cpu = o.rhs(u, 0.0, dt)
    du_gpu = gpu_rhs(tl, semi, u, dt)
    assert np.all(rel_l2(u + dt * du_gpu, u + dt * du_cpu) < 1e-12)
    assert np.all(rel_l2(du_gpu, du_cpu) < 1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("flux,speed", [("rusanov", "davis"), ("hll", "naive")])
def test_gpu_curved_flux_variants(oracle_mod, tl, flux, speed):
    m = tl.StructuredMesh((5, 5), warp)
    cm = m.curved(4)
    f = tl.FluxLaxFriedrichs(max_abs_speed=speed) if flux == "rusanov" else tl.FluxHLL()
    semi = make_semi(tl, cm, 4, f)
    u = vortex_state(tl, cm)
    o = oracle_mod.Oracle(cm, 4, flux_kind=0 if flux == "rusanov" else 1, speed_kind=1 if speed == "davis" else 0)
    dt = o.max_dt(u, 0.3)
    du_gpu = gpu_rhs(tl, semi, u, dt)
    assert np.all(rel_l2(u + dt * du_gpu, u + dt * o.rhs(u, 0.0, dt)) < 1e-12)


@pytest.mark.gpu
def test_gpu_curved_steps_match_oracle(oracle_mod, tl):
    m = tl.StructuredMesh((8, 8), warp)
    cm = tl.rotate_elements(m.curved(4), np.random.default_rng(7).integers(0, 4, 64))
    semi = make_semi(tl, cm, 4)
    u0 = vortex_state(tl, cm)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(9, 0.4, use_graph=True)
    integ.sync_time()
    u_gpu = integ.get_state()
    o = oracle_mod.Oracle(cm, 4)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 9, 0.4, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 9 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(u_gpu, u_cpu) < 1e-12)


# ------------------------------------------------------------------ MDRK on curvilinear meshes (CPU and GPU)
# mdrk_kernel_1! / _2! of src/solvers/dgsem_structured/multi_derivative_2d.jl:82-445: the TreeMesh procedure
# on contravariant fluxes; stage 2 takes the stage state in the volume terms and u^n at the interfaces.
@pytest.mark.parametrize("N", [3, 4])
def test_oracle_curved_mdrk_free_stream_conservation_rotations(oracle_mod, tl, N):
    m = tl.StructuredMesh((5, 4), warp)
    cm = m.curved(N)
    o = oracle_mod.Oracle(cm, N)
    u = np.tile(np.array([1.0, 0.3, -0.2, 2.5]), cm.n_elements * (N + 1) ** 2)
    s_, _ = o.steps(u, 3, 0.3, 0.0, 1e9, kind=1)
    assert s_ == 3 and np.abs(u - np.tile(np.array([1.0, 0.3, -0.2, 2.5]), cm.n_elements * (N + 1) ** 2)).max() < 1e-12
    u0 = vortex_state(tl, cm)
    mass0 = quad(cm, N, u0)
    u1 = u0.copy()
    o.steps(u1, 4, 0.3, 0.0, 1e9, kind=1)
    np.testing.assert_allclose(quad(cm, N, u1), mass0, rtol=1e-12)
    turns = np.random.default_rng(N).integers(0, 4, cm.n_elements)
    o2 = oracle_mod.Oracle(tl.rotate_elements(cm, turns), N)
    ur = tl.rotate_state(u0, N, turns)
    o2.steps(ur, 4, 0.3, 0.0, 1e9, kind=1)
    assert np.all(rel_l2(ur, tl.rotate_state(u1, N, turns)) < 1e-12)


def make_mdrk_semi(tl, mesh, N, bc=None):
    eq = tl.CompressibleEulerEquations2D(1.4)
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.MDRK()))
    kw = {} if bc is None else {"boundary_conditions": bc}
    return tl.SemidiscretizationHyperbolic(mesh, tl.MDRK(), eq, tl.IsentropicVortex(5.0), solver, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("N,rotated", [(3, False), (4, False), (4, True), (5, True)])
def test_gpu_curved_mdrk_matches_oracle(oracle_mod, tl, N, rotated):
    m = tl.StructuredMesh((6, 5), warp)
    cm = m.curved(N)
    if rotated:
        cm = tl.rotate_elements(cm, np.random.default_rng(N + 20).integers(0, 4, cm.n_elements))
    semi = make_mdrk_semi(tl, cm, N)
    u = vortex_state(tl, cm)
    o = oracle_mod.Oracle(cm, N)
    dt = o.max_dt(u, 0.3)
    semi.cache["dt"][0] = dt
    # the two stages through the rhs entry points
    d1_gpu = np.empty_like(u)
    tl.rhs_mdrk1(d1_gpu, u, semi, 0.0)
    d1_cpu = o.rhs(u, 0.0, dt, kind=1)
    assert np.all(rel_l2(u + dt * d1_gpu, u + dt * d1_cpu) < 1e-12)
    us = u + dt * d1_cpu
    d2_gpu = np.empty_like(u)
    tl.rhs_mdrk2(d2_gpu, u, semi, 0.0, us)
    d2_cpu = o.rhs(u, 0.0, dt, kind=2, us=us)
    assert np.all(rel_l2(u + dt * d2_gpu, u + dt * d2_cpu) < 1e-12)
    # whole MDRK steps on the device
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.MDRK(), (0.0, 1e9)))
    integ.set_state(u, 0.0)
    integ.step(7, 0.3, use_graph=True)
    integ.sync_time()
    u_cpu = u.copy()
    s, t = o.steps(u_cpu, 7, 0.3, 0.0, 1e9, kind=1, nthreads=NTH)
    assert s == integ.iter == 7 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-12)


@pytest.mark.gpu
def test_gpu_curved_mdrk_with_slip_walls(oracle_mod, tl):
    """MDRK on the warped box with slip walls on all sides (the walls take the stage-1 traces as they are)."""
    def box_warp(xi, eta):
        X, Y = 0.5 * (xi + 1.0), 0.5 * (eta + 1.0)
        s = 0.05 * np.sin(np.pi * X) * np.sin(np.pi * Y)
        return X + s, Y + s
    N = 4
    cm = tl.StructuredMesh((6, 6), box_warp, periodicity=False).curved(N)
    bc = {"x_neg": tl.boundary_condition_slip_wall_vertical, "x_pos": tl.boundary_condition_slip_wall_vertical,
          "y_neg": tl.boundary_condition_slip_wall_horizontal, "y_pos": tl.boundary_condition_slip_wall_horizontal}
    semi = make_mdrk_semi(tl, cm, N, bc)
    eq = tl.CompressibleEulerEquations2D(1.4)
    x, y = cm.xy
    rho = 1.0 + 0.2 * np.exp(-20 * ((x - 0.6) ** 2 + (y - 0.45) ** 2))
    U = eq.prim2cons(rho, 0.1 * np.sin(np.pi * x), -0.1 * np.sin(np.pi * y), 1.0 + 0 * x)
    u = np.ascontiguousarray(np.transpose(U, (2, 1, 0, 3))).reshape(-1)
    o = oracle_mod.Oracle(cm, N)
    o.set_curved_boundaries(cm.boundary_elements, cm.boundary_faces,
                            np.repeat(np.array([1, 1, 2, 2], dtype=np.int32), cm.n_boundaries_per_direction))
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.MDRK(), (0.0, 1e9)))
    integ.set_state(u, 0.0)
    integ.step(6, 0.3, use_graph=True)
    integ.sync_time()
    u_cpu = u.copy()
    s, t = o.steps(u_cpu, 6, 0.3, 0.0, 1e9, kind=1, nthreads=NTH)
    assert s == integ.iter == 6 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(integ.get_state(), u_cpu) < 1e-12)
    np.testing.assert_allclose(quad(cm, N, u_cpu)[0], quad(cm, N, u)[0], rtol=1e-12)


# ------------------------------------------------- time-averaged Dirichlet boundaries on curvilinear meshes
def _box_warp(xi, eta):
    X, Y = 0.5 * (xi + 1.0), 0.5 * (eta + 1.0)
    s = 0.05 * np.sin(np.pi * X) * np.sin(np.pi * Y)
    return X + s, Y + s


def _dirichlet_setup(tl, oracle_mod, N, td):
    """The warped unit box: Dirichlet data (a moving density wave, time-dependent) on x_neg / x_pos, slip walls
    on y_neg / y_pos (every component of the state nonzero, so that relative errors are meaningful)."""
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.StructuredMesh((6, 6), _box_warp, periodicity=False)
    cm = mesh.curved(N)
    ic = tl.DensityWave(amplitude=0.3, v=(0.4, 0.15), p=1.0, k=1.0)
    bc = {"x_neg": tl.BoundaryConditionDirichlet(ic), "x_pos": tl.BoundaryConditionDirichlet(ic),
          "y_neg": tl.boundary_condition_slip_wall_horizontal, "y_pos": tl.boundary_condition_slip_wall_horizontal}
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tdo))
    semi = tl.SemidiscretizationHyperbolic(cm, tdo, eq, ic, solver, boundary_conditions=bc)
    o = oracle_mod.Oracle(cm, N)
    o.set_curved_boundaries(cm.boundary_elements, cm.boundary_faces,
                            np.repeat(np.array([0, 0, 2, 2], dtype=np.int32), cm.n_boundaries_per_direction))
    u = np.ascontiguousarray(np.transpose(ic(cm.xy[0], cm.xy[1], 0.0, eq), (2, 1, 0, 3))).reshape(-1)
    return eq, cm, ic, semi, o, u


def _oracle_boundary_data(cm, N, ic, eq, t, dt, scaling):
    from trixilw.basis import gauss_lobatto
    nodes, _ = gauss_lobatto(N)
    xy = cm.boundary_node_coordinates(N)
    levels = np.empty((cm.n_boundaries, N + 1, N + 1, 4))
    for q in range(N + 1):
        levels[:, :, q, :] = np.transpose(ic(xy[0], xy[1], t + 0.5 * scaling * dt * (nodes[q] + 1.0), eq), (1, 0, 2))
    now = np.transpose(ic(xy[0], xy[1], t, eq), (1, 0, 2))
    return np.ascontiguousarray(levels), np.ascontiguousarray(now)


@pytest.mark.gpu
@pytest.mark.parametrize("N,td", [(3, "lw"), (4, "lw"), (4, "mdrk")])
def test_gpu_curved_dirichlet_matches_oracle(oracle_mod, tl, N, td):
    eq, cm, ic, semi, o, u = _dirichlet_setup(tl, oracle_mod, N, td)
    t, dt = 0.13, 0.4 * o.max_dt(u, 0.3) / 0.3
    semi.cache["dt"][0] = dt
    if td == "lw":
        o.set_boundary_data(*_oracle_boundary_data(cm, N, ic, eq, t, dt, 1.0))
        du = np.empty_like(u)
        tl.rhs(du, u, semi, t)
        assert np.all(rel_l2(u + dt * du, u + dt * o.rhs(u, t, dt)) < 1e-12)
    else:
        o.set_boundary_data(*_oracle_boundary_data(cm, N, ic, eq, t, dt, 0.5))
        d1 = np.empty_like(u)
        tl.rhs_mdrk1(d1, u, semi, t)
        d1_cpu = o.rhs(u, t, dt, kind=1)
        assert np.all(rel_l2(u + dt * d1, u + dt * d1_cpu) < 1e-12)
        o.set_boundary_data(*_oracle_boundary_data(cm, N, ic, eq, t, dt, 1.0))
        us = u + dt * d1_cpu
        d2 = np.empty_like(u)
        tl.rhs_mdrk2(d2, u, semi, t, us)
        assert np.all(rel_l2(u + dt * d2, u + dt * o.rhs(u, t, dt, kind=2, us=us)) < 1e-12)


@pytest.mark.gpu
def test_gpu_curved_dirichlet_solve_converges_to_the_wave(tl):
    """solve_lwfr on the warped box with the moving density wave as Dirichlet data at x and slip walls at y
    (the wave moves along x, so the walls are exact): the error against the exact wave stays at the level of
    the discretisation."""
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.StructuredMesh((8, 8), _box_warp, periodicity=False)
    ic = tl.DensityWave(amplitude=0.3, v=(0.4, 0.0), p=1.0, k=1.0)
    ic_x = lambda x, y, t, e: ic(x, 0 * y, t, e)   # a wave in x only: rho(x - 0.4 t)
    bc = {"x_neg": tl.BoundaryConditionDirichlet(ic_x), "x_pos": tl.BoundaryConditionDirichlet(ic_x),
          "y_neg": tl.boundary_condition_slip_wall_horizontal, "y_pos": tl.boundary_condition_slip_wall_horizontal}
    solver = tl.DGSEM(4, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    semi = tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, ic_x, solver, boundary_conditions=bc)
    sol = tl.solve_lwfr(tl.semidiscretize(semi, tl.LW(), (0.0, 0.5)), (), 0.0, None,
                        time_step_computation=tl.CFLBased(0.98 * 5 * 0.103))
    l2, linf = tl.l2_linf_errors(semi, sol.u[-1], 0.5)
    assert sol.t[-1] == pytest.approx(0.5) and l2[0] < 2e-4
