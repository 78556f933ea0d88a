"""Source terms (SemidiscretizationHyperbolic(...; source_terms = source_terms_convergence_test), the reference's
examples/tree_2d_dgsem/elixir_euler_source_terms.jl): calc_source and its time-derivative stencils inside every LW
volume kernel (src/solvers/dgsem_tree/dg_2d.jl:89-175, used at :425-489, :551-668, :732-911, :979-1233) and in the
MDRK stages (multi_derivative_2d.jl:321-400, :484-550).

CPU: the host form of Trixi's source_terms_convergence_test is pinned against the Euler residual of the
manufactured solution (central differences); the oracle with source terms converges at the scheme's order on the
manufactured solution (wrong source terms leave an O(1) error). GPU: one rhs of every depth (N = 1..7) and both
MDRK stages against the oracle, device steps against oracle steps, and the elixir's convergence test."""
import os

import numpy as np
import pytest

NTH = os.cpu_count() or 1


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def state(tl, mesh, N, t, eq):
    xy = mesh.node_coordinates(N)
    u = tl.initial_condition_convergence_test(xy[0], xy[1], t, eq)
    return np.ascontiguousarray(np.transpose(u, (2, 1, 0, 3))).reshape(-1)


def xnode(mesh, N):
    return np.ascontiguousarray(np.transpose(mesh.node_coordinates(N), (3, 2, 1, 0)))


# ---------------------------------------------------------------------------------------------- CPU
def test_host_source_is_the_euler_residual_of_the_manufactured_solution(tl):
    """d_t u + d_x f(u) + d_y g(u) = s for u = initial_condition_convergence_test, by central differences."""
    eq = tl.CompressibleEulerEquations2D(1.4)
    rng = np.random.default_rng(3)
    x, y, t = rng.uniform(0.0, 2.0, 50), rng.uniform(0.0, 2.0, 50), rng.uniform(0.0, 1.0, 50)
    h = 1e-5

    def flux(u, d):
        rho, v1, v2, p = eq.cons2prim(u)
        vn = v1 if d == 0 else v2
        return np.stack([u[..., 1 + d], u[..., 1] * vn + (p if d == 0 else 0.0),
                         u[..., 2] * vn + (p if d == 1 else 0.0), (u[..., 3] + p) * vn], axis=-1)

    ic = tl.initial_condition_convergence_test
    res = ((ic(x, y, t + h, eq) - ic(x, y, t - h, eq))
           + (flux(ic(x + h, y, t, eq), 0) - flux(ic(x - h, y, t, eq), 0))
           + (flux(ic(x, y + h, t, eq), 1) - flux(ic(x, y - h, t, eq), 1))) / (2 * h)
    s = tl.source_terms_convergence_test(None, x, y, t, eq)
    assert np.max(np.abs(res - s)) < 1e-8 * np.max(np.abs(s))


@pytest.mark.parametrize("kind", [0, 1])
def test_oracle_with_source_terms_converges(tl, oracle_mod, kind):
    eq = tl.CompressibleEulerEquations2D(1.4)
    N = 3
    errs = []
    for level in (2, 3, 4):
        mesh = tl.TreeMesh((0.0, 0.0), (2.0, 2.0), level)
        u = state(tl, mesh, N, 0.0, eq)
        o = oracle_mod.Oracle(mesh, N)
        o.set_source(1, xnode(mesh, N))
        _, t = o.steps(u, 100000, 0.2, 0.0, 0.4, kind=kind, nthreads=NTH)
        assert t == pytest.approx(0.4, abs=1e-14)
        errs.append(np.sqrt(np.mean((u - state(tl, mesh, N, t, eq)) ** 2)))
    orders = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert orders[0] > 3.0 and orders[1] > 3.5, orders   # N + 1 = 4 once resolved


def test_oracle_without_source_terms_misses_the_manufactured_solution(tl, oracle_mod):
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((0.0, 0.0), (2.0, 2.0), 3)
    u = state(tl, mesh, 3, 0.0, eq)
    _, t = oracle_mod.Oracle(mesh, 3).steps(u, 100000, 0.2, 0.0, 0.4, kind=0, nthreads=NTH)
    assert np.sqrt(np.mean((u - state(tl, mesh, 3, t, eq)) ** 2)) > 1e-3


# ---------------------------------------------------------------------------------------------- GPU
def make_semi(tl, mesh, N, td="lw"):
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tdo))
    return tl.SemidiscretizationHyperbolic(mesh, tdo, eq, tl.initial_condition_convergence_test, solver,
                                           source_terms=tl.source_terms_convergence_test)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_gpu_rhs_with_source_terms_matches_oracle(tl, oracle_mod, N):
    mesh = tl.TreeMesh((0.0, 0.0), (2.0, 2.0), 3)
    semi = make_semi(tl, mesh, N)
    u = semi.compute_coefficients(0.0)
    u = u * (1 + 1e-3 * np.random.default_rng(N).standard_normal(u.shape))
    o = oracle_mod.Oracle(mesh, N)
    o.set_source(1, xnode(mesh, N))
    t, dt = 0.3, 0.5 * o.max_dt(u, 0.2)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, t)
    ref = o.rhs(u, t, dt, nthreads=NTH)
    assert np.all(rel_l2(du, ref) < 1e-12), rel_l2(du, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [3, 4])
def test_gpu_mdrk_stages_with_source_terms_match_oracle(tl, oracle_mod, N):
    mesh = tl.TreeMesh((0.0, 0.0), (2.0, 2.0), 3)
    semi = make_semi(tl, mesh, N, "mdrk")
    u = semi.compute_coefficients(0.0)
    u = u * (1 + 1e-3 * np.random.default_rng(10 + N).standard_normal(u.shape))
    o = oracle_mod.Oracle(mesh, N)
    o.set_source(1, xnode(mesh, N))
    t, dt = 0.2, 0.5 * o.max_dt(u, 0.2)
    semi.cache["dt"][0] = dt
    du1 = np.empty_like(u)
    tl.rhs_mdrk1(du1, u, semi, t)
    ref1 = o.rhs(u, t, dt, kind=1, nthreads=NTH)
    assert np.all(rel_l2(du1, ref1) < 1e-12), rel_l2(du1, ref1)
    us = u + dt * ref1
    du2 = np.empty_like(u)
    tl.rhs_mdrk2(du2, u, semi, t, us)
    ref2 = o.rhs(u, t, dt, kind=2, us=us, nthreads=NTH)
    assert np.all(rel_l2(du2, ref2) < 1e-12), rel_l2(du2, ref2)


@pytest.mark.gpu
@pytest.mark.parametrize("td,N", [("lw", 4), ("lw", 3), ("mdrk", 4)])
def test_gpu_steps_with_source_terms_match_oracle(tl, oracle_mod, td, N):
    """Device CFL steps (the source at the device time of each step, CUDA graphs) against the oracle's steps."""
    mesh = tl.TreeMesh((0.0, 0.0), (2.0, 2.0), 4)
    semi = make_semi(tl, mesh, N, td)
    u0 = semi.compute_coefficients(0.0)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(12, 0.2, use_graph=True)
    integ.sync_time()
    o = oracle_mod.Oracle(mesh, N)
    o.set_source(1, xnode(mesh, N))
    u = u0.copy()
    s, t = o.steps(u, 12, 0.2, 0.0, 1e9, kind=0 if td == "lw" else 1, nthreads=NTH)
    assert s == integ.iter == 12 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(integ.get_state(), u) < 1e-12)


@pytest.mark.gpu
def test_gpu_elixir_euler_source_terms_converges(tl):
    """The reference's elixir_euler_source_terms.jl setup ([0, 2]^2, N = 4, CFL 0.2) on levels 3..5 to t = 0.5:
    the error against the manufactured solution falls at the scheme's order."""
    eq = tl.CompressibleEulerEquations2D(1.4)
    errs = []
    for level in (3, 4, 5):
        mesh = tl.TreeMesh((0.0, 0.0), (2.0, 2.0), level)
        semi = make_semi(tl, mesh, 4)
        integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 0.5)))
        integ.set_state(semi.compute_coefficients(0.0), 0.0)
        integ.step(2000, 0.2)   # (past t_end the captured steps take dt = 0)
        integ.sync_time()
        assert integ.t == pytest.approx(0.5, abs=1e-14)
        errs.append(np.sqrt(np.mean((integ.get_state() - semi.compute_coefficients(integ.t)) ** 2)))
    orders = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(orders > 3.5), (errs, orders)


# ------------------------------------------------------------------------- curvilinear (StructuredMesh)
def warp2(xi, eta):
    """[-1, 1]^2 -> [0, 2]^2 with the interior warped by 5 % of the side (periodic-compatible)."""
    X, Y = 1.0 + xi, 1.0 + eta
    s = np.sin(np.pi * X) * np.sin(np.pi * Y)
    return X + 0.05 * s, Y + 0.05 * s


def curved_state(tl, mesh, N, t, eq):
    xy = mesh.curved(N).xy
    u = tl.initial_condition_convergence_test(xy[0], xy[1], t, eq)
    return np.ascontiguousarray(np.transpose(u, (2, 1, 0, 3))).reshape(-1)


def curved_xnode(mesh, N):
    return np.ascontiguousarray(np.transpose(mesh.curved(N).xy, (3, 2, 1, 0)))


def test_curved_oracle_with_source_terms_converges(tl, oracle_mod):
    """The reference's structured kernels with the source (elixir_euler_source_terms_parallelogram.jl's kind of
    setup on a warped periodic mesh): LW converges at order 4 (N = 4)."""
    eq = tl.CompressibleEulerEquations2D(1.4)
    N = 4
    errs = []
    for cells in (4, 8, 16):
        mesh = tl.StructuredMesh((cells, cells), warp2)
        u = curved_state(tl, mesh, N, 0.0, eq)
        o = oracle_mod.Oracle(mesh, N)
        o.set_source(1, curved_xnode(mesh, N))
        _, t = o.steps(u, 100000, 0.2, 0.0, 0.4, kind=0, nthreads=NTH)
        errs.append(np.sqrt(np.mean((u - curved_state(tl, mesh, N, t, eq)) ** 2)))
    orders = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(orders > 4.0), orders


def make_curved_semi(tl, mesh, N, td="lw"):
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tdo))
    return tl.SemidiscretizationHyperbolic(mesh, tdo, eq, tl.initial_condition_convergence_test, solver,
                                           source_terms=tl.source_terms_convergence_test)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [3, 4, 5])
def test_gpu_curved_rhs_with_source_terms_matches_oracle(tl, oracle_mod, N):
    mesh = tl.StructuredMesh((6, 6), warp2)
    semi = make_curved_semi(tl, mesh, N)
    u = semi.compute_coefficients(0.0)
    u = u * (1 + 1e-3 * np.random.default_rng(20 + N).standard_normal(u.shape))
    o = oracle_mod.Oracle(mesh, N)
    o.set_source(1, curved_xnode(mesh, N))
    t, dt = 0.3, 0.5 * o.max_dt(u, 0.2)
    semi.cache["dt"][0] = dt
    du = np.empty_like(u)
    tl.rhs(du, u, semi, t)
    ref = o.rhs(u, t, dt, nthreads=NTH)
    assert np.all(rel_l2(du, ref) < 1e-12), rel_l2(du, ref)


@pytest.mark.gpu
def test_gpu_curved_mdrk_with_source_terms_matches_oracle(tl, oracle_mod):
    """MDRK on the curvilinear mesh: stage 2 takes the source at t, as the structured kernels do."""
    N = 4
    mesh = tl.StructuredMesh((6, 6), warp2)
    semi = make_curved_semi(tl, mesh, N, "mdrk")
    u = semi.compute_coefficients(0.0)
    u = u * (1 + 1e-3 * np.random.default_rng(31).standard_normal(u.shape))
    o = oracle_mod.Oracle(mesh, N)
    o.set_source(1, curved_xnode(mesh, N))
    t, dt = 0.2, 0.5 * o.max_dt(u, 0.2)
    semi.cache["dt"][0] = dt
    du1 = np.empty_like(u)
    tl.rhs_mdrk1(du1, u, semi, t)
    ref1 = o.rhs(u, t, dt, kind=1, nthreads=NTH)
    assert np.all(rel_l2(du1, ref1) < 1e-12), rel_l2(du1, ref1)
    us = u + dt * ref1
    du2 = np.empty_like(u)
    tl.rhs_mdrk2(du2, u, semi, t, us)
    ref2 = o.rhs(u, t, dt, kind=2, us=us, nthreads=NTH)
    assert np.all(rel_l2(du2, ref2) < 1e-12), rel_l2(du2, ref2)


@pytest.mark.gpu
@pytest.mark.parametrize("td", ["lw", "mdrk"])
def test_gpu_curved_steps_with_source_terms_match_oracle(tl, oracle_mod, td):
    N = 4
    mesh = tl.StructuredMesh((8, 8), warp2)
    semi = make_curved_semi(tl, mesh, N, td)
    u0 = semi.compute_coefficients(0.0)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(10, 0.2, use_graph=True)
    integ.sync_time()
    o = oracle_mod.Oracle(mesh, N)
    o.set_source(1, curved_xnode(mesh, N))
    u = u0.copy()
    s, t = o.steps(u, 10, 0.2, 0.0, 1e9, kind=0 if td == "lw" else 1, nthreads=NTH)
    assert s == integ.iter == 10 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(integ.get_state(), u) < 1e-12)
