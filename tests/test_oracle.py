"""CPU tests of the oracle (the checker): known answers for the basis, scheme invariants the reference
has by construction, agreement with an independent numpy restatement, and regression against the
committed golden fixtures."""
import os

import numpy as np
import pytest

import numpy_lw


def test_gll_known_answers(oracle_mod):
    # N = 4: nodes 0, +-sqrt(3/7), +-1; weights 32/45, 49/90, 1/10
    x, w, D, Dh = oracle_mod.basis(4)
    np.testing.assert_allclose(x, [-1, -np.sqrt(3 / 7), 0, np.sqrt(3 / 7), 1], atol=1e-15)
    np.testing.assert_allclose(w, [1 / 10, 49 / 90, 32 / 45, 49 / 90, 1 / 10], atol=1e-15)
    # N = 3: +-1, +-sqrt(1/5); weights 1/6, 5/6
    x, w, _, _ = oracle_mod.basis(3)
    np.testing.assert_allclose(x, [-1, -np.sqrt(0.2), np.sqrt(0.2), 1], atol=1e-15)
    np.testing.assert_allclose(w, [1 / 6, 5 / 6, 5 / 6, 1 / 6], atol=1e-15)


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_derivative_matrix_exact_on_polynomials(oracle_mod, N):
    x, w, D, Dh = oracle_mod.basis(N)
    for p in range(N + 1):
        np.testing.assert_allclose(D @ x ** p, p * x ** max(p - 1, 0) * (p > 0), atol=2e-13)
    # summation-by-parts: M D + D^T M = B
    M = np.diag(w)
    B = np.zeros((N + 1, N + 1)); B[0, 0] = -1; B[-1, -1] = 1
    np.testing.assert_allclose(M @ D + D.T @ M, B, atol=1e-13)
    # Dhat = -M^-1 D^T M
    np.testing.assert_allclose(Dh, -np.diag(1 / w) @ D.T @ M, atol=1e-13)
    assert abs(w.sum() - 2.0) < 1e-14


def test_host_basis_matches_oracle(oracle_mod, tl):
    from trixilw.basis import gauss_lobatto
    for N in range(1, 8):
        x, w = gauss_lobatto(N)
        xo, wo, _, _ = oracle_mod.basis(N)
        np.testing.assert_allclose(x, xo, atol=1e-15)
        np.testing.assert_allclose(w, wo, atol=1e-15)


def _setup(tl, level, N, ic, lo=-10.0, hi=10.0, periodic=True):
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((lo, lo), (hi, hi), level, periodicity=periodic)
    xy = mesh.node_coordinates(N)
    u = ic(xy[0], xy[1], 0.0, eq)
    u = np.ascontiguousarray(np.transpose(u, (2, 1, 0, 3))).reshape(-1)
    return eq, mesh, u


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("kind", [0, 1])
def test_free_stream_preservation(oracle_mod, tl, N, kind):
    eq, mesh, u = _setup(tl, 2, N, tl.ConstantState(1.3, 0.4, -0.7, 2.1))
    o = oracle_mod.Oracle(mesh, N)
    dt = o.max_dt(u, 0.3)
    du = o.rhs(u, 0.0, dt, kind=kind)
    assert np.abs(du).max() < 1e-12
    if kind == 1:
        us = u + dt * du
        du2 = o.rhs(u, 0.0, dt, kind=2, us=us)
        assert np.abs(du2).max() < 1e-12


@pytest.mark.parametrize("N", [2, 3, 4, 5])
@pytest.mark.parametrize("kind", [0, 1])
def test_conservation_periodic(oracle_mod, tl, N, kind):
    eq, mesh, u = _setup(tl, 3, N, tl.IsentropicVortex(5.0, center=(1.0, -2.0)))
    o = oracle_mod.Oracle(mesh, N)
    dt = o.max_dt(u, 0.4)
    du = o.rhs(u, 0.0, dt, kind=kind)
    _, w, _, _ = oracle_mod.basis(N)
    n = N + 1
    d = du.reshape(mesh.n_elements, n, n, 4)
    total = np.einsum("ejiv,j,i->v", d, w, w) / mesh.inverse_jacobian[0] ** 2
    scale = np.einsum("ejiv,j,i->v", np.abs(d), w, w) / mesh.inverse_jacobian[0] ** 2
    assert np.all(np.abs(total) <= 1e-13 * scale)


@pytest.mark.parametrize("N", [3, 4, 5])
def test_mirror_symmetry(oracle_mod, tl, N):
    """Mirroring x -> -x (with v1 -> -v1) commutes with the rhs."""
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    xy = mesh.node_coordinates(N)
    ic = tl.IsentropicVortex(4.0, center=(0.7, -1.3), velocity=(0.5, 1.0))
    u = np.transpose(ic(xy[0], xy[1], 0.0, eq), (2, 1, 0, 3))        # [e, j, i, v]
    # mirrored field: element at (ix, iy) takes the data of (m-1-ix, iy) with i reversed and v1 negated
    m = mesh.cells_per_dimension
    src = mesh.element_at[m - 1 - mesh.ix, mesh.iy]
    um = u[src][:, :, ::-1, :].copy()
    um[..., 1] *= -1
    o = oracle_mod.Oracle(mesh, N)
    dt = 0.01
    du = o.rhs(np.ascontiguousarray(u).reshape(-1), 0.0, dt).reshape(u.shape)
    dum = o.rhs(np.ascontiguousarray(um).reshape(-1), 0.0, dt).reshape(u.shape)
    expect = du[src][:, :, ::-1, :].copy()
    expect[..., 1] *= -1
    np.testing.assert_allclose(dum, expect, atol=1e-12 * np.abs(du).max())


@pytest.mark.parametrize("N", [3, 4, 5])
def test_numpy_restatement_agrees(oracle_mod, tl, N):
    eq, mesh, u = _setup(tl, 2, N, tl.IsentropicVortex(5.0, center=(0.5, 0.3)))
    o = oracle_mod.Oracle(mesh, N)
    dt = o.max_dt(u, 0.9 * (N + 1) * 0.103)
    du = o.rhs(u, 0.0, dt)
    x, w, D, Dh = oracle_mod.basis(N)
    n = N + 1
    du_np, U, F, G = numpy_lw.rhs(u.reshape(mesh.n_elements, n, n, 4), mesh, D, Dh, w, dt)
    rel = np.linalg.norm(du - du_np.reshape(-1)) / np.linalg.norm(du)
    assert rel < 1e-13, rel
    Uo = o.get(0).reshape(mesh.n_elements, n, n, 4)
    np.testing.assert_allclose(Uo, U, rtol=0, atol=1e-13)
    Fo = o.get(1).reshape(mesh.n_elements, n, n, 2, 4)
    np.testing.assert_allclose(Fo[..., 0, :], F, atol=1e-12)
    np.testing.assert_allclose(Fo[..., 1, :], G, atol=1e-12)


def test_domain_error_on_negative_pressure(oracle_mod, tl):
    eq, mesh, u = _setup(tl, 2, 3, tl.ConstantState(1.0, 0.1, 0.1, 1.0))
    u = u.reshape(-1, 4)
    o = oracle_mod.Oracle(mesh, 3)
    # interior node: the rhs takes no square root there (as in the reference), max_dt does
    bad = u.copy()
    bad[5, 3] = -1.0   # element 1, node (1,1): negative energy -> negative pressure
    o.rhs(bad.reshape(-1), 0.0, 1e-3)
    with pytest.raises(oracle_mod.OracleDomainError):
        o.max_dt(bad.reshape(-1), 0.5)
    # face node: the interface speed estimate takes sqrt(gamma p / rho) of the time-averaged trace
    bad = u.copy()
    bad[0, 3] = -1.0
    with pytest.raises(oracle_mod.OracleDomainError):
        o.rhs(bad.reshape(-1), 0.0, 1e-3)


def _vortex_error(oracle_mod, tl, level, N, t_end=1.0, kind=0):
    eq, mesh, u = _setup(tl, level, N, tl.IsentropicVortex(5.0))
    o = oracle_mod.Oracle(mesh, N)
    cfl = 0.98 * (N + 1) * tl.lw_fourier_cfl(min(N, 4)) if N <= 4 else 0.3
    steps, t = o.steps(u, 100000, cfl, 0.0, t_end, kind=kind, nthreads=os.cpu_count() or 1)
    assert abs(t - t_end) < 1e-12
    xy = mesh.node_coordinates(N)
    ue = np.transpose(tl.IsentropicVortex(5.0)(xy[0], xy[1], t_end, eq), (2, 1, 0, 3)).reshape(-1)
    _, w, _, _ = oracle_mod.basis(N)
    n = N + 1
    d = (u - ue).reshape(mesh.n_elements, n, n, 4)
    return np.sqrt(np.einsum("ejiv,j,i->v", d * d, w, w).sum() / mesh.inverse_jacobian[0] ** 2 / 400.0)


@pytest.mark.parametrize("N", [3, 4])
def test_vortex_convergence_order(oracle_mod, tl, N):
    # levels 5 -> 6 (32^2 -> 64^2 elements on [-10,10]^2); coarser levels are pre-asymptotic
    e1 = _vortex_error(oracle_mod, tl, 5, N)
    e2 = _vortex_error(oracle_mod, tl, 6, N)
    eoc = np.log2(e1 / e2)
    assert eoc > N + 0.4, (e1, e2, eoc)


def test_mdrk_converges(oracle_mod, tl):
    e1 = _vortex_error(oracle_mod, tl, 5, 3, kind=1)
    e2 = _vortex_error(oracle_mod, tl, 6, 3, kind=1)
    assert np.log2(e1 / e2) > 3.4, (e1, e2)


GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["lw_vortex_N3_L2", "lw_vortex_N4_L2", "lw_vortex_N5_L2", "mdrk_vortex_N4_L2",
                                  "lw_riemann_N4_L2", "sc_lw_riemann_N4_L3", "sc_mdrk_riemann_N3_L3"])
def test_golden_fixtures(oracle_mod, tl, name):
    import golden_cases
    path = os.path.join(GOLDEN, name + ".npz")
    ref = np.load(path)
    out = golden_cases.run_case(name, oracle_mod, tl)
    for k in ref.files:
        np.testing.assert_allclose(out[k], ref[k], rtol=0, atol=1e-13 * max(1.0, np.abs(ref[k]).max()), err_msg=k)


def _numpy_indicator(u, n, gamma=1.4, alpha_max=0.5, alpha_min=0.001):
    """Independent numpy restatement of the Hennemann-Gassner indicator (before smoothing)."""
    from numpy.polynomial import legendre as Lg
    x, _ = np.polynomial.legendre.leggauss(2)   # placeholder to import module
    from trixilw.basis import gauss_lobatto
    nodes, _ = gauss_lobatto(n - 1)
    V = np.stack([Lg.legval(nodes, np.eye(n)[m]) * np.sqrt(m + 0.5) for m in range(n)], axis=1)
    Vi = np.linalg.inv(V)
    uu = u.reshape(-1, n, n, 4)                                        # [e, j, i, v]
    ind = (gamma - 1) * (uu[..., 0] * uu[..., 3] - 0.5 * (uu[..., 1] ** 2 + uu[..., 2] ** 2))
    modal = np.einsum("ia,jb,eba->eji", Vi, Vi, ind)                    # modal[e, j, i]
    m2 = modal ** 2
    total = m2.sum(axis=(1, 2))
    c1 = m2[:, : n - 1, : n - 1].sum(axis=(1, 2))
    c2 = m2[:, : n - 2, : n - 2].sum(axis=(1, 2))
    f1 = np.where(total != 0, (total - c1) / np.where(total != 0, total, 1), 0)
    f2 = np.where(c1 != 0, (c1 - c2) / np.where(c1 != 0, c1, 1), 0)
    energy = np.maximum(f1, f2)
    thr = 0.5 * 10 ** (-1.8 * n ** 0.25)
    s = np.log((1 - 1e-4) / 1e-4)
    a = 1 / (1 + np.exp(-s / thr * (energy - thr)))
    a = np.where(a < alpha_min, 0.0, a)
    a = np.where(a > 1 - alpha_min, 1.0, a)
    return np.minimum(alpha_max, a)


@pytest.mark.parametrize("N", [3, 4, 5])
def test_indicator_against_numpy(oracle_mod, tl, N):
    eq, mesh, u = _setup(tl, 3, N, tl.FourQuadrantRiemann(), lo=0.0, hi=1.0, periodic=False)
    o = oracle_mod.Oracle(mesh, N)
    o.set_shock_capturing(True, 0.5, 0.001, False)         # no smoothing: compare the raw indicator
    levels, now = __import__("golden_cases").boundary_data(mesh, N, tl.FourQuadrantRiemann(), eq)
    o.set_boundary_data(levels, now)
    o.rhs(u, 0.0, 1e-4)
    ref = _numpy_indicator(u, N + 1)
    np.testing.assert_allclose(o.get(6), ref, atol=1e-12)
    assert ref.max() > 0


def test_indicator_zero_on_smooth_vortex(oracle_mod, tl):
    eq, mesh, u = _setup(tl, 5, 4, tl.IsentropicVortex(5.0))
    o = oracle_mod.Oracle(mesh, 4)
    o.set_shock_capturing(True, 0.5)
    o.rhs(u, 0.0, 1e-3)
    assert o.get(6).max() == 0.0


@pytest.mark.parametrize("kind", [0, 1])
def test_shock_capturing_free_stream_and_conservation(oracle_mod, tl, kind):
    eq, mesh, u = _setup(tl, 3, 4, tl.ConstantState(1.1, 0.2, -0.4, 0.9))
    o = oracle_mod.Oracle(mesh, 4)
    o.set_shock_capturing(True, 0.5)
    assert np.abs(o.rhs(u, 0.0, 1e-3, kind=kind)).max() < 1e-12

    def square(x, y, t, eq):
        rho = np.where((np.abs(x) < 4) & (np.abs(y) < 4), 2.0, 1.0)
        return eq.prim2cons(rho, 0.5, 0.3, 1.0)
    eq, mesh, u = _setup(tl, 4, 4, square)
    o = oracle_mod.Oracle(mesh, 4)
    o.set_shock_capturing(True, 0.5)
    du = o.rhs(u, 0.0, 1e-3, kind=kind)
    assert o.get(6).max() > 0
    _, w, _, _ = oracle_mod.basis(4)
    d = du.reshape(mesh.n_elements, 5, 5, 4)
    total = np.einsum("ejiv,j,i->v", d, w, w)
    scale = np.einsum("ejiv,j,i->v", np.abs(d), w, w)
    assert np.all(np.abs(total) <= 1e-13 * scale)


def test_riemann_shock_capturing_runs_to_t025(oracle_mod, tl):
    """Config 2 Riemann problem (32^2, N = 4, alpha_max = 0.5, CFL 0.15) stays admissible to t = 0.25."""
    import golden_cases
    eq, mesh, u = _setup(tl, 5, 4, tl.FourQuadrantRiemann(), lo=0.0, hi=1.0, periodic=False)
    o = oracle_mod.Oracle(mesh, 4)
    o.set_shock_capturing(True, 0.5)
    o.set_boundary_data(*golden_cases.boundary_data(mesh, 4, tl.FourQuadrantRiemann(), eq))
    s, t = o.steps(u, 100000, 0.15, 0.0, 0.25, nthreads=os.cpu_count() or 1)
    assert abs(t - 0.25) < 1e-12
    rho = u.reshape(-1, 4)[:, 0]
    assert rho.min() > 0.05 and rho.max() < 2.5


def test_step_loop_final_time_semantics(oracle_mod, tl):
    """isfinished is Julia's t ≈ t_end (rtol sqrt(eps)): an infinite t_end never finishes, a finite one
    clamps the last dt so that t lands on t_end exactly, and no step is taken from t_end."""
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 2)
    eq = tl.CompressibleEulerEquations2D(1.4)
    xy = mesh.node_coordinates(3)
    u0 = np.ascontiguousarray(np.transpose(tl.IsentropicVortex(5.0)(xy[0], xy[1], 0.0, eq), (2, 1, 0, 3))).reshape(-1)
    o = oracle_mod.Oracle(mesh, 3)
    u = u0.copy()
    s, t = o.steps(u, 3, 0.5, 0.0, float("inf"))
    assert s == 3 and 0.0 < t < float("inf")
    u = u0.copy()
    s, t = o.steps(u, 1000, 0.5, 0.0, 0.3)
    assert t == 0.3 and 1 < s < 1000
    s2, t2 = o.steps(u, 5, 0.5, t, 0.3)
    assert s2 == 0 and t2 == 0.3
    # within sqrt(eps) of the final time counts as finished
    s3, _ = o.steps(u0.copy(), 5, 0.5, 0.3 * (1 - 1e-9), 0.3)
    assert s3 == 0


def test_host_isfinished_semantics(tl):
    from trixilw.lwfr import LWIntegrator

    integ = LWIntegrator.__new__(LWIntegrator)
    for t, te, want in [(0.0, float("inf"), False), (1.0, 1.0, True), (1.0 - 1e-10, 1.0, True),
                        (0.5, 1.0, False), (1e-20, 0.0, True)]:
        integ.t, integ.tspan = t, (0.0, te)
        assert integ.isfinished() is want
