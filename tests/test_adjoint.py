"""Discrete adjoint of the LW step: the oracle's restatement against finite differences (CPU), and the CUDA
adjoint kernels, the checkpointed reverse sweep and the torch.autograd wrapper against the oracle (GPU).

Tolerances: finite differences are central with Richardson extrapolation; the Rusanov speed and |v| are
piecewise smooth, so a perturbation that crosses a kink limits FD accuracy to O(h): 1e-5 relative there.
GPU against oracle: 1e-12 relative L2 per variable for one step, 1e-10 over a multi-step sweep."""
import os

import numpy as np
import pytest

NTH = os.cpu_count() or 1


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def vortex(tl, level, N, beta=5.0, center=(0.7, -0.4), noise=0.0, seed=0):
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), level)
    from trixilw.batch import compute_coefficients
    u = compute_coefficients(mesh, N, tl.IsentropicVortex(beta, center=center), eq)
    if noise:
        u = u + noise * np.random.default_rng(seed).standard_normal(u.size)
    return eq, mesh, u


def fd(J, u, d, h):
    d1 = (J(u + h * d) - J(u - h * d)) / (2 * h)
    d2 = (J(u + 2 * h * d) - J(u - 2 * h * d)) / (4 * h)
    return (4 * d1 - d2) / 3


def oracle_gradient(o, u0, dts, lam_T):
    states = [u0]
    for dt in dts[:-1]:
        states.append(o.step_fixed(states[-1], dt, nthreads=NTH))
    lam = lam_T
    for u, dt in zip(reversed(states), reversed(dts)):
        lam = o.adjoint_step(u, dt, lam, nthreads=NTH)
    return lam


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("N,speed", [(3, 0), (4, 0), (4, 1), (5, 0)])
def test_oracle_adjoint_step_matches_finite_differences(oracle_mod, tl, N, speed):
    eq, mesh, u = vortex(tl, 2, N)
    o = oracle_mod.Oracle(mesh, N, speed_kind=speed)
    dt = o.max_dt(u, 0.4)
    rng = np.random.default_rng(N)
    lam = rng.standard_normal(u.size)
    g = o.adjoint_step(u, dt, lam)
    for _ in range(2):
        d = rng.standard_normal(u.size)
        ref = fd(lambda x: lam @ o.step_fixed(x, dt), u, d, 1e-6)
        assert abs(g @ d - ref) <= 1e-5 * abs(ref)


def test_oracle_multistep_gradient_matches_finite_differences(oracle_mod, tl):
    """Stands in for forward-mode differentiation through the reference at 8x8 (no Julia here): the
    oracle's reverse sweep over 10 fixed-dt steps against central differences of the oracle's forward."""
    eq, mesh, u0 = vortex(tl, 3, 4, noise=1e-3)
    o = oracle_mod.Oracle(mesh, 4)
    dts = []
    u = u0.copy()
    for _ in range(10):
        dt = o.max_dt(u, 0.5)
        dts.append(dt)
        u = o.step_fixed(u, dt, nthreads=NTH)
    target = np.random.default_rng(1).uniform(0.9, 1.1, u.size // 4)

    def J(x):
        for dt in dts:
            x = o.step_fixed(x, dt, nthreads=NTH)
        return 0.5 * np.sum((x[0::4] - target) ** 2)

    lam_T = np.zeros_like(u)
    lam_T[0::4] = u[0::4] - target
    g = oracle_gradient(o, u0, dts, lam_T)
    rng = np.random.default_rng(2)
    for _ in range(3):
        d = rng.standard_normal(u0.size)
        d /= np.linalg.norm(d)
        ref = fd(J, u0, d, 1e-5)
        assert abs(g @ d - ref) <= 1e-5 * abs(ref)


def forward_mode_directional(o, u0, dts, d, target):
    """J'(u0) d for J = 1/2 ||rho(T) - target||^2 by dual numbers through the fixed-dt steps."""
    u, t = u0, d
    for dt in dts:
        u, t = o.dual_step(u, dt, t)
    return float(np.sum((u[0::4] - target) * t[0::4])), u


@pytest.mark.parametrize("N,speed", [(3, 0), (4, 0), (4, 1), (5, 0)])
def test_dual_step_restates_the_oracle_step(oracle_mod, tl, N, speed):
    """The scalar-templated step in double is the oracle's step (to roundoff); its dual derivative is the step's
    directional derivative (central differences)."""
    eq, mesh, u = vortex(tl, 2, N, noise=1e-3)
    o = oracle_mod.Oracle(mesh, N, speed_kind=speed)
    dt = o.max_dt(u, 0.4)
    ref = o.step_fixed(u, dt)
    assert np.all(rel_l2(o.dual_step(u, dt), ref) < 1e-14)
    d = np.random.default_rng(N).standard_normal(u.size)
    val, der = o.dual_step(u, dt, d)
    assert np.all(rel_l2(val, ref) < 1e-14)
    h = 1e-6
    fdd = (o.step_fixed(u + h * d, dt) - o.step_fixed(u - h * d, dt)) / (2 * h)
    assert np.all(rel_l2(der, fdd) < 1e-7)


def test_forward_mode_matches_the_oracle_adjoint_at_8x8(oracle_mod, tl):
    """The differentiable form's second check (BASELINE: against forward-mode differentiation through the CPU
    path on an 8 x 8 mesh): 20 fixed-dt steps, J = 1/2 ||rho(T) - rho_target||^2; dual-number directional
    derivatives equal the oracle adjoint's dot products to 1e-10 relative on 16 random directions."""
    eq, mesh, u0 = vortex(tl, 3, 4, noise=1e-3)
    o = oracle_mod.Oracle(mesh, 4)
    dts, u = [], u0.copy()
    for _ in range(20):
        dt = o.max_dt(u, 0.5)
        dts.append(dt)
        u = o.step_fixed(u, dt, nthreads=NTH)
    target = np.random.default_rng(1).uniform(0.9, 1.1, u.size // 4)
    lam_T = np.zeros_like(u)
    lam_T[0::4] = u[0::4] - target
    g = oracle_gradient(o, u0, dts, lam_T)
    rng = np.random.default_rng(5)
    for _ in range(16):
        d = rng.standard_normal(u0.size)
        d /= np.linalg.norm(d)
        jd, uT = forward_mode_directional(o, u0, dts, d, target)
        assert np.all(rel_l2(uT, u) < 1e-13)
        assert abs(g @ d - jd) <= 1e-10 * abs(jd)


def test_oracle_adjoint_rejects_unsupported(oracle_mod, tl):
    eq, mesh, u = vortex(tl, 2, 4)
    o = oracle_mod.Oracle(mesh, 4, flux_kind=1)
    with pytest.raises(ValueError):
        o.adjoint_step(u, 0.01, u)


# ---------------------------------------------------------------------------------------------- GPU
def make_semi(tl, mesh, N, speed="naive"):
    eq = tl.CompressibleEulerEquations2D(1.4)
    flux = tl.FluxLaxFriedrichs(max_abs_speed=speed) if speed != "naive" else tl.flux_lax_friedrichs
    solver = tl.DGSEM(N, flux, tl.VolumeIntegralFR(tl.LW()))
    return tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, tl.IsentropicVortex(5.0), solver)


@pytest.mark.gpu
@pytest.mark.parametrize("N,speed", [(3, 0), (4, 0), (4, 1), (5, 0), (5, 1)])
def test_gpu_adjoint_step_matches_oracle(oracle_mod, tl, N, speed):
    eq, mesh, u = vortex(tl, 3, N, noise=1e-3)
    semi = make_semi(tl, mesh, N, "davis" if speed else "naive")
    o = oracle_mod.Oracle(mesh, N, speed_kind=speed)
    dt = o.max_dt(u, 0.4)
    lam = np.random.default_rng(N).standard_normal(u.size)
    g_cpu = o.adjoint_step(u, dt, lam, nthreads=NTH)
    g_gpu = tl.adjoint_step(semi, lam, u, dt)
    assert np.all(rel_l2(g_gpu, g_cpu) < 1e-12)


@pytest.mark.gpu
def test_gpu_fixed_dt_solve_matches_oracle(oracle_mod, tl):
    eq, mesh, u0 = vortex(tl, 3, 4)
    semi = make_semi(tl, mesh, 4)
    o = oracle_mod.Oracle(mesh, 4)
    dts = [0.05, 0.04, 0.045, 0.03]
    u = u0.copy()
    for dt in dts:
        u = o.step_fixed(u, dt, nthreads=NTH)
    assert np.all(rel_l2(tl.solve_dts(semi, u0, dts), u) < 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("ck", [1, 7, 13, 25])
def test_gpu_sweep_matches_oracle_and_checkpoint_interval(oracle_mod, tl, ck):
    eq, mesh, u0 = vortex(tl, 3, 4, noise=1e-3)
    semi = make_semi(tl, mesh, 4)
    nsteps, cfl = 25, 0.4
    uT = tl.forward_record(semi, u0, nsteps, cfl, ck)
    dts = tl.adjoint.dt_sequence(semi, nsteps)
    o = oracle_mod.Oracle(mesh, 4)
    u = u0.copy()
    for dt in dts:
        u = o.step_fixed(u, dt, nthreads=NTH)
    assert np.all(rel_l2(uT, u) < 1e-11)
    lam_T = np.random.default_rng(3).standard_normal(u0.size)
    g = tl.adjoint_sweep(semi, lam_T)
    g_ref = oracle_gradient(o, u0, dts, lam_T)
    assert np.all(rel_l2(g, g_ref) < 1e-10)
    # the record pass leaves the last segment in its buffer; a second sweep (which recomputes it once three or
    # more segments have reused the buffers) and the serial, phase-timed sweep give the same bits
    np.testing.assert_array_equal(tl.adjoint_sweep(semi, lam_T), g)
    g_timed, (rec_ms, adj_ms) = tl.adjoint_sweep(semi, lam_T, timing=True)
    np.testing.assert_array_equal(g_timed, g)
    assert rec_ms >= 0.0 and adj_ms > 0.0
    if ck != 1:
        tl.forward_record(semi, u0, nsteps, cfl, 1)
        np.testing.assert_array_equal(tl.adjoint_sweep(semi, lam_T), g)


@pytest.mark.gpu
def test_gpu_objective_gradient_finite_differences(tl):
    """The differentiable-form check at a small size: J = 1/2 ||rho(T) - rho_target||^2 after 40 steps on
    16x16, N = 4, checkpoints every 10 steps, 8 random unit directions, 1e-6 relative."""
    eq, mesh, u0 = vortex(tl, 4, 4, beta=5.0, center=(0.0, 0.0), noise=1e-3)
    semi = make_semi(tl, mesh, 4)
    _, _, ut0 = vortex(tl, 4, 4, beta=4.5, center=(0.0, 0.0))
    nsteps, cfl = 40, tl.trixi2lw(0.98, semi.solver)
    target = tl.forward_record(semi, ut0, nsteps, cfl, 10)[0::4].copy()
    J, g, uT = tl.adjoint_solve(semi, u0, nsteps, cfl, 10, target)
    assert J == pytest.approx(0.5 * np.sum((uT[0::4] - target) ** 2), rel=1e-12)
    dts = tl.adjoint.dt_sequence(semi, nsteps)

    def Jf(x):
        return 0.5 * np.sum((tl.solve_dts(semi, x, dts)[0::4] - target) ** 2)

    rng = np.random.default_rng(0)
    for _ in range(8):
        d = rng.standard_normal(u0.size)
        d /= np.linalg.norm(d)
        ref = fd(Jf, u0, d, 1e-4)
        assert abs(g @ d - ref) <= 1e-6 * abs(ref) + 1e-14


@pytest.mark.gpu
def test_gpu_adjoint_matches_forward_mode_at_8x8(oracle_mod, tl):
    """The device's checkpointed adjoint gradient on the 8 x 8, N = 4 vortex (200 steps of the workload's CFL,
    checkpoints every 20; rho_target from a strength-4.5 run; u0 = strength 5 + N(0, 1e-3^2)) against dual-number
    forward mode through the oracle's steps at the recorded dt sequence: 1e-10 relative on 8 random directions."""
    eq, mesh, u0 = vortex(tl, 3, 4, beta=5.0, center=(0.0, 0.0), noise=1e-3)
    semi = make_semi(tl, mesh, 4)
    _, _, ut0 = vortex(tl, 3, 4, beta=4.5, center=(0.0, 0.0))
    nsteps, cfl = 200, tl.trixi2lw(0.98, semi.solver)
    target = tl.forward_record(semi, ut0, nsteps, cfl, 20)[0::4].copy()
    J, g, uT = tl.adjoint_solve(semi, u0, nsteps, cfl, 20, target)
    dts = tl.adjoint.dt_sequence(semi, nsteps)
    o = oracle_mod.Oracle(mesh, 4)
    rng = np.random.default_rng(11)
    for _ in range(8):
        d = rng.standard_normal(u0.size)
        d /= np.linalg.norm(d)
        jd, uT_cpu = forward_mode_directional(o, u0, dts, d, target)
        assert np.all(rel_l2(uT, uT_cpu) < 1e-10)
        assert abs(g @ d - jd) <= 1e-10 * abs(jd)


def make_mdrk_semi(tl, mesh, N):
    eq = tl.CompressibleEulerEquations2D(1.4)
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.MDRK()))
    return tl.SemidiscretizationHyperbolic(mesh, tl.MDRK(), eq, tl.IsentropicVortex(5.0), solver)


def test_dual_mdrk_step_restates_the_oracle_step(oracle_mod, tl):
    for N in (3, 4, 5):
        eq, mesh, u = vortex(tl, 2, N, noise=1e-3)
        o = oracle_mod.Oracle(mesh, N)
        dt = o.max_dt(u, 0.4)
        ref = u.copy()
        o.steps(ref, 1, 0.4, 0.0, 1e9, kind=1, fixed_dt=dt)
        assert np.all(rel_l2(o.dual_step(u, dt, kind=1), ref) < 1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [3, 4, 5])
def test_gpu_mdrk_adjoint_step_matches_forward_mode(oracle_mod, tl, N):
    """The discrete adjoint of one two-stage MDRK step (both stages, the jump in u^n at the interfaces of both,
    the stage-2 time averages built on stage 1's F2 and U2) against dual-number directional derivatives."""
    eq, mesh, u = vortex(tl, 3, N, noise=1e-3)
    semi = make_mdrk_semi(tl, mesh, N)
    o = oracle_mod.Oracle(mesh, N)
    dt = o.max_dt(u, 0.4)
    rng = np.random.default_rng(N)
    lam = rng.standard_normal(u.size)
    g = tl.adjoint_step(semi, lam, u, dt)
    for _ in range(4):
        d = rng.standard_normal(u.size)
        _, der = o.dual_step(u, dt, d, kind=1)
        assert abs(g @ d - lam @ der) <= 1e-11 * np.abs(lam).sum() * np.abs(der).max()
        assert abs(g @ d - lam @ der) <= 1e-10 * abs(lam @ der)


@pytest.mark.gpu
def test_gpu_mdrk_fixed_dt_solve_matches_oracle(oracle_mod, tl):
    eq, mesh, u0 = vortex(tl, 3, 4)
    semi = make_mdrk_semi(tl, mesh, 4)
    o = oracle_mod.Oracle(mesh, 4)
    dts = [0.05, 0.04, 0.045]
    u = u0.copy()
    for dt in dts:
        o.steps(u, 1, 0.4, 0.0, 1e9, kind=1, fixed_dt=dt)
    assert np.all(rel_l2(tl.solve_dts(semi, u0, dts), u) < 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("ck", [1, 6, 40])
def test_gpu_mdrk_gradient_matches_forward_mode(oracle_mod, tl, ck):
    """The checkpointed MDRK gradient of J = 1/2 ||rho(T) - rho_target||^2 over 40 CFL steps on 8 x 8, N = 4,
    against dual-number forward mode through the oracle's MDRK steps at the recorded dt sequence (1e-10), and the
    same gradient for every checkpoint interval."""
    eq, mesh, u0 = vortex(tl, 3, 4, beta=5.0, center=(0.0, 0.0), noise=1e-3)
    semi = make_mdrk_semi(tl, mesh, 4)
    _, _, ut0 = vortex(tl, 3, 4, beta=4.5, center=(0.0, 0.0))
    nsteps, cfl = 40, 0.4
    target = tl.forward_record(semi, ut0, nsteps, cfl, ck)[0::4].copy()
    J, g, uT = tl.adjoint_solve(semi, u0, nsteps, cfl, ck, target)
    dts = tl.adjoint.dt_sequence(semi, nsteps)
    o = oracle_mod.Oracle(mesh, 4)
    rng = np.random.default_rng(ck)
    for _ in range(4):
        d = rng.standard_normal(u0.size)
        d /= np.linalg.norm(d)
        u, t = u0, d
        for dt in dts:
            u, t = o.dual_step(u, dt, t, kind=1)
        jd = float(np.sum((u[0::4] - target) * t[0::4]))
        assert np.all(rel_l2(uT, u) < 1e-10)
        assert abs(g @ d - jd) <= 1e-10 * abs(jd)


@pytest.mark.gpu
def test_torch_autograd_function(tl):
    import torch
    eq, mesh, u0 = vortex(tl, 3, 4, noise=1e-3)
    semi = make_semi(tl, mesh, 4)
    for dev in ("cpu", "cuda"):
        x = torch.tensor(u0, dtype=torch.float64, device=dev, requires_grad=True)
        y = tl.lw_solve(x, semi, 12, 0.4, 5)
        w = torch.linspace(-1.0, 1.0, y.numel(), dtype=torch.float64, device=dev)
        (y * w).sum().backward()
        ref = tl.adjoint_sweep(semi, w.cpu().numpy())
        np.testing.assert_array_equal(x.grad.cpu().numpy(), ref)
