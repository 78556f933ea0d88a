"""Adaptive (error-controlled) LW stepping: the controller of perform_step!(..., ::Adaptive, ::LW) driven by
the oracle's trial steps on the CPU, and libtlw's device trial step (volume kernel with the temporal error
estimate, admissibility check) against that run on the GPU."""
import math
import os

import numpy as np
import pytest

NTH = os.cpu_count() or 1
TOL = {"abstol": 1e-6, "reltol": 1e-6}


def vortex(tl, mesh, N):
    eq = tl.CompressibleEulerEquations2D(1.4)
    xy = mesh.node_coordinates(N)
    v = tl.IsentropicVortex(5.0, center=(0.7, -0.4))(xy[0], xy[1], 0.0, eq)
    return np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)


def oracle_adaptive(oracle_mod, mesh, N, u0, t_end, dt0, tol=TOL, oracle_obj=None):
    """The reference's adaptive loop with the oracle as the trial step (oracle_obj: a configured oracle)."""
    from trixilw.lwfr import AdaptiveController
    o = oracle_obj or oracle_mod.Oracle(mesh, N)
    o.set_temporal_errors(True, tol["abstol"], tol["reltol"])
    ctl = AdaptiveController(N + 1, 0.0, t_end, dt0)
    u = u0.copy()
    dts = []
    while not ctl.finished():
        dt = ctl.dt
        try:
            du = o.rhs(u, 0.0, dt, nthreads=NTH)
            err = math.sqrt(np.sum(o.get(4)) / (mesh.n_elements * (N + 1) ** 2))
            ut = u + dt * du
            x = ut.reshape(-1, 4)
            p = 0.4 * (x[:, 3] - 0.5 * (x[:, 1] ** 2 + x[:, 2] ** 2) / x[:, 0])
            ok = bool(np.all(x[:, 0] > 0) and np.all(p > 0))
        except oracle_mod.OracleDomainError:
            err, ok, ut = float("nan"), False, None
        if ctl.judge(err, ok):
            u = ut
            dts.append(dt)
    return u, ctl, dts


def test_dt_factor(tl):
    from trixilw.lwfr import dt_factor
    assert dt_factor({-1: 1.0, 0: 1.0, 1: 1.0}, 5) == 1.0
    assert dt_factor({-1: 1.0, 0: 1.0, 1: 100.0}, 5) > dt_factor({-1: 1.0, 0: 1.0, 1: 10.0}, 5) > 1.0
    assert dt_factor({-1: 1.0, 0: 1.0, 1: 0.01}, 5) < 0.81


def test_oracle_adaptive_run(oracle_mod, tl):
    m = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    u0 = vortex(tl, m, 4)
    u, ctl, dts = oracle_adaptive(oracle_mod, m, 4, u0, 1.0, 1e-3)
    assert ctl.t == 1.0 and ctl.iter == len(dts) and 5 < ctl.iter < 200
    assert max(dts) > 10 * dts[0]            # the controller grows the step from the tiny initial one
    assert np.all(np.isfinite(u))


@pytest.mark.gpu
def test_gpu_adaptive_matches_oracle_run(oracle_mod, tl):
    m = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    eq = tl.CompressibleEulerEquations2D(1.4)
    solver = tl.DGSEM(4, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    semi = tl.SemidiscretizationHyperbolic(m, tl.LW(), eq, tl.IsentropicVortex(5.0, center=(0.7, -0.4)), solver)
    u0 = vortex(tl, m, 4)
    upd = tl.semidiscretize(semi, tl.LW(), (0.0, 1.0))
    upd.u0_ode[:] = u0
    sol = tl.solve_lwfr(upd, (), 1e-3, TOL, tl.Adaptive())
    u_cpu, ctl, dts = oracle_adaptive(oracle_mod, m, 4, u0, 1.0, 1e-3)
    assert sol.t[0] == 1.0
    assert sol.stats.nreject == ctl.nreject
    d = (sol.u[0] - u_cpu).reshape(-1, 4)
    assert np.all(np.linalg.norm(d, axis=0) / np.linalg.norm(u_cpu.reshape(-1, 4), axis=0) < 1e-10)


def test_host_controller_stops_when_dt_stalls(tl):
    """Every trial rejected (a persistently non-admissible state): the reference would retry for ever; the
    controller raises DomainError once dt no longer moves t."""
    from trixilw.lwfr import ADAPTIVE_DT_FLOOR, AdaptiveController
    ctl = AdaptiveController(5, 0.5, 1.0, 1e-3)
    with pytest.raises(tl.DomainError):
        for _ in range(10_000):
            ctl.judge(float("nan"), False)
    assert ctl.dt <= ADAPTIVE_DT_FLOOR * 1.0 and 400 < ctl.n_fail < 1000


def _negative_pressure_semi(tl):
    m = tl.TreeMesh((-1.0, -1.0), (1.0, 1.0), 2)
    eq = tl.CompressibleEulerEquations2D(1.4)
    solver = tl.DGSEM(4, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    semi = tl.SemidiscretizationHyperbolic(m, tl.LW(), eq, tl.IsentropicVortex(5.0), solver)
    upd = tl.semidiscretize(semi, tl.LW(), (0.0, 1.0))
    u = upd.u0_ode.reshape(-1, 4)
    u[:, 1:3] = 0.0
    u[:, 3] = -1.0          # rho e < 0 everywhere: every trial takes the square root of a negative pressure
    return upd


@pytest.mark.gpu
@pytest.mark.parametrize("on_device", [False, True])
def test_gpu_adaptive_run_with_a_non_admissible_state_ends(tl, on_device):
    """A run that can never accept a trial stops with DomainError (host controller and device controller)."""
    upd = _negative_pressure_semi(tl)
    with pytest.raises(tl.DomainError):
        tl.solve_lwfr(upd, (), 1e-3, TOL, tl.Adaptive(on_device=on_device, chunk=64))
