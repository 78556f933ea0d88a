"""Host-side mirror of the reference's LW time loop, with the step loop itself on the device.

Mirrors solve_lwfr / LWIntegrator / perform_step!(..., ::CFLBased, ::LW|::MDRK)
(src/solvers/lwfr.jl:31-263, src/solvers/mdrk.jl:1-29): each step computes dt = cfl * max_dt(u)
(clamped to the final time by set_dt!), evaluates the rhs and updates u = uprev + dt * du. Here that
whole step - the CFL reduction included - runs in libtlw (``tlw_step``) and dt never leaves the GPU; the
host only synchronises between callback intervals.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import DomainError, check, lib
from .basis import gauss_lobatto
from .limiters import install as install_limiters
from .semidiscretization import Adaptive, CFLBased, LWUpdate, SemidiscretizationHyperbolic, _ptr


@dataclass
class Stats:
    naccept: int = 0
    nreject: int = 0


@dataclass
class LWSolution:
    u: list
    prob: LWUpdate
    t: list
    stats: Stats = field(default_factory=Stats)


class LWIntegrator:
    """State of a device-resident LW/MDRK run (LWIntegrator, src/solvers/lwfr.jl:31-56)."""

    def __init__(self, lw_update: LWUpdate, tolerances=None):
        self.p: SemidiscretizationHyperbolic = lw_update.p
        self.tspan = lw_update.tspan
        self.t = self.tspan[0]
        self.dt = 0.0
        self.iter = 0
        self.tolerances = tolerances or {"abstol": 0.0, "reltol": 0.0}
        self.stats = Stats()

    @property
    def handle(self):
        return self.p.handle

    def set_state(self, u: np.ndarray, t: float):
        check(self.handle, lib().tlw_set_state(self.handle, _ptr(u), _lib.TLW_WHERE_HOST, float(t)))
        self.t = float(t)

    def get_state(self) -> np.ndarray:
        u = np.empty(4 * self.p.ndofs())
        t = ctypes.c_double()
        check(self.handle, lib().tlw_get_state(self.handle, _ptr(u), _lib.TLW_WHERE_HOST, ctypes.byref(t)))
        self.t = t.value
        return u

    def sync_time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        steps = ctypes.c_int64()
        check(self.handle, lib().tlw_get_time(self.handle, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(steps)))
        self.t, self.dt, self.iter = t.value, dt.value, int(steps.value)
        self.stats.naccept = self.iter
        return self.t

    def step(self, nsteps: int, cfl: float, fixed_dt: float = 0.0, use_graph: bool = True):
        check(self.handle, lib().tlw_step(self.handle, int(nsteps), float(cfl), float(fixed_dt),
                                          float(self.tspan[1]), 1 if use_graph else 0))

    def step_host(self, u_in: np.ndarray, u_out: np.ndarray, t: float, nsteps: int, cfl: float,
                  fixed_dt: float = 0.0):
        """Asynchronous host-buffer stepping (tlw_step_host): u_in at time t is uploaded, advanced nsteps steps and
        downloaded into u_out; both arrays must stay alive and untouched until ``synchronize``. Consecutive calls
        overlap their copies (pinned arrays, e.g. from ``pinned_state``, make the copies asynchronous)."""
        n = 4 * self.p.ndofs()
        if u_in.size != n or u_out.size != n or u_in.dtype != np.float64 or u_out.dtype != np.float64:
            raise ValueError("u_in / u_out: float64 state vectors of the mesh's size")
        if not (u_in.flags.c_contiguous and u_out.flags.c_contiguous):
            raise ValueError("u_in / u_out must be contiguous")
        check(self.handle, lib().tlw_step_host(self.handle, _ptr(u_in), _ptr(u_out), float(t), int(nsteps),
                                               float(cfl), float(fixed_dt), float(self.tspan[1])))

    def synchronize(self):
        check(self.handle, lib().tlw_synchronize(self.handle))

    def pinned_state(self) -> np.ndarray:
        """A page-locked host state vector of the mesh's size (through torch's pinned allocator)."""
        import torch
        return torch.empty(4 * self.p.ndofs(), dtype=torch.float64, pin_memory=True).numpy()

    def isfinished(self) -> bool:
        # integrator.t ≈ last(tspan) (src/solvers/lwfr.jl:147-149): Julia isapprox, rtol = sqrt(eps)
        te = self.tspan[1]
        if self.t == te:
            return True
        if not (math.isfinite(self.t) and math.isfinite(te)):
            return False
        return abs(self.t - te) <= math.sqrt(np.finfo(float).eps) * max(abs(self.t), abs(te)) or self.t >= te


def solve_lwfr(lw_update: LWUpdate, callbacks=(), dt_initial: float = 0.0, tolerances=None,
               time_step_computation=None, limiters=(), chunk: int = 64, use_graph: bool = True) -> LWSolution:
    """solve_lwfr(lw_update, callbacks, dt_initial, tolerances; time_step_computation) (lwfr.jl:233-263).

    callbacks: objects with an ``interval`` (steps) called as ``cb(integrator, u)`` every interval steps
    and at the end. limiters: PositivityPreservingLimiterZhangShu instances; applied on the device once
    before the loop and after every step as solve_lwfr does (lwfr.jl:226, 251, 257)."""
    if time_step_computation is None:
        raise NotImplementedError("give CFLBased(cfl) or Adaptive()")
    semi = lw_update.p
    n_pairs = install_limiters(semi, limiters)
    if isinstance(time_step_computation, Adaptive):
        tsc = time_step_computation
        semi_ = lw_update.p
        on_host_only = (semi_.mesh.n_boundaries > 0 and semi_.time_dependent_boundaries()) or \
            any(getattr(cb, "interval", 0) for cb in callbacks)
        if getattr(tsc, "on_device", False) and not on_host_only:
            return _solve_adaptive_device(lw_update, callbacks, dt_initial, tolerances, n_pairs > 0, tsc.chunk)
        return _solve_adaptive(lw_update, callbacks, dt_initial, tolerances, n_pairs > 0)
    assert isinstance(time_step_computation, CFLBased)
    cfl = time_step_computation.cfl_number
    integ = LWIntegrator(lw_update, tolerances)
    u0 = lw_update.u0_ode
    # exterior data first (time-dependent data is set again before every step)
    semi._prepare_boundaries(lw_update.tspan[0], 0.0, 1.0)
    integ.set_state(u0, lw_update.tspan[0])
    if n_pairs:
        check(integ.handle, lib().tlw_apply_positivity_limiter(integ.handle))
    time_dependent_bc = semi.mesh.n_boundaries > 0 and semi.time_dependent_boundaries()
    intervals = [int(cb.interval) for cb in callbacks if getattr(cb, "interval", 0)]
    stride = min(intervals) if intervals else chunk
    while not integ.isfinished():
        if time_dependent_bc:
            # exterior states depend on (t, dt): one step at a time with the dt read back
            u = integ.get_state()
            dt = semi.max_dt(u, cfl)
            dt = min(dt, integ.tspan[1] - integ.t)
            if semi.solver.volume_integral.time_discretization.code == _lib.TLW_MDRK:
                raise NotImplementedError("MDRK with time-dependent Dirichlet data is not built")
            semi._prepare_boundaries(integ.t, dt, 1.0)
            integ.step(1, cfl, fixed_dt=dt, use_graph=False)
        else:
            integ.step(stride, cfl, use_graph=use_graph)
        integ.sync_time()
        for cb in callbacks:
            if getattr(cb, "interval", 0) and integ.iter % int(cb.interval) == 0:
                cb(integ, integ.get_state())
    u = integ.get_state()
    for cb in callbacks:
        cb(integ, u)
    return LWSolution([u], lw_update, [integ.t], integ.stats)


CONTROLLER = (0.6, -0.2, 0.0)   # (beta1, beta2, beta3), src/solvers/lwfr.jl:162


def dt_factor(epsilon: dict, k: int, controller=CONTROLLER) -> float:
    """dt_factor (src/solvers/adaptive.jl:94-99): 1 + atan(eps_1^(b1/k) eps_0^(b2/k) eps_-1^(b3/k) - 1)."""
    b1, b2, b3 = controller
    f = epsilon[1] ** (b1 / k) * epsilon[0] ** (b2 / k) * epsilon[-1] ** (b3 / k)
    return 1.0 + math.atan(f - 1.0)


# next dt relative to |t| at or below which a run of rejections stops (the device controller has the same)
ADAPTIVE_DT_FLOOR = 1e-14


class AdaptiveController:
    """The step-size logic of perform_step!(..., ::Adaptive, ::LW) (src/solvers/adaptive.jl:101-172), apart
    from the trial step itself: ``propose`` gives the dt to try, ``judge`` takes the trial's total temporal
    error and admissibility and says whether to accept; the epsilon history is updated as
    load_temporal_errors! does (shifted only on the first try of a step)."""

    def __init__(self, nnodes: int, t0: float, t_end: float, dt_initial: float):
        self.k = nnodes
        self.t_end = t_end
        self.t = t0
        self.epsilon = {-1: 1.0, 0: 1.0, 1: 1.0}
        self.n_fail = 0
        self.nreject = 0
        self.iter = 0
        self.dt = self._clamp(dt_initial)
        self.factor = 1.0

    def _clamp(self, dt):   # set_dt!
        return self.t_end - self.t if self.t + dt > self.t_end else dt

    def judge(self, total_error: float, admissible: bool) -> bool:
        if self.n_fail == 0:
            self.epsilon[-1], self.epsilon[0] = self.epsilon[0], self.epsilon[1]
        if math.isfinite(total_error):   # a trial with non-finite values keeps the previous estimate
            self.epsilon[1] = 1.0 / (total_error + 1e-12)
        self.factor = dt_factor(self.epsilon, self.k)
        if admissible and not self.factor <= 0.81:
            self.nreject += self.n_fail
            self.n_fail = 0
            dt = self.dt
            self.t += dt
            self.iter += 1
            self.dt = self._clamp(min(self.factor, 1.5) * dt)
            return True
        self.n_fail += 1
        self.dt = self._clamp(min(self.factor, 0.95) * self.dt)
        if not self.dt > ADAPTIVE_DT_FLOOR * max(abs(self.t), abs(self.t_end)) and not self.finished():
            # the reference retries for ever; stop once dt no longer moves t (the device controller's floor)
            raise DomainError(f"Adaptive: dt fell to {self.dt:.3e} at t = {self.t} after {self.n_fail} rejections")
        return False

    def finished(self) -> bool:
        te = self.t_end
        return self.t == te or abs(self.t - te) <= math.sqrt(np.finfo(float).eps) * max(abs(self.t), abs(te))


def _solve_adaptive(lw_update: LWUpdate, callbacks, dt_initial: float, tolerances, limit: bool = False) -> LWSolution:
    semi = lw_update.p
    tol = tolerances or {"abstol": 1e-6, "reltol": 1e-6}
    integ = LWIntegrator(lw_update, tol)
    semi._prepare_boundaries(lw_update.tspan[0], 0.0, 1.0)
    integ.set_state(lw_update.u0_ode, lw_update.tspan[0])
    if limit:   # the trial and the accept apply it after that (tlw_adaptive_trial / tlw_adaptive_accept)
        check(integ.handle, lib().tlw_apply_positivity_limiter(integ.handle))
    ctl = AdaptiveController(semi.nnodes, lw_update.tspan[0], lw_update.tspan[1], dt_initial)
    err = ctypes.c_double()
    ok = ctypes.c_int32()
    # time-dependent exterior data is set for every trial's (t, dt)
    time_dependent_bc = semi.mesh.n_boundaries > 0 and semi.time_dependent_boundaries()
    while not ctl.finished():
        dt = ctl.dt
        if time_dependent_bc:
            semi._prepare_boundaries(ctl.t, dt, 1.0)
        check(integ.handle, lib().tlw_adaptive_trial(integ.handle, float(dt), float(tol["abstol"]),
                                                     float(tol["reltol"]), ctypes.byref(err), ctypes.byref(ok)))
        if ctl.judge(err.value, bool(ok.value)):
            check(integ.handle, lib().tlw_adaptive_accept(integ.handle, float(dt)))
            for cb in callbacks:
                if getattr(cb, "interval", 0) and ctl.iter % int(cb.interval) == 0:
                    cb(integ, integ.get_state())
    integ.sync_time()
    integ.stats.nreject = ctl.nreject
    u = integ.get_state()
    for cb in callbacks:
        cb(integ, u)
    return LWSolution([u], lw_update, [integ.t], integ.stats)


def _solve_adaptive_device(lw_update: LWUpdate, callbacks, dt_initial: float, tolerances, limit: bool,
                           chunk: int) -> LWSolution:
    """Adaptive stepping with the controller on the device: chunks of trials without host round trips."""
    semi = lw_update.p
    tol = tolerances or {"abstol": 1e-6, "reltol": 1e-6}
    integ = LWIntegrator(lw_update, tol)
    semi._prepare_boundaries(lw_update.tspan[0], 0.0, 1.0)
    integ.set_state(lw_update.u0_ode, lw_update.tspan[0])
    if limit:
        check(integ.handle, lib().tlw_apply_positivity_limiter(integ.handle))
    beta = (ctypes.c_double * 3)(*CONTROLLER)
    check(integ.handle, lib().tlw_adaptive_begin(integ.handle, float(lw_update.tspan[1]), float(dt_initial), beta))
    steps, rejected, finished = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    while True:
        check(integ.handle, lib().tlw_adaptive_run(integ.handle, int(chunk), float(tol["abstol"]),
                                                   float(tol["reltol"]), ctypes.byref(steps),
                                                   ctypes.byref(rejected), ctypes.byref(finished)))
        if finished.value:
            break
    integ.sync_time()
    integ.stats.nreject = int(rejected.value)
    u = integ.get_state()
    for cb in callbacks:
        cb(integ, u)
    return LWSolution([u], lw_update, [integ.t], integ.stats)


def l2_linf_errors(semi: SemidiscretizationHyperbolic, u_ode: np.ndarray, t: float, exact=None):
    """Per-variable L2 and Linf errors against ``exact`` (default: the initial condition at t), L2 by GLL
    quadrature on the solution nodes: sqrt(sum_e sum_ij w_i w_j |J_e| (u - u_exact)^2 / |domain|)."""
    exact = exact or semi.initial_condition
    xy = semi.node_coordinates
    ue = semi.compute_coefficients(t) if exact is semi.initial_condition else None
    if ue is None:
        v = exact(xy[0], xy[1], t, semi.equations)
        ue = np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)
    n = semi.nnodes
    _, w = gauss_lobatto(semi.polydeg)
    d = (u_ode - ue).reshape(-1, n, n, 4)
    ww = (w[None, :, None] * w[None, None, :])      # [1, j, i]
    if getattr(semi, "curved", None) is not None:
        # curvilinear: |J| per node, domain area from the same quadrature
        l2 = np.sqrt(np.einsum("ejiv,eji->v", d * d, ww * semi.curved.jacobian_nodes()) / semi.curved.area)
    else:
        jac = 1.0 / semi.mesh.inverse_jacobian          # |J| = h/2 per direction -> area factor jac^2
        l2 = np.sqrt(np.einsum("ejiv,eji->v", d * d, ww * (jac ** 2)[:, None, None]) / semi.mesh.length ** 2)
    linf = np.abs(d).max(axis=(0, 1, 2))
    return l2, linf
