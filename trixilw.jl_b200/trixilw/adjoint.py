"""Differentiable form of the LW solve: a hand-written discrete adjoint of the full LW step (libtlw,
``tlw_adjoint_*``), a checkpointed reverse sweep over a run, and a ``torch.autograd.Function`` around the
solve (the counterpart of the ChainRulesCore ``rrule`` a Julia caller would define).

The map differentiated is the reference's step u_new = u + dt * rhs(u) (src/solvers/dgsem_tree/dg_2d.jl:28-83,
perform_step! src/solvers/lwfr.jl:212-230) on a periodic TreeMesh{2} with the plain FR volume integral and
the Rusanov surface flux, N = 3, 4, 5; the dt of every step is recorded on the forward sweep and held fixed
on the reverse sweep. The reference itself has no adjoint.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib
from .semidiscretization import SemidiscretizationHyperbolic

_DP = ctypes.POINTER(ctypes.c_double)


def _host(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def adjoint_step(semi: SemidiscretizationHyperbolic, lam: np.ndarray, u: np.ndarray, dt: float) -> np.ndarray:
    """(d u_new / d u)^T lam for one LW step from u at the given dt."""
    lam, u = _host(lam), _host(u)
    out = np.empty_like(u)
    check(semi.handle, lib().tlw_adjoint_step(semi.handle, _p(out), _p(lam), _p(u), float(dt), _lib.TLW_WHERE_HOST))
    return out


def solve_dts(semi: SemidiscretizationHyperbolic, u0: np.ndarray, dts) -> np.ndarray:
    """Forward LW solve from u0 with the given dt sequence; returns u(T)."""
    u0 = _host(u0)
    dts = _host(dts)
    out = np.empty_like(u0)
    check(semi.handle, lib().tlw_solve_dts(semi.handle, _p(u0), int(dts.size), dts.ctypes.data_as(_DP), _p(out),
                                           _lib.TLW_WHERE_HOST))
    return out


def forward_record(semi: SemidiscretizationHyperbolic, u0: np.ndarray, nsteps: int, cfl: float,
                   checkpoint_every: int = 20) -> np.ndarray:
    """CFL forward sweep that records the dt sequence and checkpoints; returns u(T)."""
    u0 = _host(u0)
    out = np.empty_like(u0)
    check(semi.handle, lib().tlw_forward_record(semi.handle, _p(u0), int(nsteps), float(cfl), int(checkpoint_every),
                                                _p(out), _lib.TLW_WHERE_HOST))
    return out


def dt_sequence(semi: SemidiscretizationHyperbolic, nsteps: int) -> np.ndarray:
    out = np.empty(int(nsteps))
    check(semi.handle, lib().tlw_adjoint_dt_sequence(semi.handle, out.ctypes.data_as(_DP), int(nsteps)))
    return out


def adjoint_sweep(semi: SemidiscretizationHyperbolic, lam_T: np.ndarray, timing: bool = False):
    """(d u(T) / d u0)^T lam_T of the recorded run; with timing, also (recompute_ms, adjoint_ms)."""
    lam_T = _host(lam_T)
    out = np.empty_like(lam_T)
    ph = (ctypes.c_double * 2)() if timing else None
    check(semi.handle, lib().tlw_adjoint_sweep(semi.handle, _p(lam_T), _p(out), _lib.TLW_WHERE_HOST, ph))
    return (out, (ph[0], ph[1])) if timing else out


def adjoint_solve(semi: SemidiscretizationHyperbolic, u0: np.ndarray, nsteps: int, cfl: float,
                  checkpoint_every: int, rho_target: np.ndarray, timing: bool = False):
    """J = 1/2 sum_nodes (rho(T) - rho_target)^2 and dJ/du0 by the checkpointed discrete adjoint.

    Returns (J, grad, u(T)) and, with timing, the device milliseconds of (forward, recompute, adjoint)."""
    u0 = _host(u0)
    rho_target = _host(rho_target)
    grad = np.empty_like(u0)
    uT = np.empty_like(u0)
    J = ctypes.c_double()
    ph = (ctypes.c_double * 3)() if timing else None
    check(semi.handle, lib().tlw_adjoint_solve(semi.handle, _p(u0), int(nsteps), float(cfl), int(checkpoint_every),
                                               _p(rho_target), _p(grad), ctypes.byref(J), _p(uT),
                                               _lib.TLW_WHERE_HOST, ph))
    if timing:
        return J.value, grad, uT, (ph[0], ph[1], ph[2])
    return J.value, grad, uT


try:
    import torch

    class LWSolve(torch.autograd.Function):
        """u(T) = solve(u0): nsteps CFL LW steps; backward = the checkpointed discrete adjoint with the
        forward run's dt sequence held fixed. Tensors are float64, on the CPU or on the handle's GPU."""

        @staticmethod
        def forward(ctx, u0, semi, nsteps, cfl, checkpoint_every):
            x = u0.detach().contiguous().to(torch.float64)
            where = _lib.TLW_WHERE_DEVICE if x.is_cuda else _lib.TLW_WHERE_HOST
            out = torch.empty_like(x)
            if x.is_cuda:
                torch.cuda.current_stream(x.device).synchronize()
            check(semi.handle, lib().tlw_forward_record(semi.handle, ctypes.c_void_p(x.data_ptr()), int(nsteps),
                                                        float(cfl), int(checkpoint_every),
                                                        ctypes.c_void_p(out.data_ptr()), where))
            semi._adjoint_record = getattr(semi, "_adjoint_record", 0) + 1
            ctx.semi = semi
            ctx.record = semi._adjoint_record
            return out

        @staticmethod
        def backward(ctx, grad_out):
            semi = ctx.semi
            if semi._adjoint_record != ctx.record:
                raise RuntimeError("the handle recorded another forward run after this one; run backward first")
            g = grad_out.detach().contiguous().to(torch.float64)
            where = _lib.TLW_WHERE_DEVICE if g.is_cuda else _lib.TLW_WHERE_HOST
            out = torch.empty_like(g)
            if g.is_cuda:
                torch.cuda.current_stream(g.device).synchronize()
            check(semi.handle, lib().tlw_adjoint_sweep(semi.handle, ctypes.c_void_p(g.data_ptr()),
                                                       ctypes.c_void_p(out.data_ptr()), where, None))
            return out, None, None, None, None

    def lw_solve(u0, semi: SemidiscretizationHyperbolic, nsteps: int, cfl: float, checkpoint_every: int = 20):
        """Differentiable LW solve (``torch.autograd``)."""
        return LWSolve.apply(u0, semi, nsteps, cfl, checkpoint_every)

except ImportError:  # pragma: no cover - torch is optional for the rest of the package
    LWSolve = None
    lw_solve = None
