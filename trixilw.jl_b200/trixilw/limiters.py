"""Stage limiters: Trixi's PositivityPreservingLimiterZhangShu as TrixiLW applies it after a step
(src/callbacks/callbacks_stage/positivity_zhang_shu.jl:10-42, positivity_zhang_shu_dg2d.jl:8-176).

The limiter runs on the device inside libtlw's step (``tlw_set_positivity_limiter``): one fused pass over
the state per step that applies every (threshold, variable) pair in order, element pass then the TreeMesh
mortar pass. ``solve_lwfr(..., limiters=(limiter,))`` installs it; several limiters in the tuple are applied
in order, which is the same as one limiter with their pairs concatenated (at most four pairs in all).
"""
from __future__ import annotations

import numpy as np

from . import _lib


def density(u, equations=None):
    """Trixi density(u, equations): the first conservative variable (last axis of u holds the variables)."""
    return np.asarray(u)[..., 0]


def pressure(u, equations=None):
    """Trixi pressure(u, equations::CompressibleEulerEquations2D) = (gamma - 1)(rho_e - |rho v|^2 / (2 rho))."""
    u = np.asarray(u)
    gamma = getattr(equations, "gamma", 1.4)
    return (gamma - 1.0) * (u[..., 3] - 0.5 * (u[..., 1] ** 2 + u[..., 2] ** 2) / u[..., 0])


def density_pressure(u, equations=None):
    """Trixi density_pressure(u, equations) = rho p = (gamma - 1)(rho rho_e - |rho v|^2 / 2)."""
    u = np.asarray(u)
    gamma = getattr(equations, "gamma", 1.4)
    return (gamma - 1.0) * (u[..., 3] * u[..., 0] - 0.5 * (u[..., 1] ** 2 + u[..., 2] ** 2))


_CODES = {density: _lib.TLW_LIMIT_DENSITY, pressure: _lib.TLW_LIMIT_PRESSURE,
          density_pressure: _lib.TLW_LIMIT_DENSITY_PRESSURE}
MAX_PAIRS = 4


class PositivityPreservingLimiterZhangShu:
    """PositivityPreservingLimiterZhangShu(; thresholds, variables) (Trixi): for each pair, elements whose
    minimum of ``variable`` is below ``threshold`` are blended towards their mean so that the minimum becomes
    the threshold; on a TreeMesh with mortars each large element is also limited on its mortar traces."""

    def __init__(self, thresholds, variables):
        thresholds = tuple(float(t) for t in thresholds)
        variables = tuple(variables)
        if len(thresholds) != len(variables):
            raise ValueError("thresholds and variables must have the same length")
        codes = []
        for v in variables:
            if v not in _CODES:
                raise ValueError(f"variable {v!r} is not built: density, pressure or density_pressure")
            codes.append(_CODES[v])
        if not all(np.isfinite(thresholds)):
            raise ValueError("thresholds must be finite")
        self.thresholds = thresholds
        self.variables = variables
        self.codes = tuple(codes)

    def __call__(self, u_ode, integrator, semi, t):
        """limiter!(u_ode, integrator, semi, t): one application to the integrator's device state."""
        install(semi, (self,))
        _lib.check(semi.handle, _lib.lib().tlw_apply_positivity_limiter(semi.handle))


def pairs(limiters) -> tuple[tuple[float, ...], tuple[int, ...]]:
    thr, var = [], []
    for lim in limiters:
        if not isinstance(lim, PositivityPreservingLimiterZhangShu):
            raise NotImplementedError(f"limiter {type(lim).__name__} is not built on the device path")
        thr.extend(lim.thresholds)
        var.extend(lim.codes)
    if len(thr) > MAX_PAIRS:
        raise ValueError(f"at most {MAX_PAIRS} (threshold, variable) pairs in all")
    return tuple(thr), tuple(var)


def install(semi, limiters) -> int:
    """Sets the handle's limiter pairs (none: off); returns the number of pairs."""
    thr, var = pairs(limiters)
    t = np.ascontiguousarray(thr if thr else [0.0], dtype=np.float64)
    v = np.ascontiguousarray(var if var else [0], dtype=np.int32)
    _lib.check(semi.handle, _lib.lib().tlw_set_positivity_limiter(
        semi.handle, len(thr), t.ctypes.data, v.ctypes.data))
    return len(thr)
