"""Compressible Euler 2D on the host: state conversions and the initial/boundary conditions of the
workloads (vectorised numpy; the device library evaluates fluxes itself)."""
from __future__ import annotations

import numpy as np


class GradientVariablesConservative:
    """Gradients of the conservative variables (the reference's GradientVariablesConservative,
    src/equations/compressible_navier_stokes_2d.jl:14)."""


class CompressibleNavierStokesDiffusion2D:
    """Trixi's CompressibleNavierStokesDiffusion2D(equations; mu, Prandtl, gradient_variables): constant dynamic
    viscosity mu, Prandtl number, T = p / rho, kappa = gamma / ((gamma - 1) Pr). The device path takes the
    conservative gradient variables, as the reference's Navier-Stokes setups do."""

    def __init__(self, equations, mu: float, Prandtl: float = 0.72, gradient_variables=None):
        self.equations_hyperbolic = equations
        self.gamma = equations.gamma
        self.mu = float(mu)
        self.Pr = float(Prandtl)
        if gradient_variables is not None and not isinstance(gradient_variables, GradientVariablesConservative):
            raise NotImplementedError("the device path takes GradientVariablesConservative")


class CompressibleEulerEquations2D:
    """Trixi's CompressibleEulerEquations2D(gamma): variables (rho, rho v1, rho v2, rho e)."""

    nvariables = 4

    def __init__(self, gamma: float = 1.4):
        self.gamma = float(gamma)

    def prim2cons(self, rho, v1, v2, p):
        rho = np.asarray(rho, dtype=np.float64)
        e = p / (self.gamma - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2)
        return np.stack(np.broadcast_arrays(rho, rho * v1, rho * v2, e), axis=-1)

    def cons2prim(self, u):
        u = np.asarray(u)
        rho = u[..., 0]
        v1 = u[..., 1] / rho
        v2 = u[..., 2] / rho
        p = (self.gamma - 1.0) * (u[..., 3] - 0.5 * (u[..., 1] * v1 + u[..., 2] * v2))
        return rho, v1, v2, p


def initial_condition_convergence_test(x, y, t, eq: CompressibleEulerEquations2D):
    """Trixi's initial_condition_convergence_test: rho = rho v1 = rho v2 = c + A sin(w (x + y - t)), rho e = rho^2
    (c = 2, A = 0.1, L = 2, w = 2 pi / L), a smooth periodic solution on [0, 2]^2 when the source below is added."""
    c, A, L = 2.0, 0.1, 2.0
    w = 2.0 * np.pi / L
    ini = c + A * np.sin(w * (np.asarray(x, dtype=np.float64) + y - t))
    return np.stack(np.broadcast_arrays(ini, ini, ini, ini * ini), axis=-1)


class _SourceTermsConvergenceTest:
    """Trixi's source_terms_convergence_test(u, x, t, equations) for CompressibleEulerEquations2D: the source that
    makes initial_condition_convergence_test an exact solution (independent of u). The device evaluates it in the
    volume kernels (source kind 1); this host form is for checks."""

    kind = 1

    def __call__(self, u, x, y, t, eq: CompressibleEulerEquations2D):
        c, A, L = 2.0, 0.1, 2.0
        w = 2.0 * np.pi / L
        arg = w * (np.asarray(x, dtype=np.float64) + y - t)
        rho = c + A * np.sin(arg)
        rho_x = w * A * np.cos(arg)
        tmp = (2.0 * rho - 1.0) * (eq.gamma - 1.0)
        s2 = rho_x * (1.0 + tmp)
        return np.stack(np.broadcast_arrays(rho_x, s2, s2, 2.0 * rho_x * (rho + tmp)), axis=-1)


source_terms_convergence_test = _SourceTermsConvergenceTest()


class IsentropicVortex:
    """Isentropic vortex (Shu's form): background rho = 1, v = (1, 1), p = 1; strength beta, centre c;
    T = 1 - (gamma-1) beta^2 / (8 gamma pi^2) exp(1 - r^2), rho = T^(1/(gamma-1)), p = rho T,
    v += beta/(2 pi) exp((1 - r^2)/2) (-dy, dx). The exact solution at time t is the initial state
    advected by (t, t), wrapped periodically into the domain [lo, hi]^2."""

    def __init__(self, strength=5.0, center=(0.0, 0.0), domain=(-10.0, 10.0), velocity=(1.0, 1.0)):
        self.beta = float(strength)
        self.center = np.asarray(center, dtype=np.float64)
        self.lo, self.hi = float(domain[0]), float(domain[1])
        self.velocity = np.asarray(velocity, dtype=np.float64)

    def __call__(self, x, y, t, eq: CompressibleEulerEquations2D):
        L = self.hi - self.lo
        cx = self.center[0] + self.velocity[0] * t
        cy = self.center[1] + self.velocity[1] * t
        dx = x - cx
        dy = y - cy
        dx = dx - L * np.round(dx / L)
        dy = dy - L * np.round(dy / L)
        r2 = dx * dx + dy * dy
        g = eq.gamma
        T = 1.0 - (g - 1.0) * self.beta ** 2 / (8.0 * g * np.pi ** 2) * np.exp(1.0 - r2)
        rho = T ** (1.0 / (g - 1.0))
        du = self.beta / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2))
        v1 = self.velocity[0] - du * dy
        v2 = self.velocity[1] + du * dx
        p = rho * T
        return eq.prim2cons(rho, v1, v2, p)


class FourQuadrantRiemann:
    """Four-quadrant 2D Riemann problem on [0,1]^2 split at (0.5, 0.5): the classic configuration with
    rho in {1.5, 0.5323, 0.138, 0.5323}, p in {1.5, 0.3, 0.029, 0.3} and velocities 0 / 1.206 (quadrants
    +x+y, -x+y, -x-y, +x-y). Constant in time: used as initial and Dirichlet boundary data."""

    states = {  # (rho, v1, v2, p)
        1: (1.5, 0.0, 0.0, 1.5),
        2: (0.5323, 1.206, 0.0, 0.3),
        3: (0.138, 1.206, 1.206, 0.029),
        4: (0.5323, 0.0, 1.206, 0.3),
    }
    time_independent = True

    def __call__(self, x, y, t, eq: CompressibleEulerEquations2D):
        x, y = np.broadcast_arrays(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64))
        q = np.where(x >= 0.5, np.where(y >= 0.5, 1, 4), np.where(y >= 0.5, 2, 3))
        prim = np.zeros(x.shape + (4,))
        for k, s in self.states.items():
            prim[q == k] = s
        return eq.prim2cons(prim[..., 0], prim[..., 1], prim[..., 2], prim[..., 3])


class ConstantState:
    """Free stream (rho, v1, v2, p)."""

    time_independent = True

    def __init__(self, rho=1.0, v1=0.3, v2=-0.2, p=1.0):
        self.prim = (rho, v1, v2, p)

    def __call__(self, x, y, t, eq: CompressibleEulerEquations2D):
        x, y = np.broadcast_arrays(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64))
        rho, v1, v2, p = self.prim
        return eq.prim2cons(np.full(x.shape, rho), v1, v2, p)


class DensityWave:
    """rho = 1 + A sin(2 pi k (x + y - (v1 + v2) t)), v = (v1, v2), p = p0 (exact advection solution)."""

    def __init__(self, amplitude=0.5, v=(0.1, 0.2), p=1.0, k=1.0):
        self.A, self.v, self.p, self.k = amplitude, v, p, k

    def __call__(self, x, y, t, eq: CompressibleEulerEquations2D):
        rho = 1.0 + self.A * np.sin(2 * np.pi * self.k * (x + y - (self.v[0] + self.v[1]) * t))
        return eq.prim2cons(rho, self.v[0], self.v[1], self.p)
