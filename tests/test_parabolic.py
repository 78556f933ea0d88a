"""Compressible Navier-Stokes (LW, BR1 gradients of the conservative variables, periodic TreeMesh{2}):
the oracle's properties on the CPU (mu = 0 is Euler, free stream, conservation, the viscous decay rate of a
shear wave) and libtlw's parabolic kernels against the oracle on the GPU (1e-12 relative L2 per variable)."""
import os

import numpy as np
import pytest

NTH = os.cpu_count() or 1


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def vortex(tl, mesh, N):
    eq = tl.CompressibleEulerEquations2D(1.4)
    xy = mesh.node_coordinates(N)
    v = tl.IsentropicVortex(5.0, center=(0.7, -0.4))(xy[0], xy[1], 0.0, eq)
    return np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)


def shear_wave(tl, mesh, N, A=1e-3):
    """rho = 1, p = 1, v = (0, A sin(2 pi (x + 10) / 20)) on [-10, 10]^2."""
    eq = tl.CompressibleEulerEquations2D(1.4)
    xy = mesh.node_coordinates(N)
    k = 2 * np.pi / 20.0
    one = np.ones_like(xy[0])
    U = eq.prim2cons(one, 0 * one, A * np.sin(k * (xy[0] + 10.0)), one)
    return np.ascontiguousarray(np.transpose(U, (2, 1, 0, 3))).reshape(-1), k


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("N", [3, 4, 5])
def test_oracle_navier_stokes_properties(oracle_mod, tl, N):
    from trixilw.basis import gauss_lobatto
    m = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    u = vortex(tl, m, N)
    euler, ns0, ns = oracle_mod.Oracle(m, N), oracle_mod.Oracle(m, N), oracle_mod.Oracle(m, N)
    ns0.set_parabolic(0.0)
    ns.set_parabolic(0.05)
    dt = euler.max_dt(u, 0.4)
    d_e = euler.rhs(u, 0.0, dt)
    assert np.all(rel_l2(ns0.rhs(u, 0.0, dt), d_e) < 1e-13)
    uc = np.tile(np.array([1.0, 0.3, -0.2, 2.5]), m.n_elements * (N + 1) ** 2)
    assert np.abs(ns.rhs(uc, 0.0, 0.01)).max() < 1e-12
    du = ns.rhs(u, 0.0, ns.max_dt(u, 0.4))
    _, w = gauss_lobatto(N)
    tot = np.einsum("ejiv,e,j,i->v", du.reshape(-1, N + 1, N + 1, 4), (1.0 / m.inverse_jacobian) ** 2, w, w)
    assert np.all(np.abs(tot) < 1e-11)


def test_oracle_shear_wave_decays_at_the_viscous_rate(oracle_mod, tl):
    """A small shear wave decays as exp(-mu/rho k^2 t) (linearised Navier-Stokes)."""
    N, mu, T = 4, 0.2, 2.0
    m = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    u, k = shear_wave(tl, m, N)
    o = oracle_mod.Oracle(m, N)
    o.set_parabolic(mu)
    s, t = o.steps(u, 10 ** 6, 0.5, 0.0, T, nthreads=NTH)
    assert t == T
    xy = m.node_coordinates(N)
    v2 = u.reshape(-1, N + 1, N + 1, 4)[..., 2] / u.reshape(-1, N + 1, N + 1, 4)[..., 0]
    ref = 1e-3 * np.sin(k * (np.transpose(xy[0], (2, 1, 0)) + 10.0)) * np.exp(-mu * k * k * T)
    assert np.abs(v2 - ref).max() < 1e-4 * 1e-3


# ---------------------------------------------------------------------------------------------- GPU
def make_semi(tl, mesh, N, mu):
    eq = tl.CompressibleEulerEquations2D(1.4)
    eq_par = tl.CompressibleNavierStokesDiffusion2D(eq, mu=mu, Prandtl=0.72,
                                                    gradient_variables=tl.GradientVariablesConservative())
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    return tl.SemidiscretizationHyperbolicParabolic(mesh, (eq, eq_par), tl.IsentropicVortex(5.0), solver)


@pytest.mark.gpu
@pytest.mark.parametrize("N", [3, 4, 5, 6, 7])
@pytest.mark.parametrize("mu", [0.0, 0.01, 0.1])
def test_gpu_navier_stokes_rhs_matches_oracle(oracle_mod, tl, N, mu):
    m = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    semi = make_semi(tl, m, N, mu)
    u = vortex(tl, m, N)
    o = oracle_mod.Oracle(m, N)
    o.set_parabolic(mu)
    dt = o.max_dt(u, 0.3)
    assert semi.max_dt(u, 0.3) == pytest.approx(dt, rel=1e-13)
    du_cpu = o.rhs(u, 0.0, dt)
    semi.cache["dt"][0] = dt
    du_gpu = np.empty_like(u)
    tl.rhs(du_gpu, u, semi, 0.0)
    assert np.all(rel_l2(u + dt * du_gpu, u + dt * du_cpu) < 1e-12)
    assert np.all(rel_l2(du_gpu, du_cpu) < 1e-11)


@pytest.mark.gpu
def test_gpu_navier_stokes_steps_match_oracle(oracle_mod, tl):
    m = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    semi = make_semi(tl, m, 4, 0.05)
    u0 = vortex(tl, m, 4)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(9, 0.4, use_graph=True)
    integ.sync_time()
    u_gpu = integ.get_state()
    o = oracle_mod.Oracle(m, 4)
    o.set_parabolic(0.05)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, 9, 0.4, 0.0, 1e9, nthreads=NTH)
    assert s == integ.iter == 9 and integ.t == pytest.approx(t, rel=1e-13)
    assert np.all(rel_l2(u_gpu, u_cpu) < 1e-12)


@pytest.mark.gpu
def test_gpu_shear_wave_decay(tl):
    N, mu, T = 4, 0.2, 2.0
    m = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 4)
    semi = make_semi(tl, m, N, mu)
    u0, k = shear_wave(tl, m, N)
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, T)))
    integ.set_state(u0, 0.0)
    while not integ.isfinished():
        integ.step(200, 0.5)
        integ.sync_time()
    u = integ.get_state()
    xy = m.node_coordinates(N)
    v2 = u.reshape(-1, N + 1, N + 1, 4)[..., 2] / u.reshape(-1, N + 1, N + 1, 4)[..., 0]
    ref = 1e-3 * np.sin(k * (np.transpose(xy[0], (2, 1, 0)) + 10.0)) * np.exp(-mu * k * k * T)
    assert np.abs(v2 - ref).max() < 1e-4 * 1e-3
