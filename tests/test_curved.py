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
