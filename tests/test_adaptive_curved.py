"""Adaptive (error-controlled) LW stepping on curvilinear meshes and with shock capturing: the temporal error
estimate of the curvilinear LW kernels (src/solvers/dgsem_structured/dg_2d.jl:1595-1682 at depth 3,
:1983-2075 at depth 4) and of the TreeMesh kernel under VolumeIntegralFRShockCapturing (which calls the same
kernel for every element, dg_2d.jl:1648-1804). The oracle's estimate is checked on the CPU against the TreeMesh
one (affine mesh), under element rotations and against the blending factors; libtlw's device trial step
and whole adaptive runs against the oracle on the GPU."""
import ctypes
import math
import os

import numpy as np
import pytest

from test_adaptive import TOL, oracle_adaptive
from test_curved import rel_l2, vortex_state, warp
from test_curved_sc import RECONSTRUCTIONS, blast_state

NTH = os.cpu_count() or 1


def affine(xi, eta):
    return 10.0 * xi, 10.0 * eta


def total_error(o, n_elements, N):
    return math.sqrt(np.sum(o.get(4)) / (n_elements * (N + 1) ** 2))


def oracle(oracle_mod, mesh, N, sc_rec=None):
    o = oracle_mod.Oracle(mesh, N)
    o.set_temporal_errors(True, TOL["abstol"], TOL["reltol"])
    if sc_rec is not None:
        o.set_shock_capturing(True, alpha_max=0.5, alpha_min=0.001, alpha_smooth=True, reconstruction=sc_rec)
    return o


# ---------------------------------------------------------------------------------------------- CPU
def test_oracle_curved_estimate_equals_the_tree_one_on_an_affine_mesh(oracle_mod, tl):
    """N = 4: the curvilinear depth-4 estimate on the affine 8x8 StructuredMesh of [-10, 10]^2 sums to the
    TreeMesh estimate (same elements in another order)."""
    N = 4
    sm = tl.StructuredMesh((8, 8), affine)
    cm = sm.curved(N)
    tm = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
    eq = tl.CompressibleEulerEquations2D(1.4)
    xy = tm.node_coordinates(N)
    v = tl.IsentropicVortex(5.0, center=(0.7, -0.4))(xy[0], xy[1], 0.0, eq)
    ut = np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)
    uc = vortex_state(tl, cm)
    ot, oc = oracle(oracle_mod, tm, N), oracle(oracle_mod, sm, N)
    dt = ot.max_dt(ut, 0.5)
    ot.rhs(ut, 0.0, dt)
    oc.rhs(uc, 0.0, dt)
    et, ec = ot.get(4), oc.get(4)
    assert np.all(np.isfinite(ec)) and ec.max() > 0.0
    assert np.sum(ec) == pytest.approx(np.sum(et), rel=1e-9)
    assert np.sort(ec) == pytest.approx(np.sort(et), rel=1e-6, abs=1e-12 * et.max())


@pytest.mark.parametrize("N", [3, 4])
def test_oracle_curved_estimate_invariant_under_element_rotations(oracle_mod, tl, N):
    m = tl.StructuredMesh((5, 4), warp)
    cm = m.curved(N)
    turns = np.random.default_rng(N + 3).integers(0, 4, cm.n_elements)
    rm = tl.rotate_elements(cm, turns)
    u = vortex_state(tl, cm)
    o, o2 = oracle(oracle_mod, m, N), oracle(oracle_mod, rm, N)
    dt = o.max_dt(u, 0.4)
    o.rhs(u, 0.0, dt)
    o2.rhs(tl.rotate_state(u, N, turns), 0.0, dt)
    e1, e2 = o.get(4), o2.get(4)
    assert e1.max() > 1.0
    np.testing.assert_allclose(e2, e1, rtol=1e-8, atol=1e-10 * e1.max())


@pytest.mark.parametrize("rec", [0, 2])
def test_oracle_estimate_does_not_depend_on_the_blending(oracle_mod, tl, rec):
    """The shock-capturing path calls the LW kernel for every element with the DG weight 1 - alpha, and the
    estimate does not involve that weight: it equals the estimate of the plain FR volume integral."""
    N = 4
    m = tl.StructuredMesh((6, 6), warp)
    cm = m.curved(N)
    u = blast_state(cm)
    o_sc, o_fr = oracle(oracle_mod, m, N, sc_rec=rec), oracle(oracle_mod, m, N)
    dt = o_fr.max_dt(u, 0.2)
    o_sc.rhs(u, 0.0, dt)
    o_fr.rhs(u, 0.0, dt)
    assert o_sc.get(6).max() > 0.1                   # some elements are blended
    np.testing.assert_array_equal(o_sc.get(4), o_fr.get(4))


def test_oracle_curved_adaptive_run(oracle_mod, tl):
    m = tl.StructuredMesh((6, 6), warp)
    cm = m.curved(3)
    u, ctl, dts = oracle_adaptive(oracle_mod, m, 3, vortex_state(tl, cm), 0.5, 1e-3)
    assert ctl.t == 0.5 and ctl.iter == len(dts) and 3 < ctl.iter < 200
    assert max(dts) > 10 * dts[0]
    assert np.all(np.isfinite(u))


# ---------------------------------------------------------------------------------------------- GPU
def semi_for(tl, mesh, N, sc_rec=None):
    eq = tl.CompressibleEulerEquations2D(1.4)
    if sc_rec is None:
        vi = tl.VolumeIntegralFR(tl.LW())
    else:
        vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5, alpha_min=0.001),
                                               tl.VolumeIntegralFR(tl.LW()),
                                               reconstruction=RECONSTRUCTIONS[sc_rec](tl))
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, vi)
    return tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, tl.ConstantState(), solver)


def device_trial(tl, semi, u, dt):
    """One tlw_adaptive_trial from u, accepted: (total temporal error, admissible, the trial state)."""
    from trixilw._lib import check, lib
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)), TOL)
    integ.set_state(u, 0.0)
    err, ok = ctypes.c_double(), ctypes.c_int32()
    check(integ.handle, lib().tlw_adaptive_trial(integ.handle, float(dt), TOL["abstol"], TOL["reltol"],
                                                 ctypes.byref(err), ctypes.byref(ok)))
    check(integ.handle, lib().tlw_adaptive_accept(integ.handle, float(dt)))
    return err.value, bool(ok.value), integ.get_state()


CASES = [  # (mesh kind, N, reconstruction or None for the FR volume integral)
    ("curved", 3, None), ("curved", 4, None), ("curved", 5, None), ("curved", 3, 0), ("curved", 4, 1),
    ("curved", 4, 2), ("tree", 4, 0), ("tree", 5, 0)]


@pytest.mark.gpu
@pytest.mark.parametrize("kind,N,rec", CASES)
def test_gpu_trial_estimate_matches_oracle(oracle_mod, tl, kind, N, rec):
    if kind == "curved":
        m = tl.StructuredMesh((8, 8), warp)
        mesh = tl.rotate_elements(m.curved(N), np.random.default_rng(N).integers(0, 4, 64))
        u = blast_state(mesh) if rec is not None else vortex_state(tl, mesh)
    else:
        mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
        eq = tl.CompressibleEulerEquations2D(1.4)
        xy = mesh.node_coordinates(N)
        x, y = xy[0], xy[1]
        inside = (x - 0.5) ** 2 + (y + 0.7) ** 2 < 9.0
        rho = np.where(inside, 1.0, 0.125)
        p = np.where(inside, 10.0, 1.0)
        v = np.stack([rho, 0 * rho, 0 * rho, p / 0.4], axis=-1)
        u = np.ascontiguousarray(np.transpose(v, (2, 1, 0, 3))).reshape(-1)
    o = oracle(oracle_mod, mesh, N, sc_rec=rec)
    if rec is not None:   # a few steps first: nonzero MUSCL slopes, a smeared blast
        o.set_temporal_errors(False)
        o.steps(u, 4, 0.2, 0.0, 1e9, nthreads=NTH)
        o.set_temporal_errors(True, TOL["abstol"], TOL["reltol"])
    dt = o.max_dt(u, 0.3)
    du = o.rhs(u, 0.0, dt, nthreads=NTH)
    e_cpu = total_error(o, mesh.n_elements, N)
    e_gpu, ok, u_gpu = device_trial(tl, semi_for(tl, mesh, N, rec), u, dt)
    assert ok and e_cpu > 0.0
    assert e_gpu == pytest.approx(e_cpu, rel=1e-8)
    assert np.all(rel_l2(u_gpu, u + dt * du) < 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("rec", [None, 2])
def test_gpu_curved_adaptive_run_matches_oracle(oracle_mod, tl, rec):
    """Whole adaptive runs (N = 4, rotated warped 8x8 mesh; the vortex with the FR volume integral, the blast
    with MUSCL-Hancock shock capturing): the same accepted and rejected steps and the same final state."""
    N = 4
    m = tl.StructuredMesh((8, 8), warp)
    cm = tl.rotate_elements(m.curved(N), np.random.default_rng(11).integers(0, 4, 64))
    u0 = blast_state(cm) if rec is not None else vortex_state(tl, cm)
    t_end = 0.05 if rec is not None else 0.5
    semi = semi_for(tl, cm, N, rec)
    upd = tl.semidiscretize(semi, tl.LW(), (0.0, t_end))
    upd.u0_ode[:] = u0
    sol = tl.solve_lwfr(upd, (), 1e-4, TOL, tl.Adaptive())
    o = oracle_mod.Oracle(cm, N)
    if rec is not None:
        o.set_shock_capturing(True, alpha_max=0.5, alpha_min=0.001, alpha_smooth=True, reconstruction=rec)
    u_cpu, ctl, dts = oracle_adaptive(oracle_mod, cm, N, u0, t_end, 1e-4, oracle_obj=o)
    assert sol.t[0] == t_end and ctl.iter > 3
    assert sol.stats.nreject == ctl.nreject
    assert np.all(rel_l2(sol.u[0], u_cpu) < 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["tree", "curved_sc"])
def test_gpu_device_controller_matches_host_controller(tl, kind):
    """Adaptive(on_device=True): the controller on the device gives the host controller's run (the same
    accepted steps and rejections, the same final state up to the last bits of pow / atan)."""
    if kind == "tree":
        N = 4
        mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 3)
        eq = tl.CompressibleEulerEquations2D(1.4)
        solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
        semi_of = lambda: tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq,
                                                          tl.IsentropicVortex(5.0, center=(0.7, -0.4)), solver)
        u0, t_end, dt0 = None, 1.0, 1e-3
    else:
        N = 4
        m = tl.StructuredMesh((8, 8), warp)
        mesh = tl.rotate_elements(m.curved(N), np.random.default_rng(11).integers(0, 4, 64))
        semi_of = lambda: semi_for(tl, mesh, N, 2)
        u0, t_end, dt0 = blast_state(mesh), 0.05, 1e-4
    runs = []
    for on_device in (False, True):
        semi = semi_of()
        upd = tl.semidiscretize(semi, tl.LW(), (0.0, t_end))
        if u0 is not None:
            upd.u0_ode[:] = u0
        sol = tl.solve_lwfr(upd, (), dt0, TOL, tl.Adaptive(on_device=on_device, chunk=7))
        runs.append(sol)
    host, dev = runs
    assert dev.t[0] == pytest.approx(t_end, rel=1e-14)
    assert dev.stats.naccept == host.stats.naccept > 3
    assert dev.stats.nreject == host.stats.nreject
    assert np.all(rel_l2(dev.u[0], host.u[0]) < 1e-12)
