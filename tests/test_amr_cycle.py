"""A live AMR cycle on one handle, as the reference's AMRCallback drives it (the integrator and every cache resized
after each adaptation, src/callbacks/amr.jl:2-208): conforming mesh -> a refined patch with L2 mortars -> the
conforming mesh again, re-uploaded with SemidiscretizationHyperbolic.remesh (tlw_set_tree_mesh /
tlw_set_curved_mesh and the mortar arrays) on the same library handle. In every phase a fresh state (the host's
projection, here the initial condition on the new nodes) is set and stepped with the captured-graph step loop,
and the result equals the oracle's on that mesh."""
import os

import numpy as np
import pytest

from test_curved import warp

pytestmark = pytest.mark.gpu

NTH = os.cpu_count() or 1


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def phase(tl, oracle_mod, semi, integ, mesh, N, cfl, nsteps, kind, sc=False):
    u0 = semi.compute_coefficients(0.0)
    integ.set_state(u0, 0.0)
    integ.step(nsteps, cfl, use_graph=True)
    integ.sync_time()
    u_gpu = integ.get_state()
    o = oracle_mod.Oracle(mesh, N)
    if sc:
        o.set_shock_capturing(True, 0.5, 0.001, True)
    u_cpu = u0.copy()
    s, t = o.steps(u_cpu, nsteps, cfl, 0.0, 1e9, kind=kind, nthreads=NTH)
    assert s == integ.iter == nsteps and integ.t == pytest.approx(t, rel=1e-13)
    return rel_l2(u_gpu, u_cpu)


@pytest.mark.parametrize("td,sc", [("lw", False), ("mdrk", False), ("lw", True)])
def test_tree_mesh_refine_and_coarsen_on_one_handle(tl, oracle_mod, td, sc):
    N = 4
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    vi = tl.VolumeIntegralFR(tdo)
    if sc:
        vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5), vi)
    ic = tl.IsentropicVortex(5.0, center=(0.4, -0.3))
    coarse = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 4)
    fine = tl.RefinedTreeMesh((-10.0, -10.0), (10.0, 10.0), 4, ((-4.0, -4.0), (4.0, 4.0)))
    assert fine.n_mortars > 0
    semi = tl.SemidiscretizationHyperbolic(coarse, tdo, eq, ic, tl.DGSEM(N, tl.flux_lax_friedrichs, vi))
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tdo, (0.0, 1e9)))
    handle = semi.handle
    kind = 0 if td == "lw" else 1
    cfl = 0.3
    for mesh in (coarse, fine, coarse, fine):
        if mesh is not semi.mesh:
            semi.remesh(mesh)
        assert semi.handle == handle and semi.ndofs() == mesh.ndofs(N)
        assert np.all(phase(tl, oracle_mod, semi, integ, mesh, N, cfl, 3, kind, sc) < 1e-12)


def test_curvilinear_refine_and_coarsen_on_one_handle(tl, oracle_mod):
    N = 4
    eq = tl.CompressibleEulerEquations2D(1.4)
    ic = tl.IsentropicVortex(5.0, center=(0.7, -0.4))
    coarse = tl.StructuredMesh((6, 6), warp)
    fine = tl.RefinedStructuredMesh((6, 6), warp, [(2, 2), (3, 2), (2, 3)])
    assert fine.curved(N).n_mortars > 0
    semi = tl.SemidiscretizationHyperbolic(coarse, tl.LW(), eq, ic, tl.DGSEM(N, tl.flux_lax_friedrichs,
                                                                              tl.VolumeIntegralFR(tl.LW())))
    integ = tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))
    handle = semi.handle
    for mesh in (coarse, fine, coarse):
        if mesh is not semi.mesh:
            semi.remesh(mesh)
        assert semi.handle == handle
        assert np.all(phase(tl, oracle_mod, semi, integ, mesh, N, 0.4, 3, 0) < 1e-12)
