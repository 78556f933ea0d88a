"""tlw_rhs_lw_noalloc: the LW rhs for callers that must not allocate device memory (their GPU memory is
owned by another pool, or they cannot accept cudaMalloc's implicit synchronisation). Its scratch is a
static device array inside libtlw, so this test checks, through the C ABI, that two calls in a row give
the handle-based rhs (tlw_rhs) result and the oracle's, i.e. that no stale scratch leaks from one call
into the next, that the second call leaves the device's free memory unchanged, and that a mesh too large
for the array is refused. Device buffers for inputs/outputs are the test's own.

This file is named to be collected last: a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12   # same bar as the parity tests (relative L2 per variable)


def rel_l2(a, b):
    a, b = a.reshape(-1, 4), b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.linalg.norm(b, axis=0)


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("N,flux,speed", [(4, 0, 0), (1, 0, 0), (3, 1, 0), (5, 0, 1), (7, 0, 0)])
def test_noalloc_entry_point_matches_handle_entry_point_and_oracle(tl, oracle_mod, N, flux, speed):
    import torch
    from trixilw import _lib

    L = _lib.lib()
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 4 if N >= 6 else 5)     # 16^2 or 32^2 elements
    surface_flux = tl.FluxHLL() if flux == 1 else tl.FluxLaxFriedrichs("davis" if speed == 1 else "naive")
    solver = tl.DGSEM(N, surface_flux, tl.VolumeIntegralFR(tl.LW()))
    cases = [tl.IsentropicVortex(5.0), tl.IsentropicVortex(3.0, center=(2.0, -1.0))]
    dev = torch.device("cuda", 0)
    ids = mesh.interface_neighbor_ids - 1
    xs = mesh.interface_orientations == 1
    xl = torch.tensor(ids[xs, 0], dtype=torch.int32, device=dev)
    xr = torch.tensor(ids[xs, 1], dtype=torch.int32, device=dev)
    yl = torch.tensor(ids[~xs, 0], dtype=torch.int32, device=dev)
    yr = torch.tensor(ids[~xs, 1], dtype=torch.int32, device=dev)
    ij = torch.tensor(mesh.inverse_jacobian, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    oracle = oracle_mod.Oracle(mesh, N, flux_kind=flux, speed_kind=speed)
    for call, ic in enumerate(cases):   # two calls in a row, different states
        semi = tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, ic, solver)
        u = semi.compute_coefficients(0.0)
        dt = semi.max_dt(u, 0.3)
        semi.cache["dt"][0] = dt
        du_ref = np.empty_like(u)
        tl.rhs(du_ref, u, semi, 0.0)                               # the existing (handle) entry point
        du_oracle = oracle.rhs(u, 0.0, dt)
        u_d = torch.tensor(u, device=dev)
        du_d = torch.full_like(u_d, float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = L.tlw_rhs_lw_noalloc(N, 1.4, flux, speed, mesh.n_elements, _vp(ij),
                                  int(xs.sum()), _vp(xl), _vp(xr), int((~xs).sum()), _vp(yl), _vp(yr),
                                  _vp(u_d), _vp(du_d), dt, ctypes.c_void_p(stream.cuda_stream))
        assert rc == _lib.TLW_OK
        free_after = torch.cuda.mem_get_info(dev)[0]
        if call == 1:   # the first call may load the library's module (and with it the static array)
            assert free_after == free_before
        du = du_d.cpu().numpy()
        assert np.all(rel_l2(du, du_ref) < RTOL), rel_l2(du, du_ref)
        assert np.all(rel_l2(du, du_oracle) < RTOL), rel_l2(du, du_oracle)


def test_noalloc_rejects_meshes_beyond_the_scratch(tl):
    import torch
    from trixilw import _lib

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    u = torch.zeros(8, dtype=torch.float64, device=dev)
    # N = 4: 1280 bytes of traces per element; 2**20 elements need 1.25 GiB > 32 MiB
    rc = L.tlw_rhs_lw_noalloc(4, 1.4, 0, 0, 1 << 20, _vp(u), 0, None, None, 0, None, None, _vp(u), _vp(u), 1e-3,
                              None)
    assert rc == _lib.TLW_E_ARG
