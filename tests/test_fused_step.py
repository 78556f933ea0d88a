"""The fused launch (volume and surface passes of an LW step or MDRK stage on a periodic conforming TreeMesh in one
kernel, tiles handed out by ticket, each element's surface computed after its own and its neighbours' volume
phases) against the two-launch path: the same arithmetic, so the states and rhs agree bit for bit."""
import numpy as np
import pytest

from test_gpu_parity import make_semi

pytestmark = pytest.mark.gpu


def _lib():
    from trixilw import _lib
    return _lib.lib()


def _steps(tl, semi, u0, nsteps, cfl, fused, graph):
    integ = tl.LWIntegrator(tl.semidiscretize(semi, semi.time_discretization, (0.0, 1e9)))
    _lib().tlw_set_fused_step(semi.handle, 1 if fused else 0)
    integ.set_state(u0, 0.0)
    integ.step(nsteps, cfl, use_graph=graph)
    integ.sync_time()
    return integ.get_state(), integ.t


@pytest.mark.parametrize("td", ["lw", "mdrk"])
@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_fused_steps_equal_two_launch_steps(tl, N, td):
    """32^2 periodic vortex, 9 CFL steps through the step graph and 4 without: fused = two launches, bit for bit.
    The tiles (elements per volume CTA) do not divide 1024 elements for every degree (N = 2: 14, N = 4: 5)."""
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 5)
    semi = make_semi(tl, mesh, N, tl.IsentropicVortex(5.0, center=(0.3, -0.2)), td)
    assert _lib().tlw_set_fused_step(semi.handle, 2) == 3   # enabled, and the mesh admits the fused launch
    u0 = semi.compute_coefficients(0.0)
    cfl = 0.4 if N > 4 else 0.1 if N < 3 else 0.98 * (N + 1) * 0.103
    for graph, k in ((True, 9), (False, 4)):
        a, ta = _steps(tl, semi, u0, k, cfl, True, graph)
        b, tb = _steps(tl, semi, u0, k, cfl, False, graph)
        assert ta == tb
        np.testing.assert_array_equal(a, b)
    _lib().tlw_set_fused_step(semi.handle, 1)


@pytest.mark.parametrize("td", ["lw", "mdrk"])
@pytest.mark.parametrize("N", [3, 4])
def test_fused_rhs_equals_two_launch_rhs(tl, N, td):
    """One rhs (LW) or both MDRK stages' rhs in both paths."""
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 6)
    semi = make_semi(tl, mesh, N, tl.IsentropicVortex(5.0, center=(-0.4, 0.1)), td)
    u = semi.compute_coefficients(0.0)
    dt = semi.max_dt(u, 0.4)
    semi.cache["dt"][0] = dt
    out = []
    for fused in (1, 0):
        _lib().tlw_set_fused_step(semi.handle, fused)
        du = np.empty_like(u)
        if td == "lw":
            tl.rhs(du, u, semi, 0.0)
            out.append(du)
        else:   # both MDRK stages' rhs (MODE_RHS), stage 2 at u + dt/2 du_1
            tl.rhs_mdrk1(du, u, semi, 0.0)
            du2 = np.empty_like(u)
            tl.rhs_mdrk2(du2, u, semi, 0.0, u + 0.5 * dt * du)
            out.append(np.concatenate([du, du2]))
    _lib().tlw_set_fused_step(semi.handle, 1)
    np.testing.assert_array_equal(out[0], out[1])


@pytest.mark.parametrize("td", ["lw", "mdrk"])
def test_fused_steps_full_size(tl, td):
    """512^2, N = 4 (the throughput workloads: 52,429 tiles, hundreds of CTAs resident at once): 3 steps fused =
    3 steps in two launches, bit for bit."""
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 9)
    semi = make_semi(tl, mesh, 4, tl.IsentropicVortex(5.0), td)
    u0 = semi.compute_coefficients(0.0)
    a, ta = _steps(tl, semi, u0, 3, 0.98 * 5 * 0.103, True, True)
    b, tb = _steps(tl, semi, u0, 3, 0.98 * 5 * 0.103, False, True)
    assert ta == tb
    np.testing.assert_array_equal(a, b)


def test_fused_launch_not_taken_off_its_mesh(tl):
    """A mesh with boundaries keeps the two-launch path (query: enabled, mesh not admitted)."""
    mesh = tl.TreeMesh((-1.0, -1.0), (1.0, 1.0), 3, periodicity=False)
    semi = make_semi(tl, mesh, 4, tl.IsentropicVortex(0.5))
    assert _lib().tlw_set_fused_step(semi.handle, 2) == 1
