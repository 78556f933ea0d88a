"""tlw_step_host: asynchronous host-buffer stepping with the copies of consecutive calls overlapped. Every
call's result equals the plain path's (upload, the same steps, download), whether the calls carry
independent states or feed each result back in, and the handle's state afterwards is the last result."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make(tl, level=5, N=4, strength=5.0):
    eq = tl.CompressibleEulerEquations2D(1.4)
    mesh = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), level)
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, tl.VolumeIntegralFR(tl.LW()))
    semi = tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, tl.IsentropicVortex(strength), solver)
    return semi, tl.LWIntegrator(tl.semidiscretize(semi, tl.LW(), (0.0, 1e9)))


def plain(integ, u, t, nsteps, cfl):
    integ.set_state(u, t)
    integ.step(nsteps, cfl, use_graph=False)
    return integ.get_state()


def test_step_host_independent_states_match_the_plain_path(tl):
    """Eleven calls without synchronisation (the five-buffer pool wraps around four times; 1, 2 and 3 steps a call
    leave the result in either buffer of a call's pair)."""
    semi, integ = make(tl)
    cfl = 0.5
    states = []
    strengths = (5.0, 3.0, 4.0, 2.0, 4.5, 3.5, 2.5, 5.5, 1.5, 4.2, 3.3)
    nsteps = [1 + k % 3 for k in range(len(strengths))]
    for beta in strengths:
        s, _ = make(tl, strength=beta)
        states.append(s.compute_coefficients(0.0))
    ins = [integ.pinned_state() for _ in states]
    outs = [integ.pinned_state() for _ in states]
    for a, u in zip(ins, states):
        a[:] = u
    for k in range(len(states)):      # no synchronisation between the calls
        integ.step_host(ins[k], outs[k], 0.1 * k, nsteps[k], cfl)
    integ.synchronize()
    last = integ.get_state()
    np.testing.assert_array_equal(last, outs[-1])
    _, ref_integ = make(tl)
    for k, u in enumerate(states):
        ref = plain(ref_integ, u, 0.1 * k, nsteps[k], cfl)
        np.testing.assert_array_equal(outs[k], ref)
    integ.sync_time()
    assert integ.iter == nsteps[-1] and integ.t > 0.1 * (len(states) - 1)


def test_step_host_with_steps_between_the_calls(tl):
    """Device-resident steps between asynchronous calls act on the last call's result; the later uploads into
    the buffers those steps used wait for them."""
    semi, integ = make(tl)
    u0 = semi.compute_coefficients(0.0)
    _, ref_integ = make(tl)
    ins = [integ.pinned_state() for _ in range(6)]
    outs = [integ.pinned_state() for _ in range(6)]
    mids = []
    for k in range(6):
        ins[k][:] = u0 * (1.0 + 0.01 * k)
    for k in range(6):
        integ.step_host(ins[k], outs[k], 0.0, 1, 0.5)
        integ.step(1 + k % 2, 0.5, use_graph=False)   # continues from the downloaded result
        mids.append(integ.get_state())
    integ.synchronize()
    for k in range(6):
        r1 = plain(ref_integ, ins[k], 0.0, 1, 0.5)
        np.testing.assert_array_equal(outs[k], r1)
        ref_integ.step(1 + k % 2, 0.5, use_graph=False)
        np.testing.assert_array_equal(mids[k], ref_integ.get_state())


def test_step_host_round_trip_through_the_host(tl):
    """Each call's input is the previous call's output buffer: the library orders the upload after the download."""
    semi, integ = make(tl)
    u0 = semi.compute_coefficients(0.0)
    buf = integ.pinned_state()
    buf[:] = u0
    for _ in range(7):
        integ.step_host(buf, buf, 0.0, 1, 0.5)
    integ.synchronize()
    _, ref_integ = make(tl)
    u = u0.copy()
    for _ in range(7):
        u = plain(ref_integ, u, 0.0, 1, 0.5)
    np.testing.assert_array_equal(buf, u)


def test_step_host_input_downloaded_two_calls_back(tl):
    """Three host buffers in rotation: call k reads the output of call k - 2, which may still be downloading."""
    semi, integ = make(tl)
    u0 = semi.compute_coefficients(0.0)
    bufs = [integ.pinned_state() for _ in range(3)]
    bufs[0][:] = u0
    bufs[1][:] = u0 * 1.01
    for k in range(6):
        integ.step_host(bufs[k % 3], bufs[(k + 2) % 3], 0.0, 1, 0.5)
    integ.synchronize()
    _, ref_integ = make(tl)
    ref = [u0.copy(), u0 * 1.01, None]
    for k in range(6):
        ref[(k + 2) % 3] = plain(ref_integ, ref[k % 3], 0.0, 1, 0.5)
    for b, r in zip(bufs, ref):
        np.testing.assert_array_equal(b, r)


def test_other_entry_points_after_step_host(tl):
    """tlw_set_state and tlw_step after asynchronous calls wait for their downloads and see the last result."""
    semi, integ = make(tl)
    u0 = semi.compute_coefficients(0.0)
    a, b = integ.pinned_state(), integ.pinned_state()
    a[:] = u0
    integ.step_host(a, b, 0.0, 3, 0.5)
    integ.step(2, 0.5)                  # continues from the downloaded result
    u = integ.get_state()
    _, ref_integ = make(tl)
    ref3 = plain(ref_integ, u0, 0.0, 3, 0.5)
    np.testing.assert_array_equal(b, ref3)
    ref_integ.step(2, 0.5)
    np.testing.assert_array_equal(u, ref_integ.get_state())
    integ.set_state(u0, 0.0)            # overwrites the current state after the pending download
    np.testing.assert_array_equal(integ.get_state(), u0)


def test_step_host_input_downloaded_four_calls_back(tl):
    """Five host buffers in rotation, two steps a call (the result in the upload's own device buffer): call k reads
    the output of call k - 4."""
    semi, integ = make(tl)
    u0 = semi.compute_coefficients(0.0)
    bufs = [integ.pinned_state() for _ in range(5)]
    for q in range(4):
        bufs[q][:] = u0 * (1.0 + 0.01 * q)
    for k in range(10):
        integ.step_host(bufs[k % 5], bufs[(k + 4) % 5], 0.0, 2, 0.5)
    integ.synchronize()
    _, ref_integ = make(tl)
    ref = [u0 * (1.0 + 0.01 * q) for q in range(4)] + [None]
    for k in range(10):
        ref[(k + 4) % 5] = plain(ref_integ, ref[k % 5], 0.0, 2, 0.5)
    for b, r in zip(bufs, ref):
        np.testing.assert_array_equal(b, r)


def test_step_host_after_device_steps(tl):
    """The first asynchronous call uploads into the handle's state buffers: it waits for the device steps that
    other entry points enqueued on them."""
    semi, integ = make(tl, level=6)
    u0 = semi.compute_coefficients(0.0)
    integ.set_state(u0, 0.0)
    integ.step(30, 0.5, use_graph=False)        # enqueued, still running when the call below uploads
    a, b = integ.pinned_state(), integ.pinned_state()
    a[:] = u0 * 1.02
    integ.step_host(a, b, 0.0, 1, 0.5)
    integ.synchronize()
    _, ref_integ = make(tl, level=6)
    np.testing.assert_array_equal(b, plain(ref_integ, u0 * 1.02, 0.0, 1, 0.5))
