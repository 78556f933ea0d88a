"""Domain decomposition of the LW and MDRK steps over ranks (the reference's MPI path, src/solvers/dgsem_tree/
dg_2d_parallel.jl): the partition's bookkeeping and the host collectives (world size 2 over gloo) on the CPU, and
on one GPU the library's split step (tlw_dd_begin / _volume / _finish with the halo kernels) for 2 to 4 parts
driven in lockstep in one process, equal bit for bit to the single-domain run, with the FR volume integral and
with shock capturing (alpha smoothed across the cut faces, cut faces blended)."""
import os
import socket

import numpy as np
import pytest

NTH = os.cpu_count() or 1


def rel_l2(a, b):
    a = a.reshape(-1, 4)
    b = b.reshape(-1, 4)
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


# ---------------------------------------------------------------------------------------------- CPU
@pytest.mark.parametrize("nparts,periodic", [(2, True), (3, True), (4, False), (5, True)])
def test_partition_bookkeeping(tl, nparts, periodic):
    from trixilw.domain import partition
    mesh = tl.TreeMesh((-1.0, -1.0), (1.0, 1.0), 3, periodicity=periodic)
    parts = partition(mesh, nparts)
    assert sorted(np.concatenate([p.mesh.elements for p in parts]).tolist()) == list(range(mesh.n_elements))
    # every interface is local to one part, or a halo face of exactly two parts on opposite sides
    local = sum(p.mesh.n_interfaces for p in parts)
    halo = {}
    for p in parts:
        for e, f, k in zip(p.halo_elements, p.halo_faces, p.halo_keys):
            halo.setdefault(int(k), []).append((p.rank, int(p.mesh.elements[e - 1]), int(f)))
    assert local + len(halo) == mesh.n_interfaces
    ids = mesh.interface_neighbor_ids.reshape(-1, 2) - 1
    for k, sides in halo.items():
        assert len(sides) == 2 and sides[0][0] != sides[1][0]
        got = {(g, f) for _, g, f in sides}
        o = mesh.interface_orientations[k]
        assert got == {(ids[k, 0], 1 if o == 1 else 3), (ids[k, 1], 0 if o == 1 else 2)}
    # a neighbour's send segment and this part's receive segment list the same faces in the same order
    for p in parts:
        for q, (off, cnt) in p.segments.items():
            oq, cq = parts[q].segments[p.rank]
            assert cnt == cq
            np.testing.assert_array_equal(p.halo_keys[off:off + cnt], parts[q].halo_keys[oq:oq + cq])
    assert sum(p.mesh.n_boundaries for p in parts) == mesh.n_boundaries


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, result):
    import torch
    import torch.distributed as dist

    import trixilw as tl
    from trixilw.domain import partition, torch_collectives

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        mesh = tl.TreeMesh((-1.0, -1.0), (1.0, 1.0), 3)
        part = partition(mesh, world)[rank]
        n = 4
        allreduce_max, exchange = torch_collectives()
        # what a rank sends for global face k, node l, value c: a code of (k, l, c, sender)
        H = len(part.halo_keys)
        ok_x = len(part.segments) >= 1
        # the trace buffers (12 values a node; 20 with shock capturing) and the [H] alpha buffer
        for vals in (12, 20):
            code = lambda k, r: (np.asarray(k)[:, None, None] * 1000.0 + np.arange(n)[None, :, None] * 10.0
                                 + np.arange(vals)[None, None, :] * 0.01 + r * 0.0001)
            send = torch.tensor(code(part.halo_keys, rank))
            recv = torch.zeros(H, n, vals, dtype=torch.float64)
            exchange(send, recv, part.segments)
            expect = np.empty((H, n, vals))
            for q, (off, cnt) in part.segments.items():
                expect[off:off + cnt] = code(part.halo_keys[off:off + cnt], q)
            ok_x = ok_x and bool(np.array_equal(recv.numpy(), expect))
        send = torch.tensor(part.halo_keys * 10.0 + rank)
        recv = torch.zeros(H, dtype=torch.float64)
        exchange(send, recv, part.segments)
        expect = np.empty(H)
        for q, (off, cnt) in part.segments.items():
            expect[off:off + cnt] = part.halo_keys[off:off + cnt] * 10.0 + q
        ok_x = ok_x and bool(np.array_equal(recv.numpy(), expect))
        # the CFL maximum: bits of non-negative doubles reduce like int64
        mine = np.array([1.5 + rank], dtype=np.float64).view(np.int64)
        t = torch.tensor(mine)
        allreduce_max(t)
        ok_m = t.numpy().view(np.float64)[0] == 1.5 + (world - 1)
        result[rank] = ok_x and ok_m
    finally:
        dist.destroy_process_group()


def test_gloo_halo_exchange_world2():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        result = mgr.dict()
        mp.spawn(_gloo_worker, args=(world, port, result), nprocs=world, join=True)
        assert dict(result) == {0: True, 1: True}


# ---------------------------------------------------------------------------------------------- GPU
def _square(x, y, t, eq):
    """A density square moving diagonally: discontinuous, so the indicator blends along its edges."""
    rho = np.where((np.abs(x - 0.3) < 2.0) & (np.abs(y + 0.2) < 2.0), 2.0, 1.0)
    return eq.prim2cons(rho, 0.5, 0.3, 1.0)


def _semi(tl, mesh, N, bc=None, td="lw", sc=False):
    eq = tl.CompressibleEulerEquations2D(1.4)
    tdo = tl.LW() if td == "lw" else tl.MDRK()
    vi = tl.VolumeIntegralFR(tdo)
    if sc:
        vi = tl.VolumeIntegralFRShockCapturing(tl.IndicatorHennemannGassner(alpha_max=0.5), vi)
    solver = tl.DGSEM(N, tl.flux_lax_friedrichs, vi)
    kw = {} if bc is None else {"boundary_conditions": bc}
    # with walls: a vortex at rest (no background flow into the walls)
    ic = (_square if sc else tl.IsentropicVortex(5.0, center=(0.3, -0.2)) if bc is None else
          tl.IsentropicVortex(3.0, center=(0.3, -0.2), domain=(-5.0, 5.0), velocity=(0.0, 0.0)))
    return tl.SemidiscretizationHyperbolic(mesh, tdo, eq, ic, solver, **kw)


def _lockstep(tl, parts, semis, steps, cfl):
    """The ranks' split steps in one process: the MAX all-reduce and the halo exchange done by device copies
    between the parts' buffers, with a device synchronisation between the phases."""
    import ctypes

    import torch
    from trixilw import _lib
    from trixilw.domain import DomainDecomposedLW

    L = _lib.lib()
    dds = [DomainDecomposedLW(s, p, None, None) for s, p in zip(semis, parts)]
    for _ in range(steps):
        for d in dds:
            _lib.check(d.semi.handle, L.tlw_dd_begin(d.semi.handle, cfl, 0.0, float("inf")))
        torch.cuda.synchronize()
        m = torch.max(torch.cat([d.max_bits for d in dds]))
        for d in dds:
            d.max_bits.fill_(m)
            if d.alpha_send is not None:   # shock capturing: the neighbours' raw alpha of the cut faces
                for q, (off, cnt) in d.part.segments.items():
                    oq, cq = dds[q].part.segments[d.part.rank]
                    d.alpha_recv[off:off + cnt].copy_(dds[q].alpha_send[oq:oq + cq])
        torch.cuda.synchronize()
        for _stage in range(int(L.tlw_dd_stages(dds[0].semi.handle))):
            for d in dds:
                _lib.check(d.semi.handle, L.tlw_dd_volume(d.semi.handle))
            torch.cuda.synchronize()
            for d in dds:
                for q, (off, cnt) in d.part.segments.items():
                    oq, cq = dds[q].part.segments[d.part.rank]
                    d.recv[off:off + cnt].copy_(dds[q].send[oq:oq + cq])
            torch.cuda.synchronize()
            for d in dds:
                _lib.check(d.semi.handle, L.tlw_dd_finish(d.semi.handle))
            torch.cuda.synchronize()
    return dds


def _streamed(tl, parts, semis, steps, cfl):
    """The ranks' split steps in one process with the collectives enqueued on each part's comm stream and no
    device synchronisation between the phases: a part's copies wait (by events) for the neighbours' comm streams,
    which the library has handed the packed buffers to, and each tlw_dd_* call waits for its own comm stream.
    This runs the hand-over between the kernels' stream and the comm stream as NCCL ranks would use it."""
    import torch
    from trixilw import _lib
    from trixilw.domain import DomainDecomposedLW

    L = _lib.lib()
    dds = [DomainDecomposedLW(s, p, None, None) for s, p in zip(semis, parts)]

    def comm_events():
        evs = []
        for d in dds:
            ev = torch.cuda.Event()
            ev.record(d.stream)
            evs.append(ev)
        return evs

    def join():
        # as a collective's completion: no part's comm stream goes on before every part's has arrived here
        evs = comm_events()
        for d in dds:
            for ev in evs:
                d.stream.wait_event(ev)

    def exchange(get_send, get_recv):
        evs = comm_events()
        for d in dds:
            with torch.cuda.stream(d.stream):
                for q, (off, cnt) in d.part.segments.items():
                    d.stream.wait_event(evs[q])
                    oq, cq = dds[q].part.segments[d.part.rank]
                    get_recv(d)[off:off + cnt].copy_(get_send(dds[q])[oq:oq + cq])
        join()

    for _ in range(steps):
        for d in dds:
            _lib.check(d.semi.handle, L.tlw_dd_begin(d.semi.handle, cfl, 0.0, float("inf")))
        evs = comm_events()
        maxes = []
        for d in dds:   # the MAX all-reduce: every comm stream sees every part's CFL maximum
            with torch.cuda.stream(d.stream):
                for ev in evs:
                    d.stream.wait_event(ev)
                maxes.append(torch.max(torch.cat([x.max_bits for x in dds])))
        join()
        for d, m in zip(dds, maxes):
            with torch.cuda.stream(d.stream):
                d.max_bits.fill_(m)
        if dds[0].alpha_send is not None:
            exchange(lambda d: d.alpha_send, lambda d: d.alpha_recv)
        for _stage in range(int(L.tlw_dd_stages(dds[0].semi.handle))):
            for d in dds:
                _lib.check(d.semi.handle, L.tlw_dd_volume(d.semi.handle))
            exchange(lambda d: d.send, lambda d: d.recv)
            for d in dds:
                _lib.check(d.semi.handle, L.tlw_dd_finish(d.semi.handle))
    torch.cuda.synchronize()
    return dds


@pytest.mark.gpu
@pytest.mark.parametrize("nparts,td,sc", [(3, "lw", False), (2, "mdrk", False), (3, "lw", True)])
def test_gpu_split_step_on_comm_streams_equals_single_domain(tl, nparts, td, sc):
    from trixilw.domain import partition
    N, steps, cfl = 4, 6, 0.4
    mesh = tl.TreeMesh((-5.0, -5.0), (5.0, 5.0), 4)
    whole = _semi(tl, mesh, N, None, td, sc)
    u0 = whole.compute_coefficients(0.0)
    integ = tl.LWIntegrator(tl.semidiscretize(whole, whole.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    integ.step(steps, cfl, use_graph=False)
    integ.sync_time()
    ref = integ.get_state()
    parts = partition(mesh, nparts)
    semis = [_semi(tl, p.mesh, N, None, td, sc) for p in parts]
    nn4 = 4 * (N + 1) ** 2
    integs = []
    for s, p in zip(semis, parts):
        it = tl.LWIntegrator(tl.semidiscretize(s, s.time_discretization, (0.0, 1e9)))
        it.set_state(np.ascontiguousarray(u0.reshape(-1, nn4)[p.mesh.elements].reshape(-1)), 0.0)
        integs.append(it)
    _streamed(tl, parts, semis, steps, cfl)
    got = np.empty_like(ref).reshape(-1, nn4)
    for it, p in zip(integs, parts):
        it.sync_time()
        assert it.iter == steps and it.t == integ.t
        got[p.mesh.elements] = it.get_state().reshape(-1, nn4)
    np.testing.assert_array_equal(got.reshape(-1), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("nparts,N,walls,td,sc", [(2, 4, False, "lw", False), (3, 3, False, "lw", False),
                                                  (4, 4, True, "lw", False), (2, 4, False, "mdrk", False),
                                                  (3, 5, False, "mdrk", False), (4, 3, True, "mdrk", False),
                                                  (2, 4, False, "lw", True), (3, 3, False, "lw", True),
                                                  (4, 4, False, "mdrk", True)])
def test_gpu_split_step_equals_single_domain(tl, nparts, N, walls, td, sc):
    from trixilw import _lib
    from trixilw.domain import partition
    mesh = tl.TreeMesh((-5.0, -5.0), (5.0, 5.0), 4, periodicity=not walls)
    bc = None
    if walls:
        bc = {"x_neg": tl.boundary_condition_slip_wall_vertical, "x_pos": tl.boundary_condition_slip_wall_vertical,
              "y_neg": tl.boundary_condition_slip_wall_horizontal, "y_pos": tl.boundary_condition_slip_wall_horizontal}
    whole = _semi(tl, mesh, N, bc, td, sc)
    u0 = whole.compute_coefficients(0.0)
    integ = tl.LWIntegrator(tl.semidiscretize(whole, whole.time_discretization, (0.0, 1e9)))
    integ.set_state(u0, 0.0)
    steps, cfl = 6, 0.4
    integ.step(steps, cfl, use_graph=False)
    integ.sync_time()
    ref = integ.get_state()
    if sc:   # the blending reaches the cut faces
        alpha = whole.get_cache(_lib.TLW_CACHE_ALPHA)
        assert alpha.max() > 0.1 and (alpha == 0.0).sum() > 0
    parts = partition(mesh, nparts)
    semis = [_semi(tl, p.mesh, N, bc, td, sc) for p in parts]
    nn4 = 4 * (N + 1) ** 2
    integs = []
    for s, p in zip(semis, parts):
        it = tl.LWIntegrator(tl.semidiscretize(s, s.time_discretization, (0.0, 1e9)))
        it.set_state(np.ascontiguousarray(u0.reshape(-1, nn4)[p.mesh.elements].reshape(-1)), 0.0)
        integs.append(it)
    _lockstep(tl, parts, semis, steps, cfl)
    got = np.empty_like(ref).reshape(-1, nn4)
    for it, p in zip(integs, parts):
        it.sync_time()
        assert it.iter == steps and it.t == integ.t
        got[p.mesh.elements] = it.get_state().reshape(-1, nn4)
    # the same flux for every face node in the same order of operations: equal bit for bit
    np.testing.assert_array_equal(got.reshape(-1), ref)
