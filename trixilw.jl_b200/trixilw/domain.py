"""Domain decomposition of a TreeMesh{2} over ranks (one GPU per rank), the counterpart of the reference's MPI
path (src/solvers/dgsem_tree/dg_2d_parallel.jl:23-200, dg_parallel.jl:10-34).

Each rank owns a contiguous range of elements in the mesh's space-filling-curve (Morton) order, as Trixi's
ParallelTreeMesh partitions the leaves. Its part is a TreeMesh of the local elements with the interfaces between
them and its share of the boundaries; the faces it shares with another rank's part are its halo faces. A step
(``DomainDecomposedLW.step``) is: this part's CFL maximum, a MAX all-reduce of it over the ranks, the volume
kernel with the halo traces (u, U, F.n per node, 12 doubles, the reference's 3 nv message) packed into a send
buffer, the halo exchange with the neighbouring ranks, then the interfaces, boundaries and halo faces; an MDRK
step does the volume / exchange / surface round once per stage. With shock capturing the raw blending factors
of the cut faces' elements are exchanged after the all-reduce (for the smoothing across the cut faces), and a
halo node also carries fn_low and the smoothed alpha (20 doubles with padding), so the cut faces are blended as interior
interfaces are. The kernels run on the library's stream and the collectives on its comm stream; the library hands
the order over between the two, so the trace exchange overlaps the part's x interfaces.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, lib
from .mesh import TreeMesh

HALO_VALUES = 12      # doubles per cut face node without shock capturing (20 with it: tlw_dd_halo_values)


class LocalTreeMesh(TreeMesh):
    """One rank's part of a TreeMesh: the given elements (global 0-based ids, renumbered in order), the
    interfaces with both sides local, and the boundaries of local elements (direction order kept)."""

    def __init__(self, mesh: TreeMesh, elements: np.ndarray):
        self.global_mesh = mesh
        self.elements = np.asarray(elements, dtype=np.int64)
        self.periodicity = mesh.periodicity
        self.length = mesh.length
        self.level = mesh.level
        self.n_elements = len(self.elements)
        self.inverse_jacobian = np.ascontiguousarray(mesh.inverse_jacobian[self.elements])
        g2l = np.full(mesh.n_elements, -1, dtype=np.int64)
        g2l[self.elements] = np.arange(self.n_elements)
        self.g2l = g2l
        ids = mesh.interface_neighbor_ids.reshape(-1, 2) - 1
        both = (g2l[ids[:, 0]] >= 0) & (g2l[ids[:, 1]] >= 0)
        self.interface_neighbor_ids = np.ascontiguousarray(g2l[ids[both]].reshape(-1) + 1)
        self.interface_orientations = np.ascontiguousarray(mesh.interface_orientations[both])
        self.n_interfaces = int(both.sum())
        bl = g2l[mesh.boundary_neighbor_ids - 1]
        keep = bl >= 0
        self.boundary_neighbor_ids = np.ascontiguousarray(bl[keep] + 1)
        self.boundary_directions = np.ascontiguousarray(mesh.boundary_directions[keep])
        self.boundary_orientations = np.ascontiguousarray(mesh.boundary_orientations[keep])
        self.boundary_neighbor_sides = np.ascontiguousarray(mesh.boundary_neighbor_sides[keep])
        self.n_boundaries_per_direction = np.array([(self.boundary_directions == d).sum() for d in (1, 2, 3, 4)],
                                                   dtype=np.int64)
        self.n_boundaries = int(keep.sum())

    def node_coordinates(self, polydeg: int) -> np.ndarray:
        return np.ascontiguousarray(self.global_mesh.node_coordinates(polydeg)[..., self.elements])


@dataclass
class Part:
    rank: int
    mesh: LocalTreeMesh
    halo_elements: np.ndarray        # [H] 1-based local elements
    halo_faces: np.ndarray           # [H] 0: -x, 1: +x, 2: -y, 3: +y
    halo_keys: np.ndarray            # [H] global interface index (the pairing key)
    segments: dict = field(default_factory=dict)   # neighbour rank -> (offset, count) in the halo order


def owner_of(n_elements: int, nparts: int) -> np.ndarray:
    """Rank of every element: contiguous ranges of the space-filling-curve order, sizes differing by at most one."""
    bounds = [n_elements * r // nparts for r in range(nparts + 1)]
    owner = np.empty(n_elements, dtype=np.int64)
    for r in range(nparts):
        owner[bounds[r]:bounds[r + 1]] = r
    return owner


def partition(mesh: TreeMesh, nparts: int) -> list[Part]:
    """The parts of a conforming TreeMesh for nparts ranks. Halo faces are ordered by (neighbour rank, global
    interface index), so a neighbour's send segment and this rank's receive segment list the same faces in the
    same order."""
    if getattr(mesh, "n_mortars", 0):
        raise NotImplementedError("domain decomposition: conforming TreeMesh (no mortars)")
    owner = owner_of(mesh.n_elements, nparts)
    ids = mesh.interface_neighbor_ids.reshape(-1, 2) - 1
    ori = mesh.interface_orientations
    parts = []
    for r in range(nparts):
        local = LocalTreeMesh(mesh, np.nonzero(owner == r)[0])
        rows = []
        for k in np.nonzero((owner[ids[:, 0]] == r) != (owner[ids[:, 1]] == r))[0]:
            left_local = owner[ids[k, 0]] == r
            e = ids[k, 0] if left_local else ids[k, 1]
            other = ids[k, 1] if left_local else ids[k, 0]
            face = (1 if ori[k] == 1 else 3) if left_local else (0 if ori[k] == 1 else 2)
            rows.append((int(owner[other]), int(k), int(local.g2l[e]) + 1, face))
        rows.sort()
        segments, off = {}, 0
        for q in sorted({row[0] for row in rows}):
            cnt = sum(1 for row in rows if row[0] == q)
            segments[q] = (off, cnt)
            off += cnt
        parts.append(Part(r, local,
                          np.array([row[2] for row in rows], dtype=np.int64),
                          np.array([row[3] for row in rows], dtype=np.int32),
                          np.array([row[1] for row in rows], dtype=np.int64), segments))
    return parts


class _DeviceArray:
    """A device buffer of the library seen by torch without a copy (__cuda_array_interface__)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


class DomainDecomposedLW:
    """One rank's part, stepping with the library's split step (tlw_dd_begin / _volume / _finish).

    ``allreduce_max(t)`` and ``exchange(send, recv, segments)`` are the rank's collectives on torch tensors that
    alias the library's device buffers: an int64 scalar holding the CFL maximum's bits (a non-negative double,
    so int64 order is double order), the [H, n, 12 or 20] halo buffers and, with shock capturing, the [H] alpha
    buffers. ``torch_collectives`` gives them for torch.distributed."""

    def __init__(self, semi, part: Part, allreduce_max, exchange):
        import torch

        self.semi = semi
        self.part = part
        self.allreduce_max = allreduce_max
        self.exchange = exchange
        h = semi.handle
        H = len(part.halo_elements)
        self._keep = (np.ascontiguousarray(part.halo_elements, dtype=np.int64),
                      np.ascontiguousarray(part.halo_faces, dtype=np.int32))
        check(h, lib().tlw_set_halo(h, H, self._keep[0].ctypes.data, self._keep[1].ctypes.data))
        send, recv, mx = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(h, lib().tlw_dd_buffers(h, ctypes.byref(send), ctypes.byref(recv), ctypes.byref(mx)))
        n = semi.nnodes
        dev = torch.device("cuda", semi.device)
        nv = int(lib().tlw_dd_halo_values(h))
        self.send = torch.as_tensor(_DeviceArray(send.value or 0, (H, n, nv), "<f8"), device=dev) if H else None
        self.recv = torch.as_tensor(_DeviceArray(recv.value or 0, (H, n, nv), "<f8"), device=dev) if H else None
        asend, arecv = ctypes.c_void_p(), ctypes.c_void_p()
        check(h, lib().tlw_dd_alpha_buffers(h, ctypes.byref(asend), ctypes.byref(arecv)))
        self.alpha_send = (torch.as_tensor(_DeviceArray(asend.value, (H,), "<f8"), device=dev)
                           if H and asend.value else None)
        self.alpha_recv = (torch.as_tensor(_DeviceArray(arecv.value, (H,), "<f8"), device=dev)
                           if H and arecv.value else None)
        self.max_bits = torch.as_tensor(_DeviceArray(mx.value, (1,), "<i8"), device=dev)
        # the collectives go on the library's comm stream: the split step hands the order over to it after the
        # packing, so the exchange overlaps the part's x interfaces
        sp = ctypes.c_void_p()
        check(h, lib().tlw_dd_comm_stream(h, ctypes.byref(sp)))
        self.stream = torch.cuda.ExternalStream(sp.value, device=dev)
        # the kernels' stream: a step's last work is on it (events that bracket whole steps go here)
        check(h, lib().tlw_get_stream(h, ctypes.byref(sp)))
        self.lib_stream = torch.cuda.ExternalStream(sp.value, device=dev)

    def step(self, nsteps: int, cfl: float, t_end: float = float("inf"), fixed_dt: float = 0.0):
        import torch

        h = self.semi.handle
        L = lib()
        stages = int(L.tlw_dd_stages(h))
        for _ in range(int(nsteps)):
            check(h, L.tlw_dd_begin(h, float(cfl), float(fixed_dt), float(t_end)))
            with torch.cuda.stream(self.stream):
                self.allreduce_max(self.max_bits)
                if self.alpha_send is not None:   # shock capturing: raw alpha across the cut faces
                    self.exchange(self.alpha_send, self.alpha_recv, self.part.segments)
            for _stage in range(stages):   # MDRK: stage 1 (into u*), then stage 2, each with its own exchange
                check(h, L.tlw_dd_volume(h))
                if self.send is not None:
                    with torch.cuda.stream(self.stream):
                        self.exchange(self.send, self.recv, self.part.segments)
                check(h, L.tlw_dd_finish(h))


def torch_collectives(group=None):
    """(allreduce_max, exchange) over torch.distributed: a MAX all-reduce and, per neighbouring rank, one send of
    this rank's segment and one receive into it (batch_isend_irecv)."""
    import torch.distributed as dist

    def allreduce_max(t):
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)

    def exchange(send, recv, segments):
        ops = []
        for q, (off, cnt) in sorted(segments.items()):
            ops.append(dist.P2POp(dist.isend, send[off:off + cnt], q, group=group))
            ops.append(dist.P2POp(dist.irecv, recv[off:off + cnt], q, group=group))
        for w in dist.batch_isend_irecv(ops):
            w.wait()

    return allreduce_max, exchange
