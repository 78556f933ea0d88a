"""Batched form of the LW step: many independent periodic TreeMesh{2} runs of uneven size and degree
(N = 3, 4, 5) advanced together on one GPU by one replayed CUDA graph per step.

Every instance advances exactly as ``solve_lwfr`` (src/solvers/lwfr.jl:233-263) would advance it alone with
``CFLBased(cfl)``: its own dt = cfl * max_dt(u) (src/solvers/lwfr.jl:176-190), clamped to its own final
time (set_dt!, src/solvers/lwfr.jl:76-90), and no further steps once it is finished
(isfinished, src/solvers/lwfr.jl:146-148). The reference has no batched driver; this is the host side of
``tlw_batch_*`` in libtlw.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib
from .equations import CompressibleEulerEquations2D
from .mesh import TreeMesh
from .semidiscretization import FluxLaxFriedrichs, _i64p, _ptr


def compute_coefficients(mesh: TreeMesh, polydeg: int, initial_condition, equations, t: float = 0.0) -> np.ndarray:
    """Flat state [v, i, j, element] of ``initial_condition`` at the GLL nodes (Trixi compute_coefficients)."""
    xy = mesh.node_coordinates(polydeg)
    u = initial_condition(xy[0], xy[1], t, equations)   # [i, j, E, 4]
    return np.ascontiguousarray(np.transpose(u, (2, 1, 0, 3))).reshape(-1)


class LWBatch:
    """Owns one ``tlw_batch``: add instances, ``finalize``, ``set_state`` each, then ``step``."""

    def __init__(self, equations: CompressibleEulerEquations2D, surface_flux=None, device: int = 0):
        sf = surface_flux or FluxLaxFriedrichs()
        opts = _lib.TlwOpts()
        opts.polydeg = 4
        opts.time_discretization = _lib.TLW_LW
        opts.surface_flux = sf.code
        opts.max_speed = (_lib.TLW_SPEED_DAVIS if getattr(sf, "max_abs_speed", "naive") == "davis"
                          else _lib.TLW_SPEED_NAIVE)
        opts.gamma = equations.gamma
        opts.device = device
        opts.volume_integral = _lib.TLW_VOLUME_FR
        self.ptr = ctypes.c_void_p()
        check(None, lib().tlw_batch_create(ctypes.byref(opts), ctypes.byref(self.ptr)), batch=True)
        self.meshes: list[TreeMesh] = []
        self.degrees: list[int] = []
        self._finalized = False

    def _check(self, rc: int):
        check(self.ptr, rc, batch=True)

    def add(self, mesh: TreeMesh, polydeg: int) -> int:
        """Adds one periodic TreeMesh{2} instance of degree ``polydeg``; returns its id."""
        if mesh.n_boundaries:
            raise ValueError("the batched form takes periodic meshes only")
        ij = np.ascontiguousarray(mesh.inverse_jacobian, dtype=np.float64)
        nid = np.ascontiguousarray(mesh.interface_neighbor_ids, dtype=np.int64)
        nor = np.ascontiguousarray(mesh.interface_orientations, dtype=np.int64)
        idx = ctypes.c_int32()
        self._check(lib().tlw_batch_add_tree_mesh(self.ptr, int(polydeg), mesh.n_elements,
                                                  ij.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                  mesh.n_interfaces, _i64p(nid), _i64p(nor), ctypes.byref(idx)))
        self.meshes.append(mesh)
        self.degrees.append(int(polydeg))
        return int(idx.value)

    def finalize(self):
        self._check(lib().tlw_batch_finalize(self.ptr))
        self._finalized = True

    def ndofs(self, i: int) -> int:
        return self.meshes[i].ndofs(self.degrees[i])

    def set_state(self, i: int, u: np.ndarray, t: float, cfl: float, t_end: float = float("inf")):
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.size != 4 * self.ndofs(i):
            raise ValueError("state size does not match the instance")
        self._check(lib().tlw_batch_set_state(self.ptr, int(i), _ptr(u), _lib.TLW_WHERE_HOST, float(t),
                                              float(cfl), float(t_end)))

    def get_state(self, i: int):
        """(u, t, accepted steps) of instance ``i``; raises DomainError if a kernel met a bad state."""
        u = np.empty(4 * self.ndofs(i))
        t = ctypes.c_double()
        steps = ctypes.c_int64()
        self._check(lib().tlw_batch_get_state(self.ptr, int(i), _ptr(u), _lib.TLW_WHERE_HOST, ctypes.byref(t),
                                              ctypes.byref(steps)))
        return u, t.value, int(steps.value)

    def step(self, nsteps: int, use_graph: bool = True):
        self._check(lib().tlw_batch_step(self.ptr, int(nsteps), 1 if use_graph else 0))

    def synchronize(self):
        self._check(lib().tlw_batch_synchronize(self.ptr))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(lib().tlw_batch_get_stream(self.ptr, ctypes.byref(s)))
        return s.value or 0

    def num_groups(self) -> int:
        return int(lib().tlw_batch_num_groups(self.ptr))

    def autotune(self, trials: int = 3) -> dict:
        """Times the launch variants on this batch and keeps the fastest; returns the choices."""
        ng = self.num_groups()
        out = (ctypes.c_int32 * (2 * ng + 1))()
        self._check(lib().tlw_batch_autotune(self.ptr, int(trials), out))
        groups = sorted(set(self.degrees))
        return {"groups": {N: {"volume_variant": out[2 * k], "interface_block": out[2 * k + 1]}
                           for k, N in enumerate(groups)},
                "concurrent_groups": bool(out[2 * ng])}

    def close(self):
        if self.ptr:
            lib().tlw_batch_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_lwfr_batch(instances, equations: CompressibleEulerEquations2D, nsteps: int, surface_flux=None,
                     autotune: bool = True, device: int = 0):
    """Runs ``nsteps`` batch steps over ``instances`` (dicts with keys mesh, polydeg, u0, cfl and optionally
    t0, t_end) and returns [(u, t, steps)] per instance."""
    b = LWBatch(equations, surface_flux, device)
    try:
        for inst in instances:
            b.add(inst["mesh"], inst["polydeg"])
        b.finalize()
        for i, inst in enumerate(instances):
            b.set_state(i, inst["u0"], inst.get("t0", 0.0), inst["cfl"], inst.get("t_end", float("inf")))
        if autotune:
            b.autotune()
        b.step(nsteps)
        b.synchronize()
        return [b.get_state(i) for i in range(len(instances))]
    finally:
        b.close()
