"""ctypes wrapper of the CPU oracle (liboracle_tlw.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by the CPU-baseline leg
of bench.py, as the checker. Parity status of the oracle: unpinned against the reference itself (no
Julia on this machine); pinned by scheme invariants, see tlw_oracle.hpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "liboracle_tlw.so")


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
            os.path.getmtime(os.path.join(_HERE, f)) for f in os.listdir(_HERE) if f.endswith((".hpp", ".cpp"))):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "liboracle_tlw.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB


_L = None


def lib():
    global _L
    if _L is None:
        build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        i32, dbl = ctypes.c_int, ctypes.c_double
        L.oracle_basis.argtypes = [i32, P, P, P, P]
        L.oracle_create.argtypes = [i32, dbl, i32, i32, i32, P, i32, P, P, P, i32, P, P, P, P]
        L.oracle_create.restype = P
        L.oracle_destroy.argtypes = [P]
        L.oracle_set_temporal_errors.argtypes = [P, i32, dbl, dbl]
        L.oracle_set_curved_mortar_jacobian.argtypes = [P, P]
        L.oracle_set_unstructured_normals.argtypes = [P, P]
        L.oracle_set_source.argtypes = [P, i32, P]
        L.oracle_dual_step.argtypes = [P, i32, P, P, dbl, P, P]
        L.oracle_set_shock_capturing.argtypes = [P, i32, dbl, dbl, i32]
        L.oracle_set_reconstruction.argtypes = [P, i32]
        L.oracle_set_curved_mortars.argtypes = [P, i32, P, P, P, P, P, P]
        L.oracle_set_boundary_data.argtypes = [P, P, P]
        L.oracle_rhs.argtypes = [P, i32, P, P, P, dbl, dbl, i32]
        L.oracle_get.argtypes = [P, i32, P]
        L.oracle_max_dt.argtypes = [P, P, dbl]
        L.oracle_max_dt.restype = dbl
        L.oracle_steps.argtypes = [P, i32, P, i32, dbl, dbl, P, dbl, i32]
        L.oracle_adjoint_step.argtypes = [P, P, dbl, P, P, i32]
        L.oracle_set_mortars.argtypes = [P, i32, P, P, P, P, P]
        L.oracle_set_parabolic.argtypes = [P, dbl, dbl]
        L.oracle_mortar_operators.argtypes = [i32, P]
        L.oracle_create_curved.argtypes = [i32, dbl, i32, i32, i32, P, P, i32, P, P, P, P, P]
        L.oracle_create_curved.restype = P
        L.oracle_set_limiter.argtypes = [P, i32, P, P]
        L.oracle_set_boundary_kinds.argtypes = [P, P]
        L.oracle_set_walls.argtypes = [P, P, P]
        L.oracle_set_curved_boundaries.argtypes = [P, i32, P, P, P]
        L.oracle_apply_limiter.argtypes = [P, P]
        L.oracle_last_error.argtypes = [P]
        L.oracle_last_error.restype = ctypes.c_char_p
        _L = L
    return _L


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def mortar_operators(N: int):
    """(forward_upper, forward_lower, reverse_upper, reverse_lower), each [n, n]."""
    n = N + 1
    out = np.empty(4 * n * n)
    assert lib().oracle_mortar_operators(N, _p(out)) == 0
    return tuple(out.reshape(4, n, n))


def basis(N: int):
    n = N + 1
    nodes, w, D, Dh = np.empty(n), np.empty(n), np.empty(n * n), np.empty(n * n)
    assert lib().oracle_basis(N, _p(nodes), _p(w), _p(D), _p(Dh)) == 0
    return nodes, w, D.reshape(n, n), Dh.reshape(n, n)


class OracleDomainError(ArithmeticError):
    pass


class Oracle:
    """One oracle instance for a TreeMesh (the mesh object of trixilw.mesh or any object with the same
    Trixi-convention arrays)."""

    def __init__(self, mesh, polydeg: int, gamma: float = 1.4, flux_kind: int = 0, speed_kind: int = 0):
        self.N = polydeg
        self.n = polydeg + 1
        self.mesh = mesh
        self.E = mesh.n_elements
        if hasattr(mesh, "curved") or hasattr(mesh, "Ja"):
            self._init_curved(mesh.curved(polydeg) if hasattr(mesh, "curved") else mesh, polydeg, gamma, flux_kind,
                              speed_kind)
            return
        ij = np.ascontiguousarray(mesh.inverse_jacobian, dtype=np.float64)
        ids = np.asarray(mesh.interface_neighbor_ids, dtype=np.int64).reshape(-1, 2)
        left = np.ascontiguousarray(ids[:, 0] - 1, dtype=np.int32)
        right = np.ascontiguousarray(ids[:, 1] - 1, dtype=np.int32)
        orient = np.ascontiguousarray(mesh.interface_orientations, dtype=np.int32)
        B = mesh.n_boundaries
        be = np.ascontiguousarray(np.asarray(mesh.boundary_neighbor_ids) - 1, dtype=np.int32)
        bo = np.ascontiguousarray(mesh.boundary_orientations, dtype=np.int32)
        bs = np.ascontiguousarray(mesh.boundary_neighbor_sides, dtype=np.int32)
        bd = np.ascontiguousarray(np.repeat(np.arange(1, 5), np.asarray(mesh.n_boundaries_per_direction)), dtype=np.int32)
        self._keep = (ij, left, right, orient, be, bo, bs, bd)
        self.h = lib().oracle_create(polydeg, gamma, flux_kind, speed_kind, self.E, _p(ij), len(orient), _p(left),
                                     _p(right), _p(orient), B, _p(be) if B else None, _p(bo) if B else None,
                                     _p(bs) if B else None, _p(bd) if B else None)
        if not self.h:
            raise RuntimeError("oracle_create failed")
        if getattr(mesh, "n_mortars", 0):
            ids = np.asarray(mesh.mortar_neighbor_ids, dtype=np.int64).reshape(-1, 3) - 1
            arrs = [np.ascontiguousarray(ids[:, k], dtype=np.int32) for k in range(3)]
            arrs += [np.ascontiguousarray(mesh.mortar_large_sides, dtype=np.int32),
                     np.ascontiguousarray(mesh.mortar_orientations, dtype=np.int32)]
            self._mkeep = arrs
            assert lib().oracle_set_mortars(self.h, len(arrs[0]), *[_p(a) for a in arrs]) == 0

    def _init_curved(self, cm, polydeg, gamma, flux_kind, speed_kind):
        """Conforming curvilinear mesh (trixilw.curved_mesh.CurvedMesh or StructuredMesh)."""
        Ja = np.ascontiguousarray(cm.Ja, dtype=np.float64)
        ij = np.ascontiguousarray(cm.inverse_jacobian_nodes, dtype=np.float64)
        pe = np.ascontiguousarray(cm.primary_elements - 1, dtype=np.int32)
        se = np.ascontiguousarray(cm.secondary_elements - 1, dtype=np.int32)
        pf = np.ascontiguousarray(cm.primary_faces, dtype=np.int32)
        sf = np.ascontiguousarray(cm.secondary_faces, dtype=np.int32)
        rv = np.ascontiguousarray(cm.secondary_reversed, dtype=np.int32)
        self._keep = (Ja, ij, pe, se, pf, sf, rv)
        self.h = lib().oracle_create_curved(polydeg, gamma, flux_kind, speed_kind, self.E, _p(Ja), _p(ij), len(pe),
                                            _p(pe), _p(pf), _p(se), _p(sf), _p(rv))
        if not self.h:
            raise RuntimeError("oracle_create_curved failed")
        if getattr(cm, "n_mortars", 0):
            self.set_curved_mortars(cm.mortar_small1, cm.mortar_small2, cm.mortar_small_faces, cm.mortar_large,
                                    cm.mortar_large_faces, cm.mortar_large_reversed)
        if getattr(cm, "unstructured", False):
            self.set_unstructured_normals(cm.unormals)

    def set_source(self, kind, node_coordinates=None):
        """Source terms (TreeMesh, LW and MDRK): kind 0 none, 1 source_terms_convergence_test; node coordinates
        [2, i, j, e] (the mesh's node_coordinates(N))."""
        if kind:
            self._xkeep = np.ascontiguousarray(node_coordinates, dtype=np.float64)
            assert lib().oracle_set_source(self.h, int(kind), _p(self._xkeep)) == 0
        else:
            assert lib().oracle_set_source(self.h, 0, None) == 0

    def set_unstructured_normals(self, normals):
        """UnstructuredMesh2D interface conventions with the caller's outward normals by face, (E, 4, n, 2); None:
        back to the StructuredMesh / P4estMesh ones."""
        if normals is None:
            assert lib().oracle_set_unstructured_normals(self.h, None) == 0
            return
        self._nkeep = np.ascontiguousarray(normals, dtype=np.float64)
        assert lib().oracle_set_unstructured_normals(self.h, _p(self._nkeep)) == 0

    def __del__(self):
        try:
            if self.h:
                lib().oracle_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def size(self):
        return 4 * self.n * self.n * self.E

    def set_temporal_errors(self, on=True, abstol: float = 1e-6, reltol: float = 1e-6):
        """Compute lw_volume_kernel_4!'s temporal error estimate (get(4) after rhs)."""
        lib().oracle_set_temporal_errors(self.h, 1 if on else 0, float(abstol), float(reltol))

    def set_parabolic(self, mu: float, Pr: float = 0.72):
        """Compressible Navier-Stokes with dynamic viscosity mu and Prandtl number Pr (periodic TreeMesh)."""
        assert lib().oracle_set_parabolic(self.h, float(mu), float(Pr)) == 0

    def set_boundary_kinds(self, kinds):
        """Per boundary (the mesh's boundary order): 0 Dirichlet, 1 slip wall vertical, 2 slip wall horizontal."""
        self._kkeep = np.ascontiguousarray(kinds, dtype=np.int32)
        assert lib().oracle_set_boundary_kinds(self.h, _p(self._kkeep)) == 0

    def set_curved_boundaries(self, elements, faces, kinds):
        """Boundary faces of a curvilinear mesh: elements 1-based, faces 0..3, kinds 1 (slip wall vertical) or
        2 (slip wall horizontal)."""
        self._cbkeep = (np.ascontiguousarray(np.asarray(elements) - 1, dtype=np.int32),
                        np.ascontiguousarray(faces, dtype=np.int32), np.ascontiguousarray(kinds, dtype=np.int32))
        assert lib().oracle_set_curved_boundaries(self.h, len(self._cbkeep[0]), *[_p(a) for a in self._cbkeep]) == 0

    def set_curved_mortars(self, small1, small2, small_faces, large, large_faces, large_reversed):
        """L2 mortars of a curvilinear mesh: elements 1-based, faces 0..3."""
        a = [np.ascontiguousarray(np.asarray(x) - (1 if k in (0, 1, 3) else 0), dtype=np.int32)
             for k, x in enumerate((small1, small2, small_faces, large, large_faces, large_reversed))]
        self._mkeep = a
        assert lib().oracle_set_curved_mortars(self.h, len(a[0]), *[_p(x) for x in a]) == 0

    def set_curved_mortar_jacobian(self, inverse_jacobian=None):
        """lw_mortars.inverse_jacobian [mortar, l] of the shock-capturing blend at the mortars (None: zeros)."""
        if inverse_jacobian is None:
            assert lib().oracle_set_curved_mortar_jacobian(self.h, None) == 0
            return
        self._mjkeep = np.ascontiguousarray(inverse_jacobian, dtype=np.float64).reshape(-1)
        assert lib().oracle_set_curved_mortar_jacobian(self.h, _p(self._mjkeep)) == 0

    def set_walls(self, kinds, data):
        """Navier-Stokes walls per boundary (1 no-slip adiabatic, 2 no-slip isothermal), data [B, l, 3] =
        (v1, v2, q or T) per boundary node."""
        self._wkeep = (np.ascontiguousarray(kinds, dtype=np.int32), np.ascontiguousarray(data, dtype=np.float64))
        assert lib().oracle_set_walls(self.h, _p(self._wkeep[0]), _p(self._wkeep[1])) == 0

    def set_positivity_limiter(self, thresholds=(5.0e-6, 5.0e-6), variables=(0, 1)):
        """Zhang-Shu limiter pairs applied after every step of ``steps`` (variables: 0 density, 1 pressure,
        2 density_pressure); an empty tuple switches it off."""
        self._lkeep = (np.ascontiguousarray(thresholds, dtype=np.float64),
                       np.ascontiguousarray(variables, dtype=np.int32))
        assert lib().oracle_set_limiter(self.h, len(thresholds), _p(self._lkeep[0]), _p(self._lkeep[1])) == 0

    def apply_positivity_limiter(self, u):
        """One application of the limiter to a copy of u."""
        u = np.array(u, dtype=np.float64, copy=True)
        assert lib().oracle_apply_limiter(self.h, _p(u)) == 0
        return u

    def set_shock_capturing(self, on=True, alpha_max=0.5, alpha_min=0.001, alpha_smooth=True, reconstruction=0):
        lib().oracle_set_shock_capturing(self.h, 1 if on else 0, alpha_max, alpha_min, 1 if alpha_smooth else 0)
        lib().oracle_set_reconstruction(self.h, int(reconstruction))

    def set_boundary_data(self, levels: np.ndarray, now: np.ndarray):
        self._bkeep = (np.ascontiguousarray(levels, dtype=np.float64), np.ascontiguousarray(now, dtype=np.float64))
        lib().oracle_set_boundary_data(self.h, _p(self._bkeep[0]), _p(self._bkeep[1]))

    def rhs(self, u, t, dt, kind: int = 0, us=None, nthreads: int = 1):
        u = np.ascontiguousarray(u, dtype=np.float64)
        us = None if us is None else np.ascontiguousarray(us, dtype=np.float64)
        du = np.empty_like(u)
        rc = lib().oracle_rhs(self.h, kind, _p(u), _p(us), _p(du), float(t), float(dt), nthreads)
        if rc == 3:
            raise OracleDomainError("sqrt of a negative number")
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error(self.h).decode())
        return du

    def adjoint_step(self, u, dt, lam, nthreads: int = 1):
        """(d u_new / d u)^T lam for one LW step u_new = u + dt rhs(u) at fixed dt."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        out = np.empty_like(u)
        rc = lib().oracle_adjoint_step(self.h, _p(u), float(dt), _p(lam), _p(out), nthreads)
        if rc == 3:
            raise OracleDomainError("sqrt of a negative number")
        if rc == 4:
            raise ValueError("adjoint: periodic mesh, FR volume integral, Rusanov flux and N >= 3 only")
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error(self.h).decode())
        return out

    def dual_step(self, u, dt, direction=None, kind: int = 0):
        """One step (kind 0 LW, 1 MDRK) of the scalar-templated restatement at a fixed dt (periodic TreeMesh, FR,
        Rusanov): returns the new state, and with a direction also its directional derivative (forward-mode dual
        numbers)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(u)
        d = None if direction is None else np.ascontiguousarray(direction, dtype=np.float64)
        dout = None if d is None else np.empty_like(u)
        rc = lib().oracle_dual_step(self.h, int(kind), _p(u), _p(d), float(dt), _p(out), _p(dout))
        if rc == 4:
            raise ValueError("dual step: periodic TreeMesh, FR volume integral, Rusanov flux and N >= 3 only")
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error(self.h).decode())
        return out if d is None else (out, dout)

    def step_fixed(self, u, dt, nthreads: int = 1):
        """One LW step u + dt rhs(u) at the given dt (returns a new array)."""
        return u + dt * self.rhs(u, 0.0, dt, nthreads=nthreads)

    def get(self, which: int) -> np.ndarray:
        sizes = {0: self.size(), 1: 2 * self.size(), 2: self.size(), 3: 2 * self.size(), 4: self.E,
                 5: 4 * self.n * 4 * self.E, 6: self.E, 7: 4 * self.n * 4 * self.E, 8: 2}
        out = np.empty(sizes[which])
        assert lib().oracle_get(self.h, which, _p(out)) == 0
        return out

    def max_dt(self, u, cfl):
        u = np.ascontiguousarray(u, dtype=np.float64)
        dt = lib().oracle_max_dt(self.h, _p(u), float(cfl))
        if dt < 0:
            raise OracleDomainError("sqrt of a negative number in max_dt")
        return dt

    def steps(self, u, nsteps: int, cfl: float, t: float, t_end: float, kind: int = 0, fixed_dt: float = 0.0,
              nthreads: int = 1):
        """In-place CFL steps; returns (steps_taken, t)."""
        assert u.dtype == np.float64 and u.flags.c_contiguous
        tt = ctypes.c_double(t)
        s = lib().oracle_steps(self.h, kind, _p(u), int(nsteps), float(cfl), float(fixed_dt), ctypes.byref(tt),
                               float(t_end), nthreads)
        if s < 0:
            raise OracleDomainError("oracle step failed")
        return s, tt.value
