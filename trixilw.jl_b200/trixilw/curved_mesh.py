"""Curvilinear conforming meshes built on the host: StructuredMesh{2} from a mapping, and the generic
form (primary / secondary element faces) that P4estMesh{2} and UnstructuredMesh2D reduce to.

Metric terms as Trixi computes them for 2D curved meshes (from the mathematics: the derivative matrix
applied to the nodal coordinates of each element):
    x_xi = D x (along i), x_eta = D x (along j), same for y
    Ja^1 = (y_eta, -x_eta),  Ja^2 = (-y_xi, x_xi),  J = x_xi y_eta - x_eta y_xi,  inverse_jacobian = 1 / J
stored as contravariant_vectors[d, a, i, j, element] = Ja^a_d (Trixi's layout) and inverse_jacobian[i, j, e].

StructuredMesh{2}(cells_per_dimension, mapping): elements in column-major cell order (x fastest), node
coordinates mapping(xi_g, eta_g) at the global reference coordinates of the GLL nodes, computed as
(cell + (xi + 1) / 2) * 2 / cells - 1 so that the two elements of a face see bitwise identical face nodes
(Trixi writes the same points as -1 + (cell - 1) dx + dx / 2 (1 + xi)). Interfaces take the right / upper
element as primary (its -xi / -eta face), which is the normal StructuredMesh's calc_interface_flux! uses
(src/solvers/dgsem_structured/dg_2d.jl:2233-2267). A non-periodic direction has boundary faces instead of the
wrap-around interfaces, listed by direction (x_neg: the -xi faces of the first column, x_pos, y_neg, y_pos),
as a P4estMesh's named boundaries :x_neg, :x_pos, :y_neg, :y_pos.
"""
from __future__ import annotations

import numpy as np

from .basis import derivative_matrix, gauss_lobatto


def metric_terms(xy: np.ndarray, polydeg: int):
    """(Ja [E, j, i, 4] = Ja^1_1, Ja^1_2, Ja^2_1, Ja^2_2 per node, inverse_jacobian [E, j, i]) of node
    coordinates xy [2, n(i), n(j), E]."""
    D = derivative_matrix(polydeg)
    x = np.transpose(xy[0], (2, 1, 0))   # [E, j, i]
    y = np.transpose(xy[1], (2, 1, 0))
    x_xi = np.einsum("ik,ejk->eji", D, x)
    y_xi = np.einsum("ik,ejk->eji", D, y)
    x_eta = np.einsum("jk,eki->eji", D, x)
    y_eta = np.einsum("jk,eki->eji", D, y)
    Ja = np.stack([y_eta, -x_eta, -y_xi, x_xi], axis=-1)
    J = x_xi * y_eta - x_eta * y_xi
    return np.ascontiguousarray(Ja), np.ascontiguousarray(1.0 / J)


class CurvedMesh:
    """A conforming curvilinear mesh in the form the library takes: per node metric terms and per
    interface (primary element, face; secondary element, face; secondary index reversed). Faces 0: -xi
    (i = 1), 1: +xi (i = n), 2: -eta (j = 1), 3: +eta (j = n); elements 1-based as Trixi stores them.
    A non-conforming one (RefinedStructuredMesh) also lists L2 mortars (mortar_* arrays)."""

    n_boundaries = 0
    n_mortars = 0

    def __init__(self, xy: np.ndarray, polydeg: int, primary_elements, primary_faces, secondary_elements,
                 secondary_faces, secondary_reversed, area: float, boundary_elements=(), boundary_faces=(),
                 n_boundaries_per_direction=(0, 0, 0, 0)):
        self.polydeg = polydeg
        self.xy = np.ascontiguousarray(xy)                   # [2, n, n, E]
        self.n_elements = xy.shape[-1]
        self.Ja, self.inverse_jacobian_nodes = metric_terms(xy, polydeg)
        if np.any(self.inverse_jacobian_nodes <= 0):
            raise ValueError("the mapping must preserve orientation (positive Jacobian)")
        self.primary_elements = np.ascontiguousarray(primary_elements, dtype=np.int64)
        self.primary_faces = np.ascontiguousarray(primary_faces, dtype=np.int32)
        self.secondary_elements = np.ascontiguousarray(secondary_elements, dtype=np.int64)
        self.secondary_faces = np.ascontiguousarray(secondary_faces, dtype=np.int32)
        self.secondary_reversed = np.ascontiguousarray(secondary_reversed, dtype=np.int32)
        self.n_interfaces = len(self.primary_elements)
        self.area = float(area)
        # boundary faces, grouped by direction (x_neg, x_pos, y_neg, y_pos); elements 1-based
        self.boundary_elements = np.ascontiguousarray(boundary_elements, dtype=np.int64)
        self.boundary_faces = np.ascontiguousarray(boundary_faces, dtype=np.int32)
        self.n_boundaries = len(self.boundary_elements)
        self.n_boundaries_per_direction = np.asarray(n_boundaries_per_direction, dtype=np.int64)

    def node_coordinates(self, polydeg: int) -> np.ndarray:
        if polydeg != self.polydeg:
            raise ValueError("this curved mesh was built for polydeg %d" % self.polydeg)
        return self.xy

    def boundary_node_coordinates(self, polydeg: int) -> np.ndarray:
        """[2, n, B] coordinates of each boundary face's nodes in the element's own index order."""
        xy = self.node_coordinates(polydeg)
        n = polydeg + 1
        out = np.empty((2, n, self.n_boundaries))
        for b, (e, f) in enumerate(zip(self.boundary_elements - 1, self.boundary_faces)):
            out[:, :, b] = (xy[:, 0, :, e] if f == 0 else xy[:, n - 1, :, e] if f == 1 else
                            xy[:, :, 0, e] if f == 2 else xy[:, :, n - 1, e])
        return out

    def ndofs(self, polydeg: int) -> int:
        return self.n_elements * (polydeg + 1) ** 2

    def jacobian_nodes(self) -> np.ndarray:
        """|J| per node [E, j, i] (quadrature weight factor)."""
        return 1.0 / self.inverse_jacobian_nodes


class StructuredMesh:
    """StructuredMesh{2}(cells_per_dimension, mapping; periodicity = true). ``mapping(xi, eta)`` maps the
    reference square [-1, 1]^2 onto the domain (vectorised over numpy arrays) and must be periodic-compatible:
    opposite sides of the square map to sides that differ by a translation."""

    n_boundaries = 0

    def __init__(self, cells_per_dimension, mapping, periodicity=True):
        if isinstance(periodicity, bool):
            periodicity = (periodicity, periodicity)
        self.periodicity = tuple(bool(p) for p in periodicity)
        self.cells = tuple(int(c) for c in cells_per_dimension)
        self.mapping = mapping
        nx, ny = self.cells
        self.n_elements = nx * ny
        px, py = self.periodicity
        self.n_boundaries_per_direction = np.array([0 if px else ny, 0 if px else ny, 0 if py else nx, 0 if py else nx],
                                                   dtype=np.int64)
        self.n_boundaries = int(self.n_boundaries_per_direction.sum())
        self._curved = {}

    def element(self, cx, cy):
        return cx + self.cells[0] * cy

    def node_coordinates(self, polydeg: int) -> np.ndarray:
        nodes, _ = gauss_lobatto(polydeg)
        nx, ny = self.cells
        cx = np.arange(nx)
        cy = np.arange(ny)
        xi_g = (cx[:, None] + 0.5 * (nodes[None, :] + 1.0)) * (2.0 / nx) - 1.0    # [cx, i]
        eta_g = (cy[:, None] + 0.5 * (nodes[None, :] + 1.0)) * (2.0 / ny) - 1.0   # [cy, j]
        n = len(nodes)
        e = np.arange(self.n_elements)
        XI = np.ascontiguousarray(np.broadcast_to(xi_g[e % nx].T[:, None, :], (n, n, self.n_elements)))
        ETA = np.ascontiguousarray(np.broadcast_to(eta_g[e // nx].T[None, :, :], (n, n, self.n_elements)))
        x, y = self.mapping(XI, ETA)
        return np.stack([np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)])

    def curved(self, polydeg: int) -> CurvedMesh:
        if polydeg not in self._curved:
            nx, ny = self.cells
            px, py = self.periodicity
            pe, pf, se, sf = [], [], [], []
            for cy in range(ny):
                for cx in range(nx):
                    if cx == 0 and not px:
                        continue
                    e = self.element(cx, cy)
                    pe.append(e); pf.append(0); se.append(self.element((cx - 1) % nx, cy)); sf.append(1)
            for cy in range(ny):
                for cx in range(nx):
                    if cy == 0 and not py:
                        continue
                    e = self.element(cx, cy)
                    pe.append(e); pf.append(2); se.append(self.element(cx, (cy - 1) % ny)); sf.append(3)
            be, bf = [], []
            if not px:
                for face, cx in ((0, 0), (1, nx - 1)):
                    for cy in range(ny):
                        be.append(self.element(cx, cy)); bf.append(face)
            if not py:
                for face, cy in ((2, 0), (3, ny - 1)):
                    for cx in range(nx):
                        be.append(self.element(cx, cy)); bf.append(face)
            xy = self.node_coordinates(polydeg)
            area = float(np.einsum("eji,j,i->", 1.0 / metric_terms(xy, polydeg)[1], *(2 * [gauss_lobatto(polydeg)[1]])))
            self._curved[polydeg] = CurvedMesh(xy, polydeg, np.array(pe) + 1, pf, np.array(se) + 1, sf,
                                               np.zeros(len(pe), dtype=np.int32), area, np.array(be, dtype=np.int64) + 1,
                                               bf, self.n_boundaries_per_direction)
        return self._curved[polydeg]

    def ndofs(self, polydeg: int) -> int:
        return self.n_elements * (polydeg + 1) ** 2

    def boundary_node_coordinates(self, polydeg: int) -> np.ndarray:
        return self.curved(polydeg).boundary_node_coordinates(polydeg)


class RefinedStructuredMesh:
    """A StructuredMesh{2}-like mesh with some cells refined once into four children, as a P4estMesh{2} is after an
    AMR step: elements are the unrefined cells and the children (each in the order of its parent cell, children
    lower-left, lower-right, upper-left, upper-right), node coordinates mapping(xi_g, eta_g) of each element's box
    in the reference square. Faces between equal elements are interfaces (the right / upper element primary, as
    on the StructuredMesh); a refined cell next to an unrefined one gives an L2 mortar: the two children on
    their faces (position 1 at the smaller coordinate along the face, the large face's index running forward)
    against the unrefined cell's face. Non-periodic directions have boundary faces, by direction."""

    def __init__(self, cells_per_dimension, mapping, refined_cells, periodicity=True):
        if isinstance(periodicity, bool):
            periodicity = (periodicity, periodicity)
        self.periodicity = tuple(bool(p) for p in periodicity)
        self.cells = tuple(int(c) for c in cells_per_dimension)
        self.mapping = mapping
        self.refined = {(int(a), int(b)) for a, b in refined_cells}
        nx, ny = self.cells
        self.boxes = []          # (level, ix, iy) with ix, iy in units of the level's cell size
        self.index = {}
        for cy in range(ny):
            for cx in range(nx):
                if (cx, cy) in self.refined:
                    for dy in (0, 1):
                        for dx in (0, 1):
                            self.index[(1, 2 * cx + dx, 2 * cy + dy)] = len(self.boxes)
                            self.boxes.append((1, 2 * cx + dx, 2 * cy + dy))
                else:
                    self.index[(0, cx, cy)] = len(self.boxes)
                    self.boxes.append((0, cx, cy))
        self.n_elements = len(self.boxes)
        px, py = self.periodicity
        side = lambda cells: sum(2 if c in self.refined else 1 for c in cells)
        self.n_boundaries_per_direction = np.array(
            [0 if px else side([(0, cy) for cy in range(ny)]), 0 if px else side([(nx - 1, cy) for cy in range(ny)]),
             0 if py else side([(cx, 0) for cx in range(nx)]), 0 if py else side([(cx, ny - 1) for cx in range(nx)])],
            dtype=np.int64)
        self.n_boundaries = int(self.n_boundaries_per_direction.sum())
        self._curved = {}

    def boundary_node_coordinates(self, polydeg: int) -> np.ndarray:
        return self.curved(polydeg).boundary_node_coordinates(polydeg)

    def node_coordinates(self, polydeg: int) -> np.ndarray:
        nodes, _ = gauss_lobatto(polydeg)
        nx, ny = self.cells
        n = len(nodes)
        XI = np.empty((n, n, self.n_elements))
        ETA = np.empty((n, n, self.n_elements))
        for e, (lev, ix, iy) in enumerate(self.boxes):
            s = 1 << lev
            xi = (ix + 0.5 * (nodes + 1.0)) * (2.0 / (nx * s)) - 1.0
            eta = (iy + 0.5 * (nodes + 1.0)) * (2.0 / (ny * s)) - 1.0
            XI[:, :, e] = xi[:, None]
            ETA[:, :, e] = eta[None, :]
        x, y = self.mapping(XI, ETA)
        return np.stack([np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)])

    def _cell_refined(self, cx, cy):
        return (cx % self.cells[0], cy % self.cells[1]) in self.refined

    def curved(self, polydeg: int) -> CurvedMesh:
        if polydeg in self._curved:
            return self._curved[polydeg]
        nx, ny = self.cells
        px, py = self.periodicity
        pe, pf, se, sf = [], [], [], []
        ms1, ms2, msf, ml, mlf = [], [], [], [], []
        bnd = {0: [], 1: [], 2: [], 3: []}
        for e, (lev, ix, iy) in enumerate(self.boxes):
            s = 1 << lev
            for d in (0, 1):   # the element's + face in direction d: +xi (face 1) or +eta (face 3)
                jx, jy = (ix + 1, iy) if d == 0 else (ix, iy + 1)
                cells_d = (nx if d == 0 else ny) * s
                at_edge = (jx if d == 0 else jy) == cells_d
                periodic = px if d == 0 else py
                if at_edge and not periodic:
                    bnd[2 * d + 1].append((e, 2 * d + 1))
                    continue
                jx, jy = jx % (nx * s), jy % (ny * s)
                # the neighbour cell at the base level and whether it is refined
                bx, by = (jx // s, jy // s)
                nref = (bx, by) in self.refined
                if lev == 0 and nref:
                    # mortar: this (large) element's + face against the two children on their - faces
                    if d == 0:
                        kids = [self.index[(1, 2 * bx, 2 * by)], self.index[(1, 2 * bx, 2 * by + 1)]]
                    else:
                        kids = [self.index[(1, 2 * bx, 2 * by)], self.index[(1, 2 * bx + 1, 2 * by)]]
                    ms1.append(kids[0]); ms2.append(kids[1]); msf.append(2 * d); ml.append(e); mlf.append(2 * d + 1)
                elif lev == 1 and not nref:
                    # the neighbour is a large element: a mortar, once per pair of children (the lower / left one)
                    if (iy if d == 0 else ix) % 2 == 0:
                        large = self.index[(0, bx, by)]
                        if d == 0:
                            kids = [e, self.index[(1, ix, iy + 1)]]
                        else:
                            kids = [e, self.index[(1, ix + 1, iy)]]
                        ms1.append(kids[0]); ms2.append(kids[1]); msf.append(2 * d + 1); ml.append(large); mlf.append(2 * d)
                else:
                    other = self.index[(lev, jx, jy)]
                    pe.append(other); pf.append(2 * d); se.append(e); sf.append(2 * d + 1)
            # the element's - faces on a non-periodic edge
            for d in (0, 1):
                if (ix if d == 0 else iy) == 0 and not (px if d == 0 else py):
                    bnd[2 * d].append((e, 2 * d))
        be = [b[0] for f in (0, 1, 2, 3) for b in bnd[f]]
        bf = [b[1] for f in (0, 1, 2, 3) for b in bnd[f]]
        per = np.array([len(bnd[f]) for f in (0, 1, 2, 3)], dtype=np.int64)
        xy = self.node_coordinates(polydeg)
        area = float(np.einsum("eji,j,i->", 1.0 / metric_terms(xy, polydeg)[1], *(2 * [gauss_lobatto(polydeg)[1]])))
        cm = CurvedMesh(xy, polydeg, np.array(pe) + 1, pf, np.array(se) + 1, sf, np.zeros(len(pe), dtype=np.int32),
                        area, np.array(be, dtype=np.int64) + 1, bf, per)
        cm.n_mortars = len(ml)
        cm.mortar_small1 = np.array(ms1, dtype=np.int64) + 1
        cm.mortar_small2 = np.array(ms2, dtype=np.int64) + 1
        cm.mortar_small_faces = np.array(msf, dtype=np.int32)
        cm.mortar_large = np.array(ml, dtype=np.int64) + 1
        cm.mortar_large_faces = np.array(mlf, dtype=np.int32)
        cm.mortar_large_reversed = np.zeros(len(ml), dtype=np.int32)
        assert np.array_equal(per, self.n_boundaries_per_direction)
        self._curved[polydeg] = cm
        return cm

    def ndofs(self, polydeg: int) -> int:
        return self.n_elements * (polydeg + 1) ** 2


# rotation of an element's local frame by a quarter turn: new node (a, b) holds old node (n-1-b, a);
# old face f becomes new face _FACE_ROT[f], and the index along it runs backwards when _FLIP_ROT[f]
_FACE_ROT = (3, 2, 0, 1)
_FLIP_ROT = (0, 0, 1, 1)


def rotate_elements(mesh: CurvedMesh, turns) -> CurvedMesh:
    """The same mesh with element e's local frame turned by turns[e] quarter turns (P4est-like element
    orientations: faces and face directions no longer line up). Metrics are recomputed from the rotated
    node coordinates. Use rotate_state to carry states along."""
    turns = np.asarray(turns, dtype=np.int64) % 4
    xy = mesh.xy.copy()
    for r in range(1, 4):
        sel = turns == r
        for _ in range(r):
            xy[:, :, :, sel] = rot_nodes(xy[:, :, :, sel])
    def face_map(f, r):
        flip = 0
        for _ in range(r):
            flip ^= _FLIP_ROT[f]
            f = _FACE_ROT[f]
        return f, flip
    pe = mesh.primary_elements - 1
    se = mesh.secondary_elements - 1
    pf, sf, rev = [], [], []
    for k in range(mesh.n_interfaces):
        fp, flp = face_map(int(mesh.primary_faces[k]), int(turns[pe[k]]))
        fs, fls = face_map(int(mesh.secondary_faces[k]), int(turns[se[k]]))
        pf.append(fp); sf.append(fs); rev.append(int(mesh.secondary_reversed[k]) ^ flp ^ fls)
    bf = [face_map(int(f), int(turns[e - 1]))[0] for e, f in zip(mesh.boundary_elements, mesh.boundary_faces)]
    return CurvedMesh(xy, mesh.polydeg, mesh.primary_elements, pf, mesh.secondary_elements, sf, rev, mesh.area,
                      mesh.boundary_elements, bf, mesh.n_boundaries_per_direction)


def rot_nodes(a: np.ndarray) -> np.ndarray:
    """One quarter turn of node arrays [..., n(i), n(j), E]: new[a, b] = old[n-1-b, a]."""
    n = a.shape[-3]
    out = np.empty_like(a)
    for ia in range(n):
        for ib in range(n):
            out[..., ia, ib, :] = a[..., n - 1 - ib, ia, :]
    return out


def rotate_state(u: np.ndarray, polydeg: int, turns) -> np.ndarray:
    """Carry a flat state [v, i, j, e] into the rotated frames of rotate_elements."""
    n = polydeg + 1
    turns = np.asarray(turns, dtype=np.int64) % 4
    E = len(turns)
    x = np.transpose(u.reshape(E, n, n, 4), (3, 2, 1, 0)).copy()    # [v, i, j, e]
    for r in range(1, 4):
        sel = turns == r
        for _ in range(r):
            x[:, :, :, sel] = rot_nodes(x[:, :, :, sel])
    return np.ascontiguousarray(np.transpose(x, (3, 2, 1, 0))).reshape(-1)
