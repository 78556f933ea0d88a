"""TreeMesh{2} connectivity built on the host, in Trixi's conventions.

The Julia host side of the reference gets these arrays from Trixi.jl's TreeMesh and containers; this
module reproduces them for a uniformly refined tree so that the library can be driven without Julia:

* elements: leaves of a uniformly refined quadtree in Trixi's cell order (children appended in the
  order (-x,-y), (+x,-y), (-x,+y), (+x,+y) at each refinement, i.e. Morton order with x the low bit);
* interfaces: per element, +x then +y neighbour, (left, right) = (element, neighbour), orientation
  1 (x) / 2 (y) (Trixi ``init_interfaces!``);
* boundaries: sorted by direction 1..4 (-x, +x, -y, +y), then element; neighbor_sides 2 for odd
  directions (element on the + side), 1 for even (Trixi ``init_boundaries!``);
* inverse_jacobian = 2 / element length.

All ids are 1-based Int64, exactly as Trixi stores them; the library converts them on upload.
"""
from __future__ import annotations

import numpy as np

from .basis import gauss_lobatto


def _morton_decode(codes: np.ndarray, level: int):
    ix = np.zeros_like(codes)
    iy = np.zeros_like(codes)
    for b in range(level):
        ix |= ((codes >> (2 * b)) & 1) << b
        iy |= ((codes >> (2 * b + 1)) & 1) << b
    return ix, iy


class TreeMesh:
    """Uniform TreeMesh{2}: ``TreeMesh(coordinates_min, coordinates_max, initial_refinement_level,
    periodicity)`` with 2^level x 2^level elements."""

    def __init__(self, coordinates_min, coordinates_max, initial_refinement_level: int, periodicity=True):
        if isinstance(periodicity, bool):
            periodicity = (periodicity, periodicity)
        self.periodicity = tuple(bool(p) for p in periodicity)
        self.level = int(initial_refinement_level)
        self.coordinates_min = np.asarray(coordinates_min, dtype=np.float64)
        self.coordinates_max = np.asarray(coordinates_max, dtype=np.float64)
        # Trixi's tree is a square: centre of the bounding box, length of its longest side
        self.center = 0.5 * (self.coordinates_min + self.coordinates_max)
        self.length = float(np.max(self.coordinates_max - self.coordinates_min))
        m = 1 << self.level
        self.cells_per_dimension = m
        codes = np.arange(m * m, dtype=np.int64)
        self.ix, self.iy = _morton_decode(codes, self.level)
        self.n_elements = m * m
        self.element_length = self.length / m
        lo = self.center - 0.5 * self.length
        self.element_centers = np.stack([lo[0] + (self.ix + 0.5) * self.element_length,
                                         lo[1] + (self.iy + 0.5) * self.element_length], axis=1)
        self.inverse_jacobian = np.full(self.n_elements, 2.0 / self.element_length)
        # element id from (ix, iy)
        self.element_at = np.empty((m, m), dtype=np.int64)
        self.element_at[self.ix, self.iy] = np.arange(self.n_elements)
        self._build_interfaces()
        self._build_boundaries()

    def _neighbors(self, direction):
        """Neighbour element (0-based) of every element in Trixi direction 1..4, -1 where none."""
        m = self.cells_per_dimension
        dx, dy = {1: (-1, 0), 2: (1, 0), 3: (0, -1), 4: (0, 1)}[direction]
        jx, jy = self.ix + dx, self.iy + dy
        ok = np.ones(self.n_elements, dtype=bool)
        if direction in (1, 2):
            if self.periodicity[0]:
                jx %= m
            else:
                ok &= (jx >= 0) & (jx < m)
        else:
            if self.periodicity[1]:
                jy %= m
            else:
                ok &= (jy >= 0) & (jy < m)
        nb = np.full(self.n_elements, -1, dtype=np.int64)
        nb[ok] = self.element_at[jx[ok], jy[ok]]
        return nb

    def _build_interfaces(self):
        # per element (in element order): the +x interface, then the +y interface (Trixi init_interfaces!)
        e = np.arange(self.n_elements, dtype=np.int64)
        pairs = np.full((self.n_elements, 2, 2), -1, dtype=np.int64)
        ors = np.zeros((self.n_elements, 2), dtype=np.int64)
        for k, direction in enumerate((2, 4)):
            nb = self._neighbors(direction)
            pairs[:, k, 0] = e
            pairs[:, k, 1] = nb
            ors[:, k] = direction // 2
        keep = pairs[:, :, 1] >= 0
        self.interface_neighbor_ids = np.ascontiguousarray(pairs[keep] + 1)
        self.interface_orientations = np.ascontiguousarray(ors[keep])
        self.n_interfaces = int(keep.sum())

    def _build_boundaries(self):
        # grouped by direction 1..4, element order inside a direction (Trixi init_boundaries!)
        elem, per_dir = [], []
        for direction in (1, 2, 3, 4):
            missing = np.nonzero(self._neighbors(direction) < 0)[0]
            elem.append(missing + 1)
            per_dir.append(len(missing))
        self.n_boundaries_per_direction = np.array(per_dir, dtype=np.int64)
        self.boundary_neighbor_ids = np.concatenate(elem).astype(np.int64)
        self.boundary_directions = np.repeat(np.arange(1, 5, dtype=np.int64), per_dir)
        self.boundary_orientations = np.where(self.boundary_directions <= 2, 1, 2).astype(np.int64)
        self.boundary_neighbor_sides = np.where(self.boundary_directions % 2 == 0, 1, 2).astype(np.int64)
        self.n_boundaries = int(len(self.boundary_neighbor_ids))

    def node_coordinates(self, polydeg: int) -> np.ndarray:
        """[2, n, n, E] node coordinates (x, y) as Trixi's elements.node_coordinates."""
        nodes, _ = gauss_lobatto(polydeg)
        h = 0.5 * self.element_length
        x = self.element_centers[:, 0][None, None, :] + h * nodes[:, None, None]   # [i, 1, E]
        y = self.element_centers[:, 1][None, None, :] + h * nodes[None, :, None]   # [1, j, E]
        n = len(nodes)
        out = np.empty((2, n, n, self.n_elements))
        out[0] = np.broadcast_to(x, (n, n, self.n_elements))
        out[1] = np.broadcast_to(y, (n, n, self.n_elements))
        return out

    def boundary_node_coordinates(self, polydeg: int) -> np.ndarray:
        """[2, n, B] coordinates of the face nodes of each boundary (Trixi boundaries.node_coordinates)."""
        xy = self.node_coordinates(polydeg)
        n = polydeg + 1
        out = np.empty((2, n, self.n_boundaries))
        for b, (e, d) in enumerate(zip(self.boundary_neighbor_ids - 1, self.boundary_directions)):
            if d == 1:
                out[:, :, b] = xy[:, 0, :, e]
            elif d == 2:
                out[:, :, b] = xy[:, n - 1, :, e]
            elif d == 3:
                out[:, :, b] = xy[:, :, 0, e]
            else:
                out[:, :, b] = xy[:, :, n - 1, e]
        return out

    def ndofs(self, polydeg: int) -> int:
        return self.n_elements * (polydeg + 1) ** 2


class RefinedTreeMesh:
    """A non-conforming TreeMesh{2}: the uniform mesh of ``initial_refinement_level`` with the cells whose
    centres lie in ``refine_box`` ((xmin, ymin), (xmax, ymax)) refined once more, as an AMR step leaves it.
    Same-size neighbours share an interface; a coarse cell next to refined ones shares an L2 mortar with the
    two small cells (Trixi mortars container: neighbor_ids [lower, upper, large] per mortar, 1-based;
    large_sides 1 when the large element is on the -side, 2 on the +side; orientations 1 = x, 2 = y; for an
    x-mortar the lower small cell has the smaller y, for a y-mortar the smaller x). Periodic.

    Elements: the coarse leaves in Morton order, then the fine leaves (four children per refined cell in the
    order (-x,-y), (+x,-y), (-x,+y), (+x,+y))."""

    n_boundaries = 0

    def __init__(self, coordinates_min, coordinates_max, initial_refinement_level: int, refine_box):
        base = TreeMesh(coordinates_min, coordinates_max, initial_refinement_level, periodicity=True)
        self.length = base.length
        self.center = base.center
        m = base.cells_per_dimension
        lo = self.center - 0.5 * self.length
        h = base.element_length
        (bx0, by0), (bx1, by1) = refine_box
        cx = lo[0] + (base.ix + 0.5) * h
        cy = lo[1] + (base.iy + 0.5) * h
        refined = (cx >= bx0) & (cx <= bx1) & (cy >= by0) & (cy <= by1)
        if not refined.any() or refined.all():
            raise ValueError("the refine box must select some but not all cells")
        leaves = {}   # (level 0 coarse / 1 fine, ix, iy) -> element
        centers, lengths = [], []
        for k in range(base.n_elements):
            if not refined[k]:
                leaves[(0, int(base.ix[k]), int(base.iy[k]))] = len(centers)
                centers.append((cx[k], cy[k]))
                lengths.append(h)
        for k in range(base.n_elements):
            if refined[k]:
                for dy in (0, 1):
                    for dx in (0, 1):
                        fx, fy = 2 * int(base.ix[k]) + dx, 2 * int(base.iy[k]) + dy
                        leaves[(1, fx, fy)] = len(centers)
                        centers.append((lo[0] + (fx + 0.5) * h / 2, lo[1] + (fy + 0.5) * h / 2))
                        lengths.append(h / 2)
        self.n_elements = len(centers)
        self.element_centers = np.array(centers)
        self.element_lengths = np.array(lengths)
        self.inverse_jacobian = 2.0 / self.element_lengths
        il, ir, io, ml, mu, mg, ms, mo = [], [], [], [], [], [], [], []
        for (lev, ix, iy), e in leaves.items():
            mm = m << lev
            for o, (dx, dy) in ((1, (1, 0)), (2, (0, 1))):
                nb = leaves.get((lev, (ix + dx) % mm, (iy + dy) % mm))
                if nb is not None:
                    il.append(e); ir.append(nb); io.append(o)
            if lev == 0:
                # mortars: a refined same-level neighbour on either side in either direction
                for o, sgn in ((1, 1), (1, -1), (2, 1), (2, -1)):
                    nx, ny = (ix + sgn) % m if o == 1 else ix, (iy + sgn) % m if o == 2 else iy
                    if (0, nx, ny) in leaves:
                        continue
                    # the two children of (nx, ny) next to the shared face
                    if o == 1:
                        c = 2 * nx + (0 if sgn == 1 else 1)
                        lower, upper = leaves[(1, c, 2 * ny)], leaves[(1, c, 2 * ny + 1)]
                    else:
                        c = 2 * ny + (0 if sgn == 1 else 1)
                        lower, upper = leaves[(1, 2 * nx, c)], leaves[(1, 2 * nx + 1, c)]
                    ml.append(lower); mu.append(upper); mg.append(e); ms.append(1 if sgn == 1 else 2); mo.append(o)
        self.interface_neighbor_ids = (np.array([il, ir], dtype=np.int64) + 1).T.reshape(-1)
        self.interface_orientations = np.array(io, dtype=np.int64)
        self.n_interfaces = len(io)
        self.mortar_neighbor_ids = (np.array([ml, mu, mg], dtype=np.int64) + 1).T.reshape(-1)
        self.mortar_large_sides = np.array(ms, dtype=np.int64)
        self.mortar_orientations = np.array(mo, dtype=np.int64)
        self.n_mortars = len(mo)
        empty = np.zeros(0, dtype=np.int64)
        self.boundary_neighbor_ids = self.boundary_orientations = self.boundary_neighbor_sides = empty
        self.boundary_directions = empty
        self.n_boundaries_per_direction = np.zeros(4, dtype=np.int64)

    def node_coordinates(self, polydeg: int) -> np.ndarray:
        nodes, _ = gauss_lobatto(polydeg)
        hl = 0.5 * self.element_lengths
        x = self.element_centers[:, 0][None, None, :] + hl[None, None, :] * nodes[:, None, None]
        y = self.element_centers[:, 1][None, None, :] + hl[None, None, :] * nodes[None, :, None]
        n = len(nodes)
        out = np.empty((2, n, n, self.n_elements))
        out[0] = np.broadcast_to(x, (n, n, self.n_elements))
        out[1] = np.broadcast_to(y, (n, n, self.n_elements))
        return out

    def ndofs(self, polydeg: int) -> int:
        return self.n_elements * (polydeg + 1) ** 2
