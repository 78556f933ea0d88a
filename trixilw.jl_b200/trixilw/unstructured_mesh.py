"""UnstructuredMesh2D in Trixi's conventions, as the library takes it (tlw_set_unstructured_mesh).

Trixi's UnstructuredMesh2D numbers the sides of a quadrilateral element 1: bottom (j = 1, nodes (i, 1)),
2: right (i = n, nodes (n, i)), 3: top (j = n, nodes (i, n)), 4: left (i = 1, nodes (1, i)), and describes an
interface by element_ids[:, k] = (primary, secondary), element_side_ids[:, k], and the secondary's node index
along the primary's, start_index[k] + (i - 1) index_increment[k] (start 1 / increment 1, or start n / increment
-1). elements.normal_directions[:, i, side, e] is the outward (unnormalised) normal of a side at its node i,
which Trixi computes from the side's node coordinates (the derivative matrix along the side):
    side 1: (y_xi, -x_xi), side 2: (y_eta, -x_eta), side 3: (-y_xi, x_xi), side 4: (-y_eta, x_eta).
The reference's UnstructuredMesh2D path (src/solvers/dgsem_unstructured_2d/dg_2d.jl) is LW on conforming meshes
without boundaries; this class is such a mesh, built from node coordinates and the connectivity above, or from a
conforming periodic curvilinear mesh (``from_curved``, e.g. a StructuredMesh with rotated element frames, which
gives interfaces in every side pairing and with reversed secondary indices).
"""
from __future__ import annotations

import numpy as np

from .basis import derivative_matrix
from .curved_mesh import CurvedMesh

# sides as the curvilinear faces (0: -xi (i = 1), 1: +xi (i = n), 2: -eta (j = 1), 3: +eta (j = n)) and back
FACE_OF_SIDE = {1: 2, 2: 1, 3: 3, 4: 0}
SIDE_OF_FACE = (4, 2, 1, 3)


def side_normals(xy: np.ndarray, polydeg: int) -> np.ndarray:
    """normal_directions in Trixi's layout [2, n, 4, E] (returned as a C-ordered array of shape (E, 4, n, 2)) from
    node coordinates xy [2, n(i), n(j), E]: the derivative matrix applied along each side."""
    D = derivative_matrix(polydeg)
    x, y = xy[0], xy[1]
    E = xy.shape[-1]
    n = polydeg + 1
    out = np.empty((E, 4, n, 2))
    xs, ys = D @ x[:, 0, :], D @ y[:, 0, :]                         # bottom: along i at j = 1
    out[:, 0, :, 0], out[:, 0, :, 1] = ys.T, -xs.T
    xs, ys = D @ x[n - 1, :, :], D @ y[n - 1, :, :]                 # right: along j at i = n
    out[:, 1, :, 0], out[:, 1, :, 1] = ys.T, -xs.T
    xs, ys = D @ x[:, n - 1, :], D @ y[:, n - 1, :]                 # top: along i at j = n
    out[:, 2, :, 0], out[:, 2, :, 1] = -ys.T, xs.T
    xs, ys = D @ x[0, :, :], D @ y[0, :, :]                         # left: along j at i = 1
    out[:, 3, :, 0], out[:, 3, :, 1] = -ys.T, xs.T
    return np.ascontiguousarray(out)


class UnstructuredMesh2D(CurvedMesh):
    """A conforming UnstructuredMesh2D without boundaries. element_ids, element_side_ids: [2, I] (1-based elements,
    sides 1..4); start_index, index_increment: [I]; normal_directions: (E, 4, n, 2) = Trixi's [2, n, 4, E]
    (default: computed from xy as Trixi does). The curvilinear form (faces, reversed flags) is kept beside it for
    the metric terms and the checker."""

    unstructured = True

    def __init__(self, xy: np.ndarray, polydeg: int, element_ids, element_side_ids, start_index, index_increment,
                 area: float, normal_directions=None):
        n = polydeg + 1
        self.element_ids = np.ascontiguousarray(np.asarray(element_ids, dtype=np.int64).reshape(2, -1))
        self.element_side_ids = np.ascontiguousarray(np.asarray(element_side_ids, dtype=np.int64).reshape(2, -1))
        self.start_index = np.ascontiguousarray(start_index, dtype=np.int64)
        self.index_increment = np.ascontiguousarray(index_increment, dtype=np.int64)
        ok = ((self.start_index == 1) & (self.index_increment == 1)) | ((self.start_index == n) & (self.index_increment == -1))
        if not np.all(ok):
            raise ValueError("start_index / index_increment: (1, 1) or (n, -1)")
        pf = [FACE_OF_SIDE[int(s)] for s in self.element_side_ids[0]]
        sf = [FACE_OF_SIDE[int(s)] for s in self.element_side_ids[1]]
        super().__init__(xy, polydeg, self.element_ids[0], pf, self.element_ids[1], sf,
                         (self.index_increment == -1).astype(np.int32), area)
        self.normal_directions = (side_normals(self.xy, polydeg) if normal_directions is None
                                  else np.ascontiguousarray(normal_directions, dtype=np.float64).reshape(-1, 4, n, 2))

    @property
    def unormals(self) -> np.ndarray:
        """The normals by curvilinear face, (E, 4(face), n, 2) (the checker's layout)."""
        out = np.empty_like(self.normal_directions)
        for side in (1, 2, 3, 4):
            out[:, FACE_OF_SIDE[side]] = self.normal_directions[:, side - 1]
        return np.ascontiguousarray(out)

    @classmethod
    def from_curved(cls, cm: CurvedMesh) -> "UnstructuredMesh2D":
        """The unstructured form of a conforming curvilinear mesh without boundaries or mortars."""
        if cm.n_boundaries or getattr(cm, "n_mortars", 0):
            raise ValueError("UnstructuredMesh2D: conforming and without boundaries")
        n = cm.polydeg + 1
        sides = np.array([[SIDE_OF_FACE[int(f)] for f in cm.primary_faces],
                          [SIDE_OF_FACE[int(f)] for f in cm.secondary_faces]], dtype=np.int64)
        rev = np.asarray(cm.secondary_reversed, dtype=bool)
        return cls(cm.xy, cm.polydeg, np.stack([cm.primary_elements, cm.secondary_elements]), sides,
                   np.where(rev, n, 1), np.where(rev, -1, 1), cm.area)
