"""CPU tests of the host side: TreeMesh connectivity in Trixi's conventions, the C ABI library loads and
exports every symbol include/tlw.h declares, and the host helpers that mirror the reference."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_treemesh_periodic_connectivity(tl):
    m = tl.TreeMesh((-1.0, -1.0), (1.0, 1.0), 3)
    assert m.n_elements == 64 and m.n_interfaces == 128 and m.n_boundaries == 0
    # every element appears exactly once as left and once as right per orientation
    ids = m.interface_neighbor_ids - 1
    for o in (1, 2):
        sel = m.interface_orientations == o
        assert sorted(ids[sel, 0]) == list(range(64))
        assert sorted(ids[sel, 1]) == list(range(64))
    # right neighbour sits one cell further in +x / +y (periodically)
    for (l, r), o in zip(ids, m.interface_orientations):
        if o == 1:
            assert m.iy[l] == m.iy[r] and (m.ix[l] + 1) % 8 == m.ix[r]
        else:
            assert m.ix[l] == m.ix[r] and (m.iy[l] + 1) % 8 == m.iy[r]
    # Morton (Z) order with x the low bit: first four elements are the 2x2 block at the origin
    assert list(zip(m.ix[:4], m.iy[:4])) == [(0, 0), (1, 0), (0, 1), (1, 1)]
    np.testing.assert_allclose(m.inverse_jacobian, 2.0 / 0.25)


def test_treemesh_boundaries(tl):
    m = tl.TreeMesh((0.0, 0.0), (1.0, 1.0), 2, periodicity=False)
    assert m.n_boundaries == 16
    assert list(m.n_boundaries_per_direction) == [4, 4, 4, 4]
    assert list(m.boundary_orientations) == [1] * 8 + [2] * 8
    assert list(m.boundary_neighbor_sides) == [2] * 4 + [1] * 4 + [2] * 4 + [1] * 4
    e = m.boundary_neighbor_ids - 1
    assert np.all(m.ix[e[:4]] == 0) and np.all(m.ix[e[4:8]] == 3)
    assert np.all(m.iy[e[8:12]] == 0) and np.all(m.iy[e[12:]] == 3)
    assert m.n_interfaces == 2 * 4 * 3
    xy = m.boundary_node_coordinates(3)
    np.testing.assert_allclose(xy[0, :, :4], 0.0)
    np.testing.assert_allclose(xy[1, :, 12:], 1.0)


def test_node_coordinates(tl):
    m = tl.TreeMesh((-10.0, -10.0), (10.0, 10.0), 1)
    xy = m.node_coordinates(4)
    assert xy.shape == (2, 5, 5, 4)
    np.testing.assert_allclose(xy[0, 0, 0, 0], -10.0)
    np.testing.assert_allclose(xy[1, 4, 4, 3], 10.0)
    np.testing.assert_allclose(xy[0, 2, 3, 1], 5.0)


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "tlw.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tlw_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(tl):
    from trixilw import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    syms = _header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.EXPORTED)
    assert L.tlw_abi_version() == 2


def test_opts_struct_layout(tmp_path):
    """The ctypes mirror of tlw_opts matches the C compiler's layout of include/tlw.h."""
    import subprocess
    from trixilw._lib import TlwOpts
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "tlw.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu\\n", sizeof(tlw_opts), offsetof(tlw_opts, gamma),'
                   ' offsetof(tlw_opts, device), offsetof(tlw_opts, reserved));return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [ctypes.sizeof(TlwOpts), TlwOpts.gamma.offset, TlwOpts.device.offset, TlwOpts.reserved.offset]


def test_lw_cfl_table(tl):
    solver = tl.DGSEM(4)
    assert tl.trixi2lw(0.98, solver) == pytest.approx(0.98 * 5 * 0.103)
    with pytest.raises(KeyError):
        tl.lw_fourier_cfl(5)


def test_semidiscretization_requires_device_library_on_cpu(tl):
    """Without a GPU the product path must fail loudly (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    eq = tl.CompressibleEulerEquations2D()
    mesh = tl.TreeMesh((-1.0, -1.0), (1.0, 1.0), 1)
    with pytest.raises(Exception):
        tl.SemidiscretizationHyperbolic(mesh, tl.LW(), eq, tl.ConstantState(), tl.DGSEM(3))
