"""The reciprocal every Euler flux evaluation takes of the density (the hardware approximation refined by
one third-order step, in place of a correctly rounded divide): at most one unit in the last place from IEEE
1/x, over the density range of the workloads (the Riemann states' 0.13 .. 1.5, the vortex core's ~0.1 .. 1)
and far beyond it, and exact on powers of two."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ulp_distance(a, b):
    """|a - b| in units in the last place, for positive finite doubles."""
    return np.abs(a.view(np.int64) - b.view(np.int64))


def test_reciprocal_within_one_ulp_of_ieee_division(tl):
    from trixilw import _lib
    rng = np.random.default_rng(0)
    x = np.concatenate([
        np.linspace(0.13, 1.5, 200_001),                       # the four-quadrant Riemann densities
        np.geomspace(1e-6, 1e6, 200_001),
        rng.uniform(1.0, 2.0, 200_000) * 2.0 ** rng.integers(-60, 60, 200_000),   # random mantissas
        2.0 ** np.arange(-100, 101, dtype=np.float64),
        np.nextafter(1.0, 2.0) + np.arange(1000) * np.finfo(float).eps,
        np.nextafter(2.0, 1.0) - np.arange(1000) * np.finfo(float).eps,
    ])
    x = np.ascontiguousarray(x)
    y = np.empty_like(x)
    rc = _lib.lib().tlw_probe_reciprocal(0, x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p),
                                         x.size)
    assert rc == _lib.TLW_OK
    ref = 1.0 / x
    d = ulp_distance(y, ref)
    assert d.max() <= 1, (d.max(), x[np.argmax(d)])
    assert np.mean(d == 0) > 0.99                      # nearly always the correctly rounded value
    p2 = 2.0 ** np.arange(-100, 101, dtype=np.float64)
    np.testing.assert_array_equal(y[-2000 - p2.size:-2000], 1.0 / p2)
