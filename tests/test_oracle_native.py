"""The oracle's C scatter (``oracle/paint_c.c``) against its NumPy statement (CPU).

Both restate ``resamplers.py:57-97``; the C loops must give the NumPy serial float32
mesh bit for bit (same operation order) and the float64-accumulated mesh to within
float64 rounding, for every resampler, with wrap-around, ties and negative cells.
"""
import numpy as np
import pytest

from oracle import _native
from oracle import paint as opaint


@pytest.mark.parametrize('order', [1, 2, 3, 4])
def test_native_scatter_matches_numpy(order):
    rng = np.random.default_rng(order)
    u = rng.uniform(-5., 21., (4000, 3)).astype('f4')
    u[:40] = (np.round(u[:40] * 2.) / 2.).astype('f4')  # half-integer ties and cell edges
    w = rng.uniform(-0.5, 1.5, 4000).astype('f4')
    shape = (16, 12, 10)
    serial = opaint.paint_mesh(shape, u, w, order, native=False)
    assert np.array_equal(_native.paint(shape, u, w, order, 'serial'), serial)
    f64 = opaint.paint_mesh(shape, u, w, order, accum='f64', native=False)
    got = _native.paint(shape, u, w, order, 'f64').astype('f4')
    assert np.all(np.abs(got.astype('f8') - f64) <= np.spacing(np.abs(f64)))
    assert np.array_equal(_native.paint(shape, u, None, order, 'serial'),
                          opaint.paint_mesh(shape, u, np.ones(4000, 'f4'), order, native=False))


@pytest.mark.parametrize('order', [1, 2, 3, 4])
def test_native_double_matches_numpy(order):
    rng = np.random.default_rng(10 + order)
    u = rng.uniform(-5., 21., (3000, 3))
    w = rng.uniform(-0.5, 1.5, 3000)
    shape = (12, 16, 10)
    ref = opaint.paint_mesh(shape, u, w, order, dtype=np.float64, native=False)
    got = _native.paint(shape, u, w, order, 'double')
    assert np.allclose(got, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
