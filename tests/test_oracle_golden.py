"""Pin the CPU oracle to the reference's own golden values and known answers.

- Threefry-2x32 known-answer vectors (Random123 / JAX ``random_test``);
- ``tests/test_mesh.py:211`` golden ``mesh.std()`` of a TSC / interlacing 3 /
  compensated paint of 1e6 ``jax.random`` positions;
- ``tests/test_mesh2.py:1032-1040`` golden ``value().std()`` of the FKP spectrum
  (CIC, interlacing 3, compensate, 128^3) for los 'x', 'firstpoint', 'endpoint';
- ``tests/test_mesh2.py:1042-1046`` golden ``value().std()`` of the correlation
  multipoles of the same FKP mesh;
- ``tests/test_mesh.py:278-281`` goldens of ``compute_fkp2_normalization`` (cellsize None,
  cellsize 10, and ``split=(42, index)``: disjoint random halves of the randoms).

The goldens were produced with x64 on and the jaxdecomp (full complex) FFT
layout; the oracle reproduces them to ~1e-14 in that mode.
"""
import json
import os

import numpy as np
import pytest

from oracle.threefry import threefry2x32
from oracle.coords import Geometry
from oracle.paint import paint
from oracle.spectrum import Bins, compute_mesh2_spectrum, fkp_particles
from tests.golden.catalogs import paint_jit_positions, uniform_particles

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'reference_goldens.json')))


@pytest.mark.parametrize('key,count,expected', [
    ((0, 0), (0, 0), (0x6b200159, 0x99ba4efe)),
    ((0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff), (0x1cb996fc, 0xbb002be7)),
    ((0x13198a2e, 0x03707344), (0x243f6a88, 0x85a308d3), (0xc4923a9c, 0x483df7a0)),
])
def test_threefry_known_answers(key, count, expected):
    y0, y1 = threefry2x32(key, [count[0]], [count[1]])
    assert (int(y0[0]), int(y1[0])) == expected


@pytest.mark.slow
def test_paint_jit_golden():
    g = GOLDEN['paint_jit']
    pos = paint_jit_positions(g['seed'], g['nparticles'])
    geom = Geometry(g['meshsize'], g['boxsize'], g['boxcenter'], dtype=np.float64, backend='jaxdecomp')
    mesh = paint(geom, pos, None, g['resampler'], g['interlacing'], g['compensate'], 'real')
    assert np.allclose(mesh.std(), g['std'], rtol=1e-12, atol=0.)


@pytest.mark.slow
def test_spectrum_ref_golden():
    g = GOLDEN['spectrum_ref']
    geom = Geometry(g['meshsize'], g['boxsize'], g['boxcenter'], dtype=np.float64, backend='jaxdecomp')
    data = uniform_particles(g['data_seed'], g['size'], g['boxsize'], g['boxcenter'])
    randoms = uniform_particles(g['randoms_seed'], g['randoms_size'], g['boxsize'], g['boxcenter'])
    pos, w, alpha = fkp_particles(data, None, randoms, None, dtype=np.float64)
    assert alpha == 0.5
    mesh = paint(geom, pos, w, g['resampler'], g['interlacing'], g['compensate'], 'real')
    bins = Bins(geom, step=g['edges_step_in_kfun'] * geom.kfun.min(), ells=tuple(g['ells']))
    for los, expected in g['value_std'].items():
        r = compute_mesh2_spectrum(mesh, bins, los)
        value = r['num_raw'] / r['norm']
        assert np.allclose(value.std(), expected, rtol=1e-12, atol=0.), los


def test_fkp2_normalization_goldens():
    """tests/test_mesh.py:278-281: compute_fkp2_normalization with cellsize None, cellsize 10, and
    split=(42, index) (disjoint random halves of the randoms drawn per particle id)."""
    from oracle.spectrum import fkp2_normalization
    g = GOLDEN['fkp2_normalization']
    data = uniform_particles(g['data_seed'], g['size'], g['boxsize'], g['boxcenter'])
    randoms = uniform_particles(g['randoms_seed'], g['size'], g['boxsize'], g['boxcenter'])
    geom = Geometry(g['meshsize'], g['boxsize'], g['boxcenter'], dtype=np.float64)
    cases = {'cellsize_none': dict(cellsize=None), 'cellsize_10': dict(cellsize=10.),
             'cellsize_10_split': dict(cellsize=10., split=(g['split_seed'], np.arange(g['size'])))}
    for name, kw in cases.items():
        assert np.allclose(fkp2_normalization(geom, data, None, randoms, None, **kw), g['norm'][name],
                           rtol=1e-12, atol=0.), name


@pytest.mark.slow
def test_correlation_ref_golden():
    """tests/test_mesh2.py:1042-1046: value().std() of the correlation multipoles of the test_ref
    FKP mesh, s step 4 cells, for los 'x', 'firstpoint' and 'endpoint'."""
    from oracle.spectrum import CorrelationBins, compute_mesh2_correlation, compute_mesh2_correlation_firstpoint
    g = GOLDEN['spectrum_ref']
    gc = GOLDEN['correlation_ref']
    geom = Geometry(g['meshsize'], g['boxsize'], g['boxcenter'], dtype=np.float64, backend='jaxdecomp')
    data = uniform_particles(g['data_seed'], g['size'], g['boxsize'], g['boxcenter'])
    randoms = uniform_particles(g['randoms_seed'], g['randoms_size'], g['boxsize'], g['boxcenter'])
    pos, w, _ = fkp_particles(data, None, randoms, None, dtype=np.float64)
    mesh = paint(geom, pos, w, g['resampler'], g['interlacing'], g['compensate'], 'real')
    bins = CorrelationBins(geom, step=gc['edges_step_in_cellsize'] * geom.cellsize.min(), ells=tuple(gc['ells']))
    norm = np.prod(geom.meshsize.astype('f8')) / np.prod(geom.cellsize.astype('f8'))
    for los, expected in gc['value_std'].items():
        if los == 'x':
            r = compute_mesh2_correlation(mesh, bins, los=los)
        else:
            r = compute_mesh2_correlation_firstpoint(mesh, bins, swap=los == 'endpoint')
        assert np.allclose((r['num_raw'] / norm).std(), expected, rtol=1e-12, atol=0.), los
