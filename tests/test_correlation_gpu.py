"""Correlation-function multipoles (compute_mesh2_correlation, fixed line of sight) and the
separation-grid binning against the CPU oracle."""
import numpy as np
import pytest
import torch

from oracle.coords import Geometry
from oracle import paint as opaint
from oracle.spectrum import CorrelationBins, compute_mesh2_correlation as ocorr

pytestmark = pytest.mark.gpu


def _catalog(n, boxsize, seed):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-0.5, 0.5, (n, 3)) * np.asarray(boxsize)).astype('f4')


@pytest.mark.parametrize('meshsize', [(32, 32, 32), (17, 12, 10), (16, 20, 15)])
def test_separation_bins_match_oracle(meshsize):
    import jaxpower_b200 as jp
    boxsize = np.array([400., 300., 350.])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    b = jp.BinMesh2CorrelationPoles(attrs, edges={'step': 15.}, ells=(0, 2, 4))
    ob = CorrelationBins(Geometry(meshsize, boxsize, 0.), step=15., ells=(0, 2, 4))
    assert np.array_equal(b._edges1d, ob.edges)
    assert np.array_equal(b.nmodes, ob.nmodes)  # exact |s| bin assignment
    assert np.allclose(b.xavg, ob.xavg, rtol=1e-6, equal_nan=True)
    # plain per-bin mean of a real mesh, with and without the s = 0 cell
    value = np.random.default_rng(1).normal(size=meshsize).astype('f4')
    for rz in (False, True):
        assert np.allclose(b(torch.as_tensor(value), remove_zero=rz), ob(value, remove_zero=rz), rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize('los', ['z', 'x', [0.6, 0., 0.8]])
@pytest.mark.parametrize('cross', [False, True])
@pytest.mark.parametrize('meshsize', [(32, 24, 20), (16, 20, 15)])
def test_correlation_matches_oracle(los, cross, meshsize):
    import jaxpower_b200 as jp
    boxsize = np.array([500., 400., 300.])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    geom = Geometry(meshsize, boxsize, 0.)
    pos1, pos2 = _catalog(30000, boxsize, 3), _catalog(20000, boxsize, 4)
    m1 = jp.ParticleField(pos1, attrs=attrs).paint(resampler='tsc', interlacing=2, compensate=True, out='complex')
    o1 = opaint.paint(geom, pos1, None, 'tsc', 2, True, 'complex')
    b = jp.BinMesh2CorrelationPoles(attrs, edges={'step': 12.}, ells=(0, 2, 4))
    ob = CorrelationBins(geom, step=12., ells=(0, 2, 4))
    if cross:
        m2 = jp.ParticleField(pos2, attrs=attrs).paint(resampler='cic', out='real')
        o2 = opaint.paint(geom, pos2, None, 'cic', 0, False, 'real')
        got = jp.compute_mesh2_correlation(m1, m2, bin=b, los=los)
        ref = ocorr(o1, ob, los=los, mesh2=o2)
    else:
        got = jp.compute_mesh2(m1, bin=b, los=los)
        ref = ocorr(o1, ob, los=los)
    assert got.ells == (0, 2, 4)
    scale = np.abs(ref['num_raw'][0]).max()
    for i, ell in enumerate((0, 2, 4)):
        pole = got.get(ell)
        assert np.allclose(pole.s, ob.xavg, rtol=1e-6, equal_nan=True)
        assert np.allclose(pole.num_raw, ref['num_raw'][i], rtol=0, atol=1e-5 * scale), ell
    assert np.isfinite(got.get(0).value()).all()


@pytest.mark.parametrize('los,cross', [('firstpoint', False), ('firstpoint', True), ('endpoint', True)])
def test_firstpoint_correlation_matches_oracle(los, cross):
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_correlation_firstpoint as ofp
    meshsize, boxsize, boxcenter = (24, 28, 20), np.array([600., 700., 500.]), np.array([800., -200., 900.])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=boxcenter)
    geom = Geometry(meshsize, boxsize, boxcenter)
    pos1 = _catalog(20000, boxsize, 5) + boxcenter.astype('f4')
    pos2 = _catalog(15000, boxsize, 6) + boxcenter.astype('f4')
    m1 = jp.ParticleField(pos1, attrs=attrs).paint(resampler='cic', interlacing=2, compensate=True, out='real')
    o1 = opaint.paint(geom, pos1, None, 'cic', 2, True, 'real')
    b = jp.BinMesh2CorrelationPoles(attrs, edges={'step': 30.}, ells=(0, 2, 4))
    ob = CorrelationBins(geom, step=30., ells=(0, 2, 4))
    if cross:
        m2 = jp.ParticleField(pos2, attrs=attrs).paint(resampler='tsc', out='complex')
        o2 = opaint.paint(geom, pos2, None, 'tsc', 0, False, 'complex')
        got = jp.compute_mesh2_correlation(m1, m2, bin=b, los=los)
        ref = ofp(o1, ob, mesh2=o2, swap=los == 'endpoint')
    else:
        got = jp.compute_mesh2_correlation(m1, bin=b, los=los)
        ref = ofp(o1, ob)
    scale = np.abs(ref['num_raw'][0]).max()
    for i, ell in enumerate((0, 2, 4)):
        assert np.allclose(got.get(ell).num_raw, ref['num_raw'][i], rtol=0, atol=2e-5 * scale), ell


def test_correlation_ref_golden_gpu():
    """tests/test_mesh2.py:1042-1046: value().std() of the correlation multipoles of the test_ref FKP
    mesh (CIC, interlacing 3, compensate, 128^3, jaxdecomp layout), s step 4 cells, ells (0, 2, 4),
    for los 'x', 'firstpoint' and 'endpoint'.  The goldens are x64; the GPU path is float32."""
    import json
    import os
    import jaxpower_b200 as jp
    from tests.golden.catalogs import uniform_particles
    golden = json.load(open(os.path.join(os.path.dirname(__file__), 'golden', 'reference_goldens.json')))
    g, gc = golden['spectrum_ref'], golden['correlation_ref']
    attrs = jp.MeshAttrs(meshsize=g['meshsize'], boxsize=g['boxsize'], boxcenter=g['boxcenter'], fft_backend='jaxdecomp')
    data = jp.ParticleField(uniform_particles(g['data_seed'], g['size'], g['boxsize'], g['boxcenter']).astype('f4'),
                            attrs=attrs)
    randoms = jp.ParticleField(uniform_particles(g['randoms_seed'], g['randoms_size'], g['boxsize'],
                                                 g['boxcenter']).astype('f4'), attrs=attrs)
    mesh = jp.FKPField(data, randoms).paint(resampler=g['resampler'], interlacing=g['interlacing'],
                                            compensate=g['compensate'])
    b = jp.BinMesh2CorrelationPoles(attrs, edges={'step': gc['edges_step_in_cellsize'] * float(attrs.cellsize.min())},
                                    ells=tuple(gc['ells']))
    for los, expected in gc['value_std'].items():
        value = jp.compute_mesh2_correlation(mesh, bin=b, los=los).value()
        assert np.isclose(value.std(), expected, rtol=3e-5, atol=0.), (los, value.std(), expected)


@pytest.mark.parametrize('los,cross,klimit', [
    ('z', False, None), ('x', True, None), ([0.6, 0., 0.8], False, (0.02, 0.2)),
    ('firstpoint', False, None), ('firstpoint', True, True), ('endpoint', True, None)])
def test_bessel_basis_matches_oracle(los, cross, klimit):
    """basis='bessel' (mesh2.py:169-177): Fourier-space mode values projected on j_ell(|k| s)."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_correlation_bessel as obessel
    local = los in ('firstpoint', 'endpoint')
    meshsize, boxsize = (24, 20, 16), np.array([480., 400., 320.])
    boxcenter = np.array([700., -100., 600.]) if local else np.zeros(3)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=boxcenter)
    geom = Geometry(meshsize, boxsize, boxcenter)
    pos1 = _catalog(20000, boxsize, 7) + boxcenter.astype('f4')
    pos2 = _catalog(15000, boxsize, 8) + boxcenter.astype('f4')
    m1 = jp.ParticleField(pos1, attrs=attrs).paint(resampler='tsc', interlacing=2, compensate=True, out='real')
    o1 = opaint.paint(geom, pos1, None, 'tsc', 2, True, 'real')
    ells = (0, 1, 2, 3, 4) if local else (0, 2, 4)
    b = jp.BinMesh2CorrelationPoles(attrs, edges={'step': 20.}, ells=ells, basis='bessel', klimit=klimit)
    ob = CorrelationBins(geom, step=20., ells=ells)
    ok = None if klimit is None else b.klimit
    if cross:
        m2 = jp.ParticleField(pos2, attrs=attrs).paint(resampler='cic', out='complex')
        o2 = opaint.paint(geom, pos2, None, 'cic', 0, False, 'complex')
        got = jp.compute_mesh2_correlation(m1, m2, bin=b, los=los)
        ref = obessel(o1, ob, los=los, mesh2=o2, klimit=ok)
    else:
        got = jp.compute_mesh2_correlation(m1, bin=b, los=los)
        ref = obessel(o1, ob, los=los, klimit=ok)
    # float32 mode values and |k| s, float64 j_ell and sums on both sides: the sums agree to
    # float32 rounding of the per-mode products
    scale = np.abs(ref['num_raw'][0]).max()
    assert scale > 0.
    for i, ell in enumerate(ells):
        assert np.allclose(got.get(ell).num_raw, ref['num_raw'][i], rtol=0, atol=2e-5 * scale), ell
    # the plain separation binning of the same estimator differs (another basis)
    assert got.get(0).s.shape == ob.xavg.shape


@pytest.mark.parametrize('los', ['z', 'firstpoint'])
def test_correlation_mode_oversampling_matches_oracle(los):
    """BinMesh2CorrelationPoles(mode_oversampling=1): separations binned by |s + shift| for the
    27 integer shifts and averaged (mesh2.py:48-61, as for k); nmodes, xavg and the multipoles
    against the oracle."""
    import jaxpower_b200 as jp
    from oracle.spectrum import compute_mesh2_correlation_firstpoint as ofp
    meshsize, boxsize = (20, 16, 12), np.array([400., 320., 240.])
    center = np.array([600., -100., 500.]) if los == 'firstpoint' else np.zeros(3)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=center)
    geom = Geometry(meshsize, boxsize, center)
    pos = _catalog(20000, boxsize, 9) + center.astype('f4')
    m = jp.ParticleField(pos, attrs=attrs).paint(resampler='tsc', interlacing=2, compensate=True, out='real')
    o = opaint.paint(geom, pos, None, 'tsc', 2, True, 'real')
    b = jp.BinMesh2CorrelationPoles(attrs, edges={'step': 25.}, ells=(0, 2), mode_oversampling=1)
    ob = CorrelationBins(geom, step=25., ells=(0, 2), mode_oversampling=1)
    assert np.array_equal(b.nmodes, ob.nmodes)
    assert np.allclose(b.xavg, ob.xavg, rtol=1e-6, equal_nan=True)
    got = jp.compute_mesh2_correlation(m, bin=b, los=los)
    ref = ofp(o, ob) if los == 'firstpoint' else ocorr(o, ob, los=los)
    scale = np.abs(ref['num_raw'][0]).max()
    for i, ell in enumerate((0, 2)):
        assert np.allclose(got.get(ell).num_raw, ref['num_raw'][i], rtol=0, atol=1e-5 * scale), ell
