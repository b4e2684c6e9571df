"""The oracle's binnings with mode oversampling (``_make_edges2``, ``mesh2.py:25-62``), on the
CPU: one binning per integer shift of the separation (or wave) vectors, nmodes the mean
count over the shifts, xavg the summed |x + shift| over that mean, and the binned values
averaged over the shifts' bin indices (``mesh2.py:94-98``, ``mesh.py:2894-2895``)."""
from itertools import product

import numpy as np
import pytest

from oracle.coords import Geometry
from oracle.spectrum import Bins, CorrelationBins, hermitian_weights, kcoords, separation_coords


@pytest.mark.parametrize('meshsize, boxsize', [(16, 64.), ((12, 16, 10), (30., 40., 25.))])
def test_mode_oversampling_counts_and_means(meshsize, boxsize):
    geom = Geometry(meshsize, boxsize)
    plain = CorrelationBins(geom, step=4.)
    over = CorrelationBins(geom, step=4., mode_oversampling=1)
    assert len(plain.ibins) == 1 and len(over.ibins) == 27
    # the unshifted binning is the plain one; it sits in the middle of the shift product
    center = list(product(range(-1, 2), repeat=3)).index((0, 0, 0))
    assert np.array_equal(over.ibins[center], plain.ibins[0])
    assert np.array_equal(over.ibin, over.ibins[0].reshape(over.snorm.shape))
    # nmodes: the mean over the shifts of each shift's count; xavg: the summed |s + shift| over it
    sx, sy, sz = separation_coords(geom)
    nb = len(over.edges) + 1
    counts, sums = np.zeros(over.nbins), np.zeros(over.nbins)
    for shift in product(range(-1, 2), repeat=3):
        a, b, c = [(x + np.float32(v)).astype('f4') for x, v in zip((sx, sy, sz), shift)]
        norm = np.broadcast_to(np.sqrt(((a * a + b * b).astype('f4') + c * c).astype('f4')), over.snorm.shape)
        ib = np.searchsorted(over.edges.astype('f4'), norm.ravel(), side='right')
        counts += np.bincount(ib, minlength=nb)[1:-1]
        sums += np.bincount(ib, weights=norm.ravel().astype('f8'), minlength=nb)[1:-1]
    assert np.allclose(over.nmodes, counts / 27., rtol=0., atol=1e-12)
    ok = over.nmodes > 0
    assert np.allclose(over.xavg[ok], sums[ok] / over.nmodes[ok], rtol=1e-12)
    # binning a constant returns it wherever a bin has modes, with and without oversampling
    ones = np.ones(tuple(geom.meshsize))
    for bins in (plain, over):
        got = bins(ones)
        assert np.allclose(got[bins.nmodes > 0], 1., rtol=1e-12)
    # every shifted |s| keeps its own bin assignment: a value equal to the bin index of the
    # plain binning averages over the shifts, not over one fixed binning
    field = plain.ibins[0].reshape(plain.snorm.shape).astype('f8')
    assert not np.allclose(over(field)[ok], plain(field)[ok]) or over.nbins < 2


def test_spectrum_mode_oversampling_counts_and_means():
    """The k-space binning: shifts of the wave vectors by integers (in h/Mpc, as the reference
    adds them), Hermitian weights in every count and sum."""
    geom = Geometry(16, 8.)  # k_f = 0.785: unit shifts move |k| by about one fundamental
    plain = Bins(geom, step=0.5)
    over = Bins(geom, step=0.5, mode_oversampling=1)
    assert len(over.ibins) == 27
    center = list(product(range(-1, 2), repeat=3)).index((0, 0, 0))
    assert np.array_equal(over.ibins[center], plain.ibin)
    w = hermitian_weights(geom).ravel()
    kx, ky, kz = kcoords(geom)
    nb = len(over.edges) + 1
    counts, sums = np.zeros(over.nbins), np.zeros(over.nbins)
    for shift in product(range(-1, 2), repeat=3):
        a, b, c = [(x + np.float32(v)).astype('f4') for x, v in zip((kx, ky, kz), shift)]
        norm = np.sqrt(((a * a + b * b).astype('f4') + c * c).astype('f4')).ravel()
        ib = np.searchsorted(over.edges.astype('f4'), norm, side='right')
        counts += np.bincount(ib, weights=w, minlength=nb)[1:-1]
        sums += np.bincount(ib, weights=norm.astype('f8') * w, minlength=nb)[1:-1]
    assert np.allclose(over.nmodes, counts / 27., rtol=1e-12, atol=0.)
    ok = over.nmodes > 0
    assert np.allclose(over.xavg[ok], sums[ok] / over.nmodes[ok], rtol=1e-12)
    ones = np.ones(over.wmodes.shape)
    for bins in (plain, over):
        assert np.allclose(bins(ones)[bins.nmodes > 0], 1., rtol=1e-12)
    with pytest.raises(NotImplementedError):
        over(ones, accum='f32')
