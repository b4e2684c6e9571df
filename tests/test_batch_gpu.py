"""Batched mocks (one paint / FFT / interlace / bin launch sequence for many catalogs,
captured in a CUDA graph) against the single-catalog path and the CPU oracle."""
import numpy as np
import pytest
import torch

from oracle.coords import Geometry
from oracle.spectrum import Bins, compute_mesh2_spectrum as ospectrum
from oracle import paint as opaint

pytestmark = pytest.mark.gpu


def _mocks(counts, boxsize, seed=0):
    rng = np.random.default_rng(seed)
    return [(rng.uniform(-0.5, 0.5, (c, 3)) * boxsize).astype('f4') for c in counts]


@pytest.mark.parametrize('tile_config', [0, 1, 2, 3, 4, 6, None])
def test_batched_matches_single(tile_config):
    import jaxpower_b200 as jp
    from jaxpower_b200.batch import BatchedSpectra
    counts = [3000, 50, 12000, 0, 7000]
    boxsize, meshsize = 500., 48
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.02}, ells=(0, 2, 4))
    mocks = _mocks(counts, boxsize)
    bs = BatchedSpectra(attrs, b, counts, resampler='tsc', interlacing=2, compensate=True, tile_config=tile_config)
    out = bs(torch.as_tensor(np.concatenate(mocks)).cuda()).cpu().numpy()
    out2 = bs().cpu().numpy()  # graph replay on the same inputs: bit-identical
    assert np.array_equal(out, out2)
    for m, pos in enumerate(mocks):
        if len(pos) == 0:
            assert np.all(out[m] == 0.)
            continue
        mesh = jp.ParticleField(pos, attrs=attrs).paint(resampler='tsc', interlacing=2, compensate=True, out='complex')
        ref = jp.compute_mesh2_spectrum(mesh, bin=b, los='z')
        for i, ell in enumerate(b.ells):
            scale = np.abs(ref.get(0).num_raw).max()
            assert np.allclose(out[m, i], ref.get(ell).num_raw, rtol=0, atol=1e-5 * scale), (m, ell)


def test_batched_vs_oracle_float64():
    import jaxpower_b200 as jp
    from jaxpower_b200.batch import BatchedSpectra
    counts = [20000, 8000]
    boxsize, meshsize = 400., 32
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.03}, ells=(0, 2, 4))
    mocks = _mocks(counts, boxsize, seed=3)
    out = BatchedSpectra(attrs, b, counts, resampler='tsc', interlacing=2)(
        torch.as_tensor(np.concatenate(mocks)).cuda()).cpu().numpy()
    geom = Geometry(meshsize, boxsize, 0., dtype=np.float64)
    ob = Bins(geom, step=0.03, ells=(0, 2, 4))
    for m, pos in enumerate(mocks):
        ref = ospectrum(opaint.paint(geom, pos.astype('f8'), None, 'tsc', 2, True, 'complex'), ob, los='z')['num_raw']
        scale = np.abs(ref[0]).max()
        assert np.allclose(out[m], ref, rtol=0, atol=1e-5 * scale)


def test_batched_long_rows_vs_oracle_float64():
    """A batch of meshes with long stored rows (97 modes: the staged row kernel of the fused
    interlaced binning, one grid row of CTAs per mesh) against the float64 oracle."""
    import jaxpower_b200 as jp
    from jaxpower_b200.batch import BatchedSpectra
    counts = [15000, 0, 6000]
    boxsize, meshsize = np.array([300., 300., 1200.]), np.array([24, 24, 192])
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.03}, ells=(0, 2, 4))
    rng = np.random.default_rng(5)
    mocks = [(rng.uniform(-0.5, 0.5, (c, 3)) * boxsize).astype('f4') for c in counts]
    out = BatchedSpectra(attrs, b, counts, resampler='tsc', interlacing=3)(
        torch.as_tensor(np.concatenate(mocks)).cuda()).cpu().numpy()
    geom = Geometry(meshsize, boxsize, 0., dtype=np.float64)
    ob = Bins(geom, step=0.03, ells=(0, 2, 4))
    for m, pos in enumerate(mocks):
        if len(pos) == 0:
            assert np.all(out[m] == 0.)
            continue
        ref = ospectrum(opaint.paint(geom, pos.astype('f8'), None, 'tsc', 3, True, 'complex'), ob, los='z')['num_raw']
        scale = np.abs(ref[0]).max()
        assert np.allclose(out[m], ref, rtol=0, atol=1e-5 * scale)


def test_batched_reports_dropped_particles():
    """A non-finite position in one mock raises, like ParticleField.paint; each replay reports its
    own inputs (the flag is cleared inside the graph), so a clean batch afterwards passes."""
    import jaxpower_b200 as jp
    from jaxpower_b200.batch import BatchedSpectra
    counts = [500, 700]
    boxsize = 300.
    attrs = jp.MeshAttrs(meshsize=24, boxsize=boxsize)
    b = jp.BinMesh2SpectrumPoles(attrs, edges={'step': 0.05}, ells=(0, 2))
    clean = torch.as_tensor(np.concatenate(_mocks(counts, boxsize, seed=4))).cuda()
    bad = clean.clone()
    bad[600, 1] = float('nan')
    bs = BatchedSpectra(attrs, b, counts, resampler='cic', interlacing=2)
    ref = bs(clean).cpu().numpy()
    with pytest.raises(ValueError):
        bs(bad)
    assert bs(bad, check=False) is not None and bs.status() != 0
    again = bs(clean).cpu().numpy()
    assert bs.status() == 0
    assert np.array_equal(ref, again)
