"""Hand-written adjoints of paint and of the binned estimators vs finite differences.

Loss = sum_{ell, b} c[ell, b] num_raw[ell, b] for fixed random coefficients c.  The GPU
gradient (autograd through the library's adjoint kernels) is compared with central
finite differences of the float64 CPU oracle (the reference's algorithm restated), on
small meshes where the oracle is fast.  The reference itself checks nothing here (its
gradients come from JAX autodiff, unavailable on these machines).
"""
import numpy as np
import pytest
import torch

from oracle.coords import Geometry
from oracle import paint as opaint
from oracle.spectrum import Bins, compute_mesh2_spectrum as ospectrum

pytestmark = pytest.mark.gpu


def _setup(seed=0, n=400, meshsize=16, boxsize=200., boxcenter=0.):
    rng = np.random.default_rng(seed)
    pos = (rng.uniform(-0.45, 0.45, (n, 3)) * boxsize + boxcenter).astype('f4')
    w = rng.uniform(0.5, 1.5, n).astype('f4')
    return pos, w


def _oracle_loss(pos, w, meshsize, boxsize, boxcenter, resampler, interlacing, compensate, out, step, ells, los, coef,
                 backend='jax', oversampling=0):
    geom = Geometry(meshsize, boxsize, boxcenter, dtype=np.float64, backend=backend)
    mesh = opaint.paint(geom, pos.astype('f8'), w.astype('f8'), resampler, interlacing, compensate, out)
    r = ospectrum(mesh, Bins(geom, step=step, ells=ells, mode_oversampling=oversampling), los=los)
    return float(np.sum(coef * r['num_raw']))


@pytest.mark.parametrize('resampler,interlacing,compensate,out,los,ells,backend,oversampling', [
    ('tsc', 3, True, 'real', 'z', (0, 2, 4), 'jax', 0),
    ('tsc', 2, False, 'complex', 'x', (0, 2, 4), 'jax', 0),
    ('pcs', 1, True, 'real', 'z', (0, 2, 4), 'jax', 0),
    ('cic', 0, False, 'real', 'z', (0, 2, 4), 'jax', 0),
    ('tsc', 3, True, 'real', 'firstpoint', (0, 2, 4), 'jax', 0),
    # odd multipoles: zero for a global line of sight (auto spectrum), imaginary parts for a
    # local one, with the sign of the end-point conjugation
    ('cic', 2, True, 'real', 'z', (0, 1, 2, 3), 'jax', 0),
    ('tsc', 2, True, 'real', 'firstpoint', (0, 1, 2, 3), 'jax', 0),
    ('tsc', 2, False, 'real', 'endpoint', (1, 3), 'jax', 0),
    # a complex input mesh to the first-point estimator: A0 itself and irfftn of it
    ('tsc', 2, True, 'complex', 'firstpoint', (0, 2, 4), 'jax', 0),
    ('cic', 3, False, 'complex', 'endpoint', (0, 1, 2), 'jax', 0),
    # the 'jaxdecomp' FFT semantics: full-grid interlacing phases on the Nyquist planes
    ('tsc', 3, True, 'real', 'z', (0, 2, 4), 'jaxdecomp', 0),
    ('cic', 2, True, 'real', 'firstpoint', (0, 1, 2), 'jaxdecomp', 0),
    # mode oversampling: each mode's coefficient averaged over the shifted binnings
    ('tsc', 2, True, 'real', 'z', (0, 2, 4), 'jax', 1),
    ('cic', 2, False, 'real', 'firstpoint', (0, 2), 'jax', 1),
])
def test_position_gradient_vs_finite_differences(resampler, interlacing, compensate, out, los, ells, backend,
                                                oversampling):
    import jaxpower_b200 as jp
    from jaxpower_b200.autodiff import paint_value, spectrum_value
    local = los in ('firstpoint', 'endpoint')
    meshsize, boxsize, boxcenter, step = 16, 200., (300. if local else 0.), 0.05
    pos, w = _setup(meshsize=meshsize, boxsize=boxsize, boxcenter=boxcenter)
    attrs = jp.MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=boxcenter, fft_backend=backend)
    bins = jp.BinMesh2SpectrumPoles(attrs, edges={'step': step}, ells=ells, mode_oversampling=oversampling)
    rng = np.random.default_rng(1)
    coef = rng.normal(size=(len(ells), bins.nbins))
    tpos = torch.as_tensor(pos, device='cuda').requires_grad_(True)
    tw = torch.as_tensor(w, device='cuda').requires_grad_(True)
    mesh = paint_value(tpos, tw, attrs, resampler=resampler, interlacing=interlacing, compensate=compensate, out=out)
    num = spectrum_value(mesh, attrs, bins, los)
    loss = (num * torch.as_tensor(coef, device='cuda')).sum()
    loss.backward()
    gpos = tpos.grad.cpu().numpy().astype('f8')
    gw = tw.grad.cpu().numpy().astype('f8')
    # forward parity first
    ref = _oracle_loss(pos, w, meshsize, boxsize, boxcenter, resampler, interlacing, compensate, out, step, ells, los, coef, backend, oversampling)
    assert np.isclose(float(loss), ref, rtol=1e-4)
    h = 1e-3 * boxsize / meshsize
    scale = np.abs(gpos).max()
    assert scale > 0.
    for p in (0, 7, 123, 311):
        for d in range(3):
            pp, pm = pos.astype('f8').copy(), pos.astype('f8').copy()
            pp[p, d] += h
            pm[p, d] -= h
            fd = (_oracle_loss(pp, w, meshsize, boxsize, boxcenter, resampler, interlacing, compensate, out, step, ells, los, coef, backend, oversampling)
                  - _oracle_loss(pm, w, meshsize, boxsize, boxcenter, resampler, interlacing, compensate, out, step, ells, los, coef, backend, oversampling)) / (2 * h)
            assert abs(gpos[p, d] - fd) <= 2e-3 * scale + 2e-3 * abs(fd), (p, d, gpos[p, d], fd)
    # weights: the loss is quadratic in w, check two weights
    for p in (3, 200):
        wp, wm = w.astype('f8').copy(), w.astype('f8').copy()
        hw = 1e-3
        wp[p] += hw
        wm[p] -= hw
        fd = (_oracle_loss(pos, wp, meshsize, boxsize, boxcenter, resampler, interlacing, compensate, out, step, ells, los, coef, backend, oversampling)
              - _oracle_loss(pos, wm, meshsize, boxsize, boxcenter, resampler, interlacing, compensate, out, step, ells, los, coef, backend, oversampling)) / (2 * hw)
        assert abs(gw[p] - fd) <= 2e-3 * np.abs(gw).max() + 2e-3 * abs(fd), (p, gw[p], fd)
