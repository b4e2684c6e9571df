"""Learned aliasing correction: the BF16 MLP kernels (forward, backward, AdamW) against
the CPU oracle, training on the GPU, and the gain of the trained correction over the
plain coarse-mesh estimator on held-out lognormal mocks."""
import numpy as np
import pytest
import torch

from oracle import mlp as omlp

pytestmark = pytest.mark.gpu


def _flat(seed, scale=1.):
    rng = np.random.default_rng(seed)
    p = {}
    for name, shape in omlp.LAYOUT:
        p[name] = (rng.normal(size=shape) * scale / np.sqrt(shape[-1]) if name.startswith('W')
                   else 0.1 * rng.normal(size=shape))
    return omlp.flatten(p).astype('f4')


def _mlp(flat):
    from jaxpower_b200.learned import MLP
    return MLP(w=torch.as_tensor(flat))


@pytest.mark.parametrize('batch', [1, 37, 200, 1000])
def test_forward_matches_oracle(batch):
    flat = _flat(0)
    x = np.random.default_rng(1).normal(size=(batch, omlp.IN)).astype('f4')
    got = _mlp(flat)(torch.as_tensor(x)).cpu().numpy()
    ref, _ = omlp.forward(flat.astype('f8'), x)
    scale = max(np.abs(ref).max(), 1e-3)
    err = np.abs(got - ref) / scale
    # bf16 activations may round differently when an f32 pre-activation sits on a rounding
    # boundary; everything else differs by float32 summation order only
    assert np.median(err) < 2e-6
    assert err.max() < 2e-3


@pytest.mark.parametrize('batch', [1, 127, 128, 129, 3000])
def test_tcgen05_forward_matches_mma_forward(batch):
    """The tcgen05 forward pass (accumulators in tensor memory) against the mma.sync one and
    the oracle, outputs and stored pre-activations / activations."""
    from jaxpower_b200 import _lib
    flat = _flat(7)
    mlp = _mlp(flat)
    x = torch.as_tensor(np.random.default_rng(8).normal(size=(batch, omlp.IN)).astype('f4')).cuda()
    outs = []
    for name in ('pk_mlp_forward', 'pk_mlp_forward_tc'):
        y = torch.empty(batch, device='cuda')
        z = torch.empty((3, batch, omlp.H), device='cuda')
        h = torch.empty_like(z)
        extra = (_lib.ptr(mlp.status),) if name.endswith('_tc') else ()
        _lib.call(name, _lib.stream_handle(), _lib.ptr(x), None, batch, _lib.ptr(mlp.wb), _lib.ptr(mlp.w),
                  _lib.ptr(y), _lib.ptr(z), _lib.ptr(h), *extra)
        outs.append((y.cpu().numpy(), z.cpu().numpy(), h.cpu().numpy()))
    mlp.check()
    (y0, z0, h0), (y1, z1, h1) = outs
    scale = max(np.abs(y0).max(), 1e-3)
    assert np.abs(y1 - y0).max() <= 1e-5 * scale
    assert np.allclose(z1, z0, rtol=0, atol=1e-5 * np.abs(z0).max())
    assert np.allclose(h1, h0, rtol=0, atol=1e-5 * np.abs(h0).max())
    ref, _ = omlp.forward(flat.astype('f8'), x.cpu().numpy())
    assert np.median(np.abs(y1 - ref)) < 2e-6 * max(np.abs(ref).max(), 1e-3)


def test_gradient_matches_oracle():
    flat = _flat(2)
    rng = np.random.default_rng(3)
    x = rng.normal(size=(300, omlp.IN)).astype('f4')
    dy = rng.normal(size=300).astype('f4')
    got = _mlp(flat).gradient(torch.as_tensor(x), torch.as_tensor(dy)).cpu().numpy()
    _, cache = omlp.forward(flat.astype('f8'), x)
    ref = omlp.backward(flat.astype('f8'), cache, dy.astype('f8'))
    off = 0
    for name, shape in omlp.LAYOUT:
        n = int(np.prod(shape))
        g, r = got[off:off + n], ref[off:off + n]
        off += n
        if not np.any(r):
            assert np.all(g == 0.), name
            continue
        assert np.linalg.norm(g - r) <= 2e-3 * np.linalg.norm(r), name
        assert np.allclose(g, r, rtol=0, atol=5e-3 * np.abs(r).max()), name


@pytest.mark.parametrize('batch', [1, 127, 128, 129, 3000, 40000])
def test_tcgen05_backward_matches_mma_backward(batch):
    """The tcgen05 backward (weight gradients accumulated in tensor memory over a persistent
    CTA's tiles; 40000 samples give several tiles per CTA) against the mma.sync backward and
    the oracle, through a sample gather."""
    from jaxpower_b200 import _lib
    flat = _flat(9)
    mlp = _mlp(flat)
    rng = np.random.default_rng(10)
    n = batch + 17
    x = torch.as_tensor(rng.normal(size=(n, omlp.IN)).astype('f4')).cuda()
    idx = torch.as_tensor(rng.permutation(n)[:batch].astype('i4')).cuda()
    dy = torch.as_tensor(rng.normal(size=batch).astype('f4')).cuda()
    y = torch.empty(batch, device='cuda')
    z = torch.empty((3, batch, omlp.H), device='cuda')
    h = torch.empty_like(z)
    _lib.call('pk_mlp_forward_tc', _lib.stream_handle(), _lib.ptr(x), _lib.ptr(idx), batch, _lib.ptr(mlp.wb),
              _lib.ptr(mlp.w), _lib.ptr(y), _lib.ptr(z), _lib.ptr(h), _lib.ptr(mlp.status))
    nbytes = _lib.c_size_t()
    _lib.call('pk_mlp_backward_workspace_size', batch, _lib.ctypes.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device='cuda')
    grads = []
    for name in ('pk_mlp_backward', 'pk_mlp_backward_tc'):
        grad = torch.full((mlp.nparams,), float('nan'), device='cuda')
        extra = (_lib.ptr(mlp.status),) if name.endswith('_tc') else ()
        _lib.call(name, _lib.stream_handle(), _lib.ptr(x), _lib.ptr(idx), batch, _lib.ptr(mlp.wb), _lib.ptr(z),
                  _lib.ptr(h), _lib.ptr(dy), _lib.ptr(grad), _lib.ptr(ws), ws.numel(), *extra)
        grads.append(grad.cpu().numpy())
    mlp.check()
    g0, g1 = grads
    assert np.all(np.isfinite(g1))
    xs = x.cpu().numpy()[idx.cpu().numpy()]
    _, cache = omlp.forward(flat.astype('f8'), xs)
    ref = omlp.backward(flat.astype('f8'), cache, dy.cpu().numpy().astype('f8'))
    off = 0
    for name, shape in omlp.LAYOUT:
        size = int(np.prod(shape))
        a, b, r = g0[off:off + size], g1[off:off + size], ref[off:off + size]
        off += size
        if not np.any(r):
            assert np.all(b == 0.), name
            continue
        # both kernels round the same operands to bf16 and sum in float32 in different orders
        # (a dZ on a bf16 rounding boundary can round either way)
        assert np.linalg.norm(b - a) <= 2e-4 * np.linalg.norm(a), name
        assert np.linalg.norm(b - r) <= 2e-3 * np.linalg.norm(r), name


def test_tcgen05_backward_is_deterministic():
    from jaxpower_b200 import _lib
    flat = _flat(11)
    mlp = _mlp(flat)
    x = torch.randn(70000, omlp.IN, generator=torch.Generator().manual_seed(0)).cuda()
    dy = torch.randn(70000, generator=torch.Generator().manual_seed(1)).cuda()
    _, cache = mlp.forward(x, cache=True)
    assert torch.equal(mlp.gradient(x, dy, cache), mlp.gradient(x, dy, cache))
    mlp.check()


def test_gradient_is_deterministic():
    flat = _flat(4)
    x = torch.randn(5000, omlp.IN, generator=torch.Generator().manual_seed(0))
    dy = torch.randn(5000, generator=torch.Generator().manual_seed(1))
    mlp = _mlp(flat)
    assert torch.equal(mlp.gradient(x, dy), mlp.gradient(x, dy))


def test_adam_matches_oracle():
    from jaxpower_b200 import _lib
    flat = _flat(5)
    mlp = _mlp(flat)
    rng = np.random.default_rng(6)
    w, m, v = flat.astype('f8'), np.zeros(len(flat)), np.zeros(len(flat))
    lr_table = torch.tensor([1e-2, 5e-3, 2e-3], dtype=torch.float32, device='cuda')
    for step in range(1, 4):
        g = rng.normal(size=len(flat)).astype('f4')
        gd = torch.as_tensor(g).cuda()
        _lib.call('pk_mlp_adam', _lib.stream_handle(), _lib.ptr(mlp.w), _lib.ptr(mlp.wb), _lib.ptr(mlp.m),
                  _lib.ptr(mlp.v), _lib.ptr(gd), _lib.ptr(lr_table), 3, _lib.ptr(mlp.step), 0.9, 0.999, 1e-8, 1e-4)
        w, m, v = omlp.adam(w, m, v, g.astype('f8'), float(lr_table[step - 1]), step, weight_decay=1e-4)
    assert int(mlp.step.item()) == 3
    assert np.allclose(mlp.w.cpu().numpy(), w, rtol=1e-6, atol=1e-6)
    assert np.array_equal(mlp.wb.float().cpu().numpy(), omlp.bf16(mlp.w.cpu().numpy()).astype('f4'))


def test_training_fits_and_is_reproducible():
    from jaxpower_b200.learned import MLP
    g = torch.Generator().manual_seed(0)
    x = torch.rand(16384, 4, generator=g) * 2 - 1
    t = torch.sin(3 * x[:, 0]) + x[:, 1]**2 - 0.5 * x[:, 2] * x[:, 3]
    runs = []
    for _ in range(2):
        mlp = MLP(seed=1)
        hist = mlp.fit(x, t, steps=600, batch=2048, lr=3e-3, seed=2)
        runs.append(mlp.state())
    assert hist[-1] < 0.02 * float(t.var())
    pred = mlp(x).cpu()
    assert float(((pred - t)**2).mean()) < 0.02 * float(t.var())
    assert np.array_equal(runs[0], runs[1])  # deterministic kernels, graph replays


def _small_data():
    from jaxpower_b200.learned import mock_spectra
    return mock_spectra(range(448), meshsizes=(32, 128), boxsize=500., nbar=5e-4, gen_meshsize=64,
                        kstep=0.02, group=32)


def test_learned_correction_beats_plain():
    from jaxpower_b200.learned import LearnedCorrection, spectrum_errors, ensemble_bias
    data = _small_data()
    nheld = 64
    train = dict(data, nparticles=data['nparticles'][:-nheld],
                 spectra={n: v[:-nheld] for n, v in data['spectra'].items()})
    corr, report = LearnedCorrection.train(train, 32, 128, steps=1500, batch=2048, lr=2e-3)
    assert report['corrected_bins'] > 0
    low, high = data['spectra'][32][-nheld:], data['spectra'][128][-nheld:]
    fixed = corr(low, data['nparticles'][-nheld:])
    kmax = 0.8 * np.pi * 32 / 500.
    # the learned correction removes most of the coarse mesh's aliasing bias ...
    b_plain, b_corr = ensemble_bias(low, high, data['k'], kmax), ensemble_bias(fixed, high, data['k'], kmax)
    assert b_corr.max() < 0.3 * b_plain.max(), (b_corr.max(), b_plain.max())
    # ... and lowers the per-mock error
    _, e_plain = spectrum_errors(low, high, data['k'], kmax)
    _, e_corr = spectrum_errors(fixed, high, data['k'], kmax)
    assert np.sqrt((e_corr**2).mean()) < 0.8 * np.sqrt((e_plain**2).mean())
    # fallback: another configuration gets the plain estimator back, bit for bit
    other = dict(corr.config, meshsize=64)
    assert np.array_equal(corr(low, data['nparticles'][-nheld:], config=other), low)
    assert corr.matches(corr.config)
    # uncorrected bins are the plain values
    assert np.array_equal(fixed[:, ~corr.mask], low[:, ~corr.mask])
