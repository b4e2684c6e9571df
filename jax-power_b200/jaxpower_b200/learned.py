"""Learned aliasing correction of low-resolution power-spectrum multipoles.

Not in the reference: a new method on top of its estimator.  A catalog painted on a
coarse mesh (here CIC, 128^3) gives multipoles biased by aliasing near the Nyquist
frequency; the same catalog painted on a 4x finer mesh gives the label.  A small BF16
MLP (``MLP``: 16 -> 128 -> 128 -> 128 -> 1, SiLU, bf16 tensor-core operands with float32
accumulation; forward pass on the tcgen05 tensor cores (accumulators in tensor memory),
backward and AdamW kernels, all in ``csrc/mlp.cu``) maps per-bin
features of the coarse spectrum

    k / k_Nyq, (k / k_Nyq)^2, one-hot ell, log(nbar P0), P2 / P0, P4 / P0, P_ell / P0,
    log(nbar V_cell)

to the correction r = (P_ell,fine - P_ell,coarse) / P0,coarse, as the training-set mean of r
per (ell, k bin) plus the network's standardised, realisation-dependent deviation from it
(calibrated so that its mean over the training mocks is zero in every bin).

``LearnedCorrection`` keeps the plain compensated coarse estimator as its fallback: it
applies the network only to spectra whose configuration (mesh, box, resampler,
interlacing, compensation, multipoles, k edges) matches the training one and whose
features lie inside the training range, and only in bins where, on held-out mocks, the
corrected spectrum was closer to the fine-mesh result than the plain one (the plain
estimator is the reference the network's error is measured against).  Elsewhere it
returns the plain values.

Training catalogs are lognormal mocks generated on the GPU by ``mock.lognormal_particles``
and measured at both resolutions by ``batch.BatchedSpectra``.
"""
import math

import numpy as np
import torch

from . import _lib
from .mesh import MeshAttrs, _device, _workspace

__all__ = ['MLP', 'LearnedCorrection', 'mock_spectra', 'spectrum_errors', 'ensemble_bias',
           'ensemble_bias_significance', 'ensemble_bias_chi2', 'NFEATURES']

NFEATURES = 16
HIDDEN = 128
_ELLS = (0, 2, 4)


def _layout():
    """(name, offset, shape) of the flat parameter vector (matches csrc/mlp.cu)."""
    shapes = [('W0', (HIDDEN, NFEATURES)), ('b0', (HIDDEN,)), ('W1', (HIDDEN, HIDDEN)), ('b1', (HIDDEN,)),
              ('W2', (HIDDEN, HIDDEN)), ('b2', (HIDDEN,)), ('W3', (8, HIDDEN)), ('b3', (8,))]
    out, off = [], 0
    for name, shape in shapes:
        out.append((name, off, shape))
        off += int(np.prod(shape))
    return out, off


class MLP:
    """The correction network; parameters live on the device.

    ``w`` (float32 master), ``wb`` (bf16 copy used as tensor-core operand), AdamW moments
    ``m``, ``v`` and the device step counter ``step``.
    """

    def __init__(self, seed=0, w=None):
        lib = _lib.load()
        layout, n = _layout()
        self.nparams = int(lib.pk_mlp_num_params())
        if self.nparams != n:
            raise RuntimeError('parameter layout mismatch: library {} vs {}'.format(self.nparams, n))
        dev = _device()
        if w is None:
            g = torch.Generator().manual_seed(int(seed))
            w = torch.zeros(n, dtype=torch.float32)
            for name, off, shape in layout:
                if name.startswith('W'):
                    fan_in = shape[1]
                    scale = 1. / math.sqrt(fan_in) if name != 'W3' else 0.1 / math.sqrt(fan_in)
                    w[off:off + int(np.prod(shape))] = torch.randn(int(np.prod(shape)), generator=g) * scale
        self.w = torch.as_tensor(w, dtype=torch.float32).to(dev).contiguous()
        self.wb = torch.empty(n, dtype=torch.bfloat16, device=dev)
        self.m = torch.zeros(n, dtype=torch.float32, device=dev)
        self.v = torch.zeros(n, dtype=torch.float32, device=dev)
        self.step = torch.zeros(1, dtype=torch.int32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)  # set if a tensor-core wait ran out
        _lib.call('pk_mlp_cast', _lib.stream_handle(), _lib.ptr(self.w), _lib.ptr(self.wb))

    def params(self, name):
        """View of one parameter block (e.g. 'W1') of the float32 master weights."""
        for n, off, shape in _layout()[0]:
            if n == name:
                return self.w[off:off + int(np.prod(shape))].view(shape)
        raise KeyError(name)

    @staticmethod
    def _x(x):
        x = torch.as_tensor(x, dtype=torch.float32, device=_device())
        if x.ndim != 2 or x.shape[1] > NFEATURES:
            raise ValueError('inputs must be (batch, <= {:d}) features'.format(NFEATURES))
        if x.shape[1] < NFEATURES:
            x = torch.nn.functional.pad(x, (0, NFEATURES - x.shape[1]))
        return x.contiguous()

    def forward(self, x, cache=False):
        """y = MLP(x) (float32, (batch,)); with ``cache`` also returns (z, h) for ``gradient``."""
        x = self._x(x)
        b = x.shape[0]
        y = torch.empty(b, dtype=torch.float32, device=x.device)
        z = h = None
        if cache:
            z = torch.empty((3, b, HIDDEN), dtype=torch.float32, device=x.device)
            h = torch.empty_like(z)
        _lib.call('pk_mlp_forward_tc', _lib.stream_handle(), _lib.ptr(x), None, b, _lib.ptr(self.wb),
                  _lib.ptr(self.w), _lib.ptr(y), _lib.ptr(z), _lib.ptr(h), _lib.ptr(self.status))
        return (y, (z, h)) if cache else y

    def check(self):
        """Raise if a tensor-core step of an earlier forward or backward pass did not complete
        (synchronises)."""
        if int(self.status.item()):
            raise RuntimeError('MLP: a tensor-core step did not complete within its wait limit')

    __call__ = forward

    def gradient(self, x, dy, cache=None):
        """d(sum_i dy_i y_i) / d(params) (flat float32), from the forward pass's cache."""
        x = self._x(x)
        b = x.shape[0]
        if cache is None:
            _, cache = self.forward(x, cache=True)
        z, h = cache
        dy = torch.as_tensor(dy, dtype=torch.float32, device=x.device).contiguous()
        grad = torch.empty(self.nparams, dtype=torch.float32, device=x.device)
        nbytes = _lib.c_size_t()
        _lib.call('pk_mlp_backward_workspace_size', b, _lib.ctypes.byref(nbytes))
        ws = _workspace(nbytes.value)
        _lib.call('pk_mlp_backward_tc', _lib.stream_handle(), _lib.ptr(x), None, b, _lib.ptr(self.wb),
                  _lib.ptr(z), _lib.ptr(h), _lib.ptr(dy), _lib.ptr(grad), _lib.ptr(ws), ws.numel(),
                  _lib.ptr(self.status))
        return grad

    def _trainer(self, x, target, weight, batch, nsteps_table, lr_table, weight_decay):
        """Buffers and an enqueuer of one training step (forward with stored activations, loss,
        backward, reduction, AdamW: 5 kernels) on the samples perm[s * batch:(s + 1) * batch]."""
        dev = x.device
        n = x.shape[0]
        nb = n // batch
        perm = torch.zeros(nb * batch, dtype=torch.int32, device=dev)
        y = torch.empty(batch, dtype=torch.float32, device=dev)
        dy = torch.empty_like(y)
        z = torch.empty((3, batch, HIDDEN), dtype=torch.float32, device=dev)
        h = torch.empty_like(z)
        grad = torch.empty(self.nparams, dtype=torch.float32, device=dev)
        losses = torch.zeros(nb, dtype=torch.float32, device=dev)
        nbytes = _lib.c_size_t()
        _lib.call('pk_mlp_backward_workspace_size', batch, _lib.ctypes.byref(nbytes))
        ws = _workspace(nbytes.value)

        def step(s):
            stream = _lib.stream_handle()
            idx = _lib.ctypes.c_void_p(perm.data_ptr() + 4 * s * batch)
            _lib.call('pk_mlp_forward_tc', stream, _lib.ptr(x), idx, batch, _lib.ptr(self.wb), _lib.ptr(self.w),
                      _lib.ptr(y), _lib.ptr(z), _lib.ptr(h), _lib.ptr(self.status))
            _lib.call('pk_mlp_mse', stream, _lib.ptr(y), _lib.ptr(target), _lib.ptr(weight), idx, batch,
                      _lib.ptr(dy), _lib.ctypes.c_void_p(losses.data_ptr() + 4 * s))
            _lib.call('pk_mlp_backward_tc', stream, _lib.ptr(x), idx, batch, _lib.ptr(self.wb), _lib.ptr(z),
                      _lib.ptr(h), _lib.ptr(dy), _lib.ptr(grad), _lib.ptr(ws), ws.numel(), _lib.ptr(self.status))
            _lib.call('pk_mlp_adam', stream, _lib.ptr(self.w), _lib.ptr(self.wb), _lib.ptr(self.m),
                      _lib.ptr(self.v), _lib.ptr(grad), _lib.ptr(lr_table), nsteps_table, _lib.ptr(self.step),
                      0.9, 0.999, 1e-8, float(weight_decay))

        return step, perm, losses, nb

    def fit(self, x, target, weight=None, steps=2000, batch=4096, lr=2e-3, lr_final=2e-5, weight_decay=0.,
            seed=0, graph=True):
        """Minimise the (weighted) MSE with AdamW on the device; returns the mean loss per epoch.

        Each epoch draws a permutation of the samples; its steps (forward, loss, backward,
        reduction, AdamW: 5 kernels each, on the tcgen05 tensor cores for the forward and
        backward passes) are captured once in a CUDA graph and replayed.  The learning rate
        follows a cosine from ``lr`` to ``lr_final`` over ``steps``.
        """
        x = self._x(x)
        dev = x.device
        n = x.shape[0]
        batch = int(min(batch, n))
        target = torch.as_tensor(target, dtype=torch.float32, device=dev).contiguous()
        weight = None if weight is None else torch.as_tensor(weight, dtype=torch.float32, device=dev).contiguous()
        nb = n // batch
        epochs = max(1, -(-int(steps) // nb))
        total = epochs * nb
        t = np.arange(total)
        lrs = lr_final + 0.5 * (lr - lr_final) * (1. + np.cos(np.pi * t / max(total - 1, 1)))
        lr_table = torch.as_tensor(lrs, dtype=torch.float32, device=dev)
        step, perm, losses, nb = self._trainer(x, target, weight, batch, total, lr_table, weight_decay)
        self.step.zero_()
        self.m.zero_()
        self.v.zero_()

        def epoch():
            for s in range(nb):
                step(s)

        gen = torch.Generator(device=dev)
        gen.manual_seed(int(seed))
        history = []
        g = None
        for e in range(epochs):
            perm.copy_(torch.randperm(n, generator=gen, device=dev)[:nb * batch].to(torch.int32))
            if graph and g is None and e == 0:
                epoch()  # first epoch eagerly (warm-up), later ones replay the graph
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):  # recorded, not executed
                    epoch()
            elif g is not None:
                g.replay()
            else:
                epoch()
            history.append(losses.mean())
        out = torch.stack(history).cpu().numpy()
        self.check()
        return out

    def fit_step_seconds(self, x, target, batch=4096, steps=20, lr=1e-4, seed=0):
        """Device time of one training step at ``batch`` (CUDA events around a replay of a CUDA
        graph of ``steps`` steps over the first samples of a random permutation; the weights are
        updated, with a small constant learning rate)."""
        x = self._x(x)
        dev = x.device
        batch = int(min(batch, x.shape[0]))
        target = torch.as_tensor(target, dtype=torch.float32, device=dev).contiguous()
        lr_table = torch.full((1,), float(lr), dtype=torch.float32, device=dev)
        step, perm, _, nb = self._trainer(x, target, None, batch, 1, lr_table, 0.)
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(seed))
        perm.copy_(torch.randperm(x.shape[0], generator=gen, device=dev)[:perm.numel()].to(torch.int32))
        for s in range(min(steps, nb)):
            step(s)  # warm-up
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for s in range(steps):
                step(s % nb)
        g.replay()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        g.replay()
        b.record()
        torch.cuda.synchronize()
        self.check()
        return a.elapsed_time(b) / 1e3 / steps

    def state(self):
        return self.w.detach().cpu().numpy().copy()


# --------------------------------------------------------------------------- data

def spectrum_norm(meshsize, boxsize, nparticles):
    """Factor turning the raw multipoles of a count mesh into overdensity power P_delta:
    P = num_raw / (N^3 / V_cell) * (N^3 / N_p)^2."""
    ncells = float(np.prod(np.asarray(meshsize, dtype='f8')))
    vcell = float(np.prod(np.asarray(boxsize, dtype='f8') / np.asarray(meshsize, dtype='f8')))
    return (ncells / vcell)**-1 * (ncells / np.asarray(nparticles, dtype='f8'))**2


def mock_spectra(seeds, meshsizes=(128, 512), boxsize=1000., nbar=1e-3, gen_meshsize=256, resampler='cic',
                 interlacing=0, compensate=True, kstep=0.01, ells=_ELLS, group=8, power=None):
    """Overdensity multipoles of lognormal mocks measured at several mesh sizes.

    Each seed gives one catalog (``mock.lognormal_particles`` on a ``gen_meshsize`` mesh
    with the benchmark power spectrum unless ``power`` is given), painted with the same
    resampler at every mesh size of ``meshsizes`` through ``BatchedSpectra`` in groups of
    ``group`` catalogs.  k edges are ``arange(0, k_Nyq(min mesh), kstep)``.

    Returns dict(k (nbins,), edges, nparticles (nmocks,), spectra {meshsize: float64
    (nmocks, nells, nbins)}, bins {meshsize: BinMesh2SpectrumPoles}).
    """
    from .mock import lognormal_particles, power_law_pk
    from .mesh2 import BinMesh2SpectrumPoles
    from .batch import BatchedSpectra
    power = power or power_law_pk()
    seeds = list(seeds)
    gen_attrs = MeshAttrs(meshsize=gen_meshsize, boxsize=boxsize)
    kmax = np.pi * min(meshsizes) / boxsize
    edges = np.arange(0., kmax * (1. + 1e-9), kstep)
    attrs = {n: MeshAttrs(meshsize=n, boxsize=boxsize) for n in meshsizes}
    bins = {n: BinMesh2SpectrumPoles(attrs[n], edges=edges, ells=ells) for n in meshsizes}
    spectra = {n: [] for n in meshsizes}
    nparticles = []
    for start in range(0, len(seeds), group):
        cats = [lognormal_particles(gen_attrs, power, nbar, seed=int(s)) for s in seeds[start:start + group]]
        counts = [c.shape[0] for c in cats]
        nparticles += counts
        pos = torch.cat(cats)
        del cats
        for n in meshsizes:
            bs = BatchedSpectra(attrs[n], bins[n], counts, resampler=resampler, interlacing=interlacing,
                                compensate=compensate, los='z', graph=False)
            raw = bs(pos)
            norm = torch.as_tensor(spectrum_norm(attrs[n].meshsize, boxsize, counts), device=raw.device)
            spectra[n].append((raw * norm[:, None, None]).cpu().numpy())
            del bs
    k = bins[min(meshsizes)].xavg
    return dict(k=k, edges=edges, nparticles=np.array(nparticles), boxsize=boxsize, nbar=nbar,
                spectra={n: np.concatenate(v) for n, v in spectra.items()}, bins=bins)


def spectrum_errors(p, ref, k, kmax):
    """Per-mock max over bins k <= kmax and multipoles of |p - ref| / ref_0 (the monopole
    of the reference sets the scale of every multipole), and the per-bin errors."""
    sel = np.asarray(k) <= kmax
    err = np.abs(np.asarray(p) - np.asarray(ref))[:, :, sel] / np.abs(np.asarray(ref)[:, :1, sel])
    return err.max(axis=(1, 2)), err


def ensemble_bias_significance(p, ref, k, kmax):
    """max over (ell, bin) of |mean(p - ref)| / (standard error of that mean): how many
    standard errors the worst bin's mean deviation is from zero."""
    sel = np.asarray(k) <= kmax
    d = (np.asarray(p) - np.asarray(ref))[:, :, sel]
    se = d.std(axis=0, ddof=1) / np.sqrt(d.shape[0])
    return float((np.abs(d.mean(axis=0)) / np.where(se > 0, se, np.inf)).max())


def ensemble_bias_chi2(p, ref, k, kmax):
    """Mean over (ell, bin) with k <= kmax of the squared standard score of mean(p - ref): about 1
    for an unbiased estimator (bins are correlated, so it scatters more than a chi^2 / dof would),
    and 1 + nheld / ntrain for one calibrated on ntrain other mocks."""
    sel = np.asarray(k) <= kmax
    d = (np.asarray(p) - np.asarray(ref))[:, :, sel]
    se = d.std(axis=0, ddof=1) / np.sqrt(d.shape[0])
    return float(((d.mean(axis=0) / np.where(se > 0, se, np.inf))**2).mean())


def ensemble_bias(p, ref, k, kmax):
    """Systematic error over an ensemble of mocks: per (ell, bin) with k <= kmax,
    |mean(p - ref)| / mean(ref_0), shape (nells, nbins_kept).

    Per mock, p - ref also carries the coarse mesh's aliased cross terms (delta(k) times
    delta*(k + 2 k_Nyq n)), which average to zero and which no function of the binned
    coarse multipoles can predict; the ensemble mean isolates the aliasing bias.
    """
    sel = np.asarray(k) <= kmax
    d = (np.asarray(p) - np.asarray(ref))[:, :, sel].mean(axis=0)
    return np.abs(d) / np.abs(np.asarray(ref)[:, :1, sel].mean(axis=0))


# --------------------------------------------------------------------------- correction

class LearnedCorrection:
    """MLP correction of coarse-mesh multipoles towards the fine-mesh estimator.

    Parameters
    ----------
    config : dict describing the coarse estimator the network was trained for
        (meshsize, boxsize, resampler, interlacing, compensate, ells, edges)
    """

    def __init__(self, config, mlp=None, xmean=None, xstd=None, tmean=None, tstd=None, mask=None,
                 xmin=None, xmax=None):
        self.config = dict(config)
        self.mlp = mlp
        self.xmean, self.xstd, self.tmean, self.tstd = xmean, xstd, tmean, tstd
        self.mask = mask
        self.xmin, self.xmax = xmin, xmax

    # ---- features (computed on the device: no host round trip when correcting)
    def _dev(self, name):
        cache = self.__dict__.setdefault('_dev_cache', {})
        if name not in cache:
            value = self.config['edges'] if name == 'edges' else getattr(self, name)
            dtype = 'bool' if name == 'mask' else 'f8'
            cache[name] = torch.as_tensor(np.asarray(value, dtype=dtype), device=_device())
        return cache[name]

    def _raw_features(self, p, nparticles):
        """(nmocks * nells * nbins, NFEATURES) float64 features of coarse multipoles p
        ((nmocks, nells, nbins) float64 device tensor; nparticles: (nmocks,) float64 device tensor)."""
        nm, nl, nb = p.shape
        cfg = self.config
        edges = self._dev('edges')
        knyq = np.pi * cfg['meshsize'] / cfg['boxsize']
        nbar = nparticles.reshape(-1) / cfg['boxsize']**3
        vcell = (cfg['boxsize'] / cfg['meshsize'])**3
        p0 = p[:, 0]
        f = torch.zeros((nm, nl, nb, NFEATURES), dtype=torch.float64, device=p.device)
        x = 0.5 * (edges[:-1] + edges[1:]) / knyq
        f[..., 0] = x
        f[..., 1] = x * x
        for il, ell in enumerate(cfg['ells']):
            f[:, il, :, 2 + _ELLS.index(ell)] = 1.
        f[..., 5] = torch.log(torch.clamp(nbar[:, None, None] * p0[:, None, :], min=1e-6))
        for j, ell in enumerate((2, 4)):
            if ell in cfg['ells']:
                f[..., 6 + j] = (p[:, list(cfg['ells']).index(ell)] / p0)[:, None, :]
        f[..., 8] = p / p0[:, None, :]
        f[..., 9] = torch.log(nbar * vcell)[:, None, None]
        return f.reshape(-1, NFEATURES)

    @classmethod
    def train(cls, data, meshsize, label_meshsize, resampler='cic', interlacing=0, compensate=True,
              val_fraction=0.125, steps=3000, batch=4096, lr=2e-3, seed=0, kmax_fraction=1.):
        """Train on ``mock_spectra`` output; returns (correction, report).

        The last ``val_fraction`` of the mocks is held out to choose the corrected bins.
        """
        ells = tuple(data['bins'][meshsize].ells)
        config = dict(meshsize=int(meshsize), boxsize=float(data['boxsize']), resampler=resampler,
                      interlacing=int(interlacing), compensate=bool(compensate), ells=ells,
                      edges=np.asarray(data['edges'], dtype='f8'))
        self = cls(config)
        dev = _device()
        p_low = torch.as_tensor(np.asarray(data['spectra'][meshsize], dtype='f8'), device=dev)
        p_high = torch.as_tensor(np.asarray(data['spectra'][label_meshsize], dtype='f8'), device=dev)
        npart = torch.as_tensor(np.asarray(data['nparticles'], dtype='f8'), device=dev)
        nm, nl, nb = p_low.shape
        nval = max(1, int(round(val_fraction * nm)))
        ntr = nm - nval
        x = self._raw_features(p_low[:ntr], npart[:ntr])
        t = (p_high[:ntr] - p_low[:ntr]) / p_low[:ntr, :1]  # (ntr, nells, nbins)
        table = t.mean(dim=0)  # mean correction per (ell, bin)
        res = t - table[None]
        tstd = res.pow(2).mean(dim=(0, 2)).sqrt()  # per ell
        tstd[tstd < 1e-12] = 1.
        self.tmean, self.tstd = table.cpu().numpy(), tstd.cpu().numpy()
        xstd = x.std(dim=0, unbiased=False)
        xstd[xstd < 1e-12] = 1.
        self.xmean, self.xstd = x.mean(dim=0).cpu().numpy(), xstd.cpu().numpy()
        xs = (x - self._dev('xmean')) / self._dev('xstd')
        self.xmin, self.xmax = xs.min(dim=0).values.cpu().numpy(), xs.max(dim=0).values.cpu().numpy()
        ts = (res / tstd[None, :, None]).reshape(-1)
        self.mlp = MLP(seed=seed)
        history = self.mlp.fit(xs, ts, steps=steps, batch=batch, lr=lr, seed=seed)
        # calibrate: the network's mean predicted deviation over the training set, per
        # (ell, bin), is folded into the table, so the mean correction over the training mocks
        # is exactly the training-set mean (the network keeps only the realisation-dependent
        # part)
        y = torch.cat([self.mlp(xs[i:i + 65536].to(torch.float32)) for i in range(0, xs.shape[0], 65536)])
        ybar = (y.double().reshape(ntr, nl, nb) * tstd[None, :, None]).mean(dim=0)
        self.tmean = (table - ybar).cpu().numpy()
        self.__dict__.pop('_dev_cache', None)
        # choose the bins to correct on the held-out mocks
        self.mask = np.ones((nl, nb), dtype=bool)
        corr = self._apply(p_low[ntr:], npart[ntr:], use_mask=False).cpu().numpy()
        lo, hi = p_low[ntr:].cpu().numpy(), p_high[ntr:].cpu().numpy()
        e_corr = np.abs(corr - hi) / np.abs(hi[:, :1])
        e_plain = np.abs(lo - hi) / np.abs(hi[:, :1])
        rms_corr, rms_plain = np.sqrt((e_corr**2).mean(axis=0)), np.sqrt((e_plain**2).mean(axis=0))
        kcen = 0.5 * (config['edges'][:-1] + config['edges'][1:])
        knyq = np.pi * meshsize / config['boxsize']
        # a bin falls back to the plain estimator only where the network is clearly worse on the
        # validation mocks: rms error above the plain one by more than 10 % (about three standard
        # errors of an rms over 512 mocks) and above 0.1 % of P0.  Falling back on statistical
        # ties would bring the plain estimator's small but significant low-k offsets back into
        # bins the network leaves unbiased.
        self.mask = (((rms_corr <= 1.1 * rms_plain) | (rms_corr <= 1e-3))
                     & (kcen <= kmax_fraction * knyq)[None, :])
        self.__dict__.pop('_dev_cache', None)
        self.__dict__.pop('_graphs', None)
        report = dict(loss_history=history, ntrain=ntr, nval=nval, corrected_bins=int(self.mask.sum()),
                      total_bins=int(self.mask.size), val_rms_corrected=rms_corr, val_rms_plain=rms_plain)
        return self, report

    def _apply(self, p, nparticles, use_mask=True):
        """Corrected multipoles of p ((nmocks, nells, nbins) float64 device tensor)."""
        nm, nl, nb = p.shape
        xs = (self._raw_features(p, nparticles) - self._dev('xmean')) / self._dev('xstd')
        y = self.mlp(xs.to(torch.float32)).double().reshape(nm, nl, nb)
        r = self._dev('tmean')[None] + y * self._dev('tstd')[None, :, None]
        corr = p + r * p[:, :1]
        # spectra with features outside the training range (widened by half its span) fall
        # back entirely
        xmin, xmax = self._dev('xmin'), self._dev('xmax')
        margin = 0.5 * (xmax - xmin) + 1e-6
        inside = ((xs >= xmin - margin) & (xs <= xmax + margin)).reshape(nm, -1).all(dim=1)
        use = inside[:, None, None].expand(nm, nl, nb)
        if use_mask:
            use = use & self._dev('mask')[None]
        return torch.where(use, corr, p)

    def matches(self, config):
        """True if an estimator configuration is the one the network was trained for."""
        c = self.config
        try:
            return (int(config['meshsize']) == c['meshsize'] and np.isclose(float(config['boxsize']), c['boxsize'])
                    and config['resampler'] == c['resampler'] and int(config['interlacing']) == c['interlacing']
                    and bool(config['compensate']) == c['compensate'] and tuple(config['ells']) == tuple(c['ells'])
                    and len(config['edges']) == len(c['edges'])
                    and np.allclose(np.asarray(config['edges'], dtype='f8'), c['edges']))
        except (KeyError, TypeError, ValueError):
            return False

    def __call__(self, p_low, nparticles, config=None):
        """Corrected overdensity multipoles ((nmocks, nells, nbins) or (nells, nbins)).

        ``p_low`` is a NumPy array (result returned as NumPy) or a device tensor (result
        stays on the device, no host synchronisation).  Falls back to the plain values when
        ``config`` (if given) differs from the training configuration, for spectra outside
        the training feature range and in bins where the correction did not beat the plain
        estimator on held-out mocks.
        """
        on_device = isinstance(p_low, torch.Tensor)
        dev = _device()
        p = p_low.to(torch.float64) if on_device else torch.as_tensor(np.asarray(p_low, dtype='f8'), device=dev)
        single = p.ndim == 2
        if single:
            p = p[None]
        if config is not None and not self.matches(config):
            out = p.clone()
        else:
            npart = nparticles if isinstance(nparticles, torch.Tensor) else np.atleast_1d(np.asarray(nparticles))
            npart = torch.as_tensor(npart, dtype=torch.float64, device=dev).reshape(-1)
            out = self._graphed(p.contiguous(), npart) if self.graph else self._apply(p, npart)
        out = out[0] if single else out
        return out if on_device else out.cpu().numpy()

    graph = True  # replay the correction from a CUDA graph per input shape

    def _graphed(self, p, npart):
        graphs = self.__dict__.setdefault('_graphs', {})
        key = tuple(p.shape)
        if key not in graphs:
            sp, sn = p.clone(), npart.clone()
            self._apply(sp, sn)  # warm-up: builds the device constants outside capture
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                out = self._apply(sp, sn)
            graphs[key] = (g, sp, sn, out)
        g, sp, sn, out = graphs[key]
        sp.copy_(p)
        sn.copy_(npart)
        g.replay()
        return out.clone()
