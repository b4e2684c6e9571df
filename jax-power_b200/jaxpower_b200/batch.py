"""Batched power spectra of many catalogs (mocks) sharing a mesh geometry.

The reference computes mock spectra one at a time (``ParticleField.paint`` +
``compute_mesh2_spectrum`` per mock, ``mesh.py:2604-2754`` / ``mesh2.py:253-374``).  Here
a batch of catalogs goes through one paint launch sequence (``pk_paint_batch``: tiles of
every mock in one grid), one batched cuFFT R2C and one ``pk_bin_global_interlaced`` (the
interlaced, compensated meshes binned as they are formed, never stored; for other
multipole sets ``pk_interlace_compensate_batch`` then ``pk_bin_global_batch``), all on
static buffers and captured once in a CUDA graph;
each further batch of the same sizes is a graph replay.  The paint tile configuration is
picked by the autotuner (``autotune.py``).

Supports the global line of sight (the mock-covariance use case) with interlacing <= 4.
"""
import numpy as np
import torch

from . import _lib
from . import resamplers
from .autotune import best_tile_config, make_key
from .mesh import _plan, _device, _workspace
from .mesh2 import _los, _ell_factors, _fusable, _plain_bins

__all__ = ['BatchedSpectra']


class BatchedSpectra:
    """Multipoles of ``len(counts)`` catalogs with the given particle counts.

    Parameters
    ----------
    attrs : MeshAttrs shared by all catalogs
    bin : BinMesh2SpectrumPoles on ``attrs``
    counts : particles per catalog (the concatenated positions follow this order)
    resampler, interlacing, compensate, los : as ``ParticleField.paint`` / ``compute_mesh2_spectrum``
    tile_config : paint tile configuration, or None to autotune on the first call's inputs
    graph : capture the batch in a CUDA graph (at the first call, replayed by every call)
    """

    def __init__(self, attrs, bin, counts, resampler='tsc', interlacing=2, compensate=True, los='z',
                 tile_config=None, graph=True, weights=False):
        _plain_bins(bin, 'BatchedSpectra')
        self.attrs, self.bin = attrs, bin
        self.order = resamplers.get_resampler(resampler).order
        self.interlacing = max(int(interlacing), 1)
        if self.interlacing > 4:
            raise NotImplementedError('batched spectra support interlacing <= 4')
        self.compensate = bool(compensate)
        self.los, self.vlos, _ = _los(los)
        if self.vlos is None:
            raise NotImplementedError('batched spectra support a global line of sight')
        counts = np.asarray(counts, dtype='i8')
        self.nmocks = len(counts)
        offsets = np.concatenate([[0], np.cumsum(counts)]).astype('i8')
        self.n = int(offsets[-1])
        dev = _device()
        self.offsets = torch.as_tensor(offsets, device=dev)
        self.positions = torch.zeros((self.n, 3), dtype=torch.float32, device=dev)
        self.weights = torch.ones(self.n, dtype=torch.float32, device=dev) if weights else None
        shape = tuple(int(s) for s in attrs.meshsize)
        nz = shape[2] // 2 + 1
        M, I = self.nmocks, self.interlacing
        self.real = torch.empty((M, I) + shape, dtype=torch.float32, device=dev)
        self.cplx = torch.empty((M, I, shape[0], shape[1], nz), dtype=torch.complex64, device=dev)
        # even multipoles (ell <= 4): bin straight from the shifted meshes, no combined mesh
        self.fused = _fusable(bin.ells)
        self.comb = None if self.fused else torch.empty((M, shape[0], shape[1], nz), dtype=torch.complex64,
                                                         device=dev)
        self.nells, self.nbins = len(bin.ells), bin.nbins
        self.raw = torch.zeros(M * self.nells * self.nbins, dtype=torch.float64, device=dev)
        self.status_flag = torch.zeros(1, dtype=torch.int32, device=dev)
        nbytes = _lib.c_size_t()
        _lib.call('pk_bin_batch_workspace_size', _lib.i32(shape), len(bin._edges1d), self.nells, M,
                  _lib.ctypes.byref(nbytes))
        self.bin_ws = _workspace(nbytes.value)
        self.plan = _plan(shape, M * I, 0)
        factors = torch.tensor(_ell_factors(bin.ells, self.vlos), dtype=torch.float64, device=dev)
        self.scale = factors[:, None] / torch.as_tensor(bin.nmodes, dtype=torch.float64, device=dev)[None, :]
        self.tile_config = tile_config
        self.use_graph = bool(graph)
        self.graph = None
        self.paint_ws = None
        self._ready = False

    def _prepare(self):
        """Autotune (on the first real inputs), allocate the paint workspace, capture the graph."""
        if self.tile_config is None:
            shape = tuple(int(s) for s in self.attrs.meshsize)
            key = make_key('paint', shape, self.order, self.interlacing, self.nmocks,
                           int(np.log2(max(self.n // max(self.nmocks, 1), 1))))
            self.tile_config = best_tile_config(key, self._paint_with)
        self.paint_ws = self._paint_workspace(self.tile_config)
        if self.use_graph:
            self._enqueue()  # warm-up outside capture
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._enqueue()
            self.graph = g
        self._ready = True

    def _paint_workspace(self, config):
        nbytes = _lib.c_size_t()
        _lib.call('pk_paint_batch_workspace_size', self.n, self.nmocks, _lib.i32(self.attrs.meshsize), self.order,
                  self.interlacing, config, _lib.ctypes.byref(nbytes))
        return _workspace(nbytes.value)

    def _paint_with(self, config, ws=None):
        a = self.attrs
        if ws is None:
            ws = self._paint_workspace(config)
        _lib.call('pk_paint_batch', _lib.stream_handle(), _lib.ptr(self.positions), _lib.ptr(self.weights),
                  _lib.ptr(self.offsets), self.n, self.nmocks, _lib.i32(a.meshsize), _lib.f32(a.boxsize),
                  _lib.f32(a.boxcenter), _lib.f32(a.cellsize), self.order, self.interlacing, 0, self.interlacing,
                  config, _lib.ptr(self.real), _lib.ptr(ws), ws.numel(), _lib.ptr(self.status_flag))

    def _enqueue(self):
        a, b = self.attrs, self.bin
        stream = _lib.stream_handle()
        self.status_flag.zero_()  # inside the graph: every replay reports its own inputs
        self._paint_with(self.tile_config, self.paint_ws)
        _lib.call('pk_fft_exec', self.plan, stream, _lib.ptr(self.real), _lib.ptr(self.cplx))
        if self.fused:
            _lib.call('pk_bin_global_interlaced', stream, _lib.ptr(self.cplx), self.nmocks, self.interlacing,
                      self.order if self.compensate else 0, _lib.i32(a.meshsize), _lib.f32(a.kfun), _lib.f32(self.vlos),
                      _lib.ptr(b.d_edges), len(b._edges1d), b._step, a.backend_code, self.nells, _lib.i32(b.ells),
                      _lib.ptr(self.raw), _lib.ptr(self.bin_ws), self.bin_ws.numel())
            return
        _lib.call('pk_interlace_compensate_batch', stream, _lib.ptr(self.cplx), self.nmocks, self.interlacing,
                  _lib.i32(a.meshsize), self.order if self.compensate else 0, a.backend_code, 0, 1.,
                  _lib.ptr(self.comb))
        _lib.call('pk_bin_global_batch', stream, _lib.ptr(self.comb), None, self.nmocks, _lib.i32(a.meshsize),
                  _lib.f32(a.kfun), _lib.f32(self.vlos), _lib.ptr(b.d_edges), len(b._edges1d), b._step,
                  a.backend_code, self.nells, _lib.i32(b.ells), _lib.ptr(self.raw), _lib.ptr(self.bin_ws),
                  self.bin_ws.numel())

    def __call__(self, positions=None, weights=None, check=True):
        """Multipoles ``num_raw`` of every catalog: (nmocks, nells, nbins) float64 on the device.

        ``positions`` (concatenated, (n, 3)) are copied into the static input buffer first.
        ``check``: raise ``ValueError`` if a particle was dropped (non-finite position or
        weight, or a position far outside the box), as ``ParticleField.paint`` does; this waits
        for the batch.  With ``check=False`` the call stays asynchronous and ``status()`` reads
        the flag later.
        """
        if positions is not None:
            self.positions.copy_(positions)
        if weights is not None:
            if self.weights is None:
                raise ValueError('construct with weights=True to pass weights')
            self.weights.copy_(weights)
        if not self._ready:
            self._prepare()
        if self.graph is not None:
            self.graph.replay()
        else:
            self._enqueue()
        if check and self.status():
            raise ValueError('non-finite or out-of-range particle positions / weights in the batch '
                             '(those particles were not painted)')
        return self.raw.view(self.nmocks, self.nells, self.nbins) * self.scale

    def status(self):
        """Nonzero if the last batch dropped a particle (waits for that batch)."""
        return int(self.status_flag.item())
