"""Mesh data model, particles and painting (host side of the CUDA library).

Mirrors the single-GPU parts of ``jaxpower/mesh.py``:

- ``MeshAttrs`` (``mesh.py:1453-1719``): meshsize / boxsize / boxcenter, cellsize,
  kfun, knyq, rcoords / kcoords, create, r2c / c2r;
- ``RealMeshField`` / ``ComplexMeshField`` (``mesh.py:1724-2196``);
- ``ParticleField`` (``mesh.py:2398-2670``) and ``FKPField`` (``mesh.py:2913-2999``);
- ``_paint`` (``mesh.py:2673-2754``): paint, interlacing, compensation, out;
- ``_read`` (``mesh.py:2064-2110``); ``get_mesh_attrs`` / ``next_fft_size``
  (``mesh.py:2271-2381``).

Arrays are torch CUDA tensors; every computation on them goes through the C ABI
of ``libjaxpower_b200.so`` (paint / read / FFT / interlace / compensate).  The
complex layout is the Hermitian ``(N0, N1, N2 // 2 + 1)`` one.  ``fft_backend``
selects the reference's FFT-backend semantics ('jax': rfftn; 'jaxdecomp': full
complex FFT, reproduced on the Hermitian storage).  Only float32 meshes are
supported (the reference's default dtype with x64 off).
"""
import math
import operator
from functools import lru_cache

import numpy as np
import torch

from . import _lib
from . import resamplers

__all__ = ['MeshAttrs', 'RealMeshField', 'ComplexMeshField', 'ParticleField', 'FKPField', 'split_particles',
           'get_mesh_attrs', 'next_fft_size', 'r2c', 'c2r', 'paint', 'read']


def _device():
    if not torch.cuda.is_available():
        raise RuntimeError('jaxpower_b200 needs a CUDA device (B200); there is no CPU fallback')
    return torch.device('cuda', torch.cuda.current_device())


def _fill3(value, dtype):
    return np.broadcast_to(np.asarray(value, dtype=dtype), (3,)).copy()


def _as_positions(positions):
    if isinstance(positions, torch.Tensor):
        t = positions
    else:
        t = torch.as_tensor(np.asarray(positions))
    t = t.to(device=_device(), dtype=torch.float32)
    if t.ndim != 2 or t.shape[-1] != 3:
        raise ValueError('positions must have shape (N, 3), got {}'.format(tuple(t.shape)))
    return t.contiguous()


def _as_weights(weights, n):
    if weights is None:
        return None
    t = weights if isinstance(weights, torch.Tensor) else torch.as_tensor(np.asarray(weights))
    t = t.to(device=_device(), dtype=torch.float32)
    if t.ndim == 0:
        t = t.expand(n)
    if t.shape != (n,):
        raise ValueError('weights must have shape ({},), got {}'.format(n, tuple(t.shape)))
    return t.contiguous()


def _workspace(nbytes):
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=_device())


# ---------------------------------------------------------------------- FFT plans

class _Plan(_lib.c_void_p):
    """A cuFFT plan handle (``pk_fft_plan``) destroyed, with its work area, when the last
    reference goes: the plan cache below and any holder that outlives it (a captured CUDA
    graph's owner such as ``BatchedSpectra``) keep it alive."""

    nbytes = 0

    def __del__(self):
        if self.value:
            try:
                _lib.load().pk_fft_plan_destroy(self)
            except Exception:  # interpreter shutdown
                pass
            self.value = None


# Least-recently-used plan cache.  Each plan holds its own work area (about the size of its
# complex batch), which the torch caching allocator cannot see, so the cache is bounded by
# count and by those bytes; an evicted plan is destroyed once nothing else refers to it.
_PLANS = {}
_PLAN_CACHE_MAX = 16
_PLAN_CACHE_BYTES_FRACTION = 0.125


def _plan(meshsize, batch, direction):
    # one plan per stream: a cuFFT plan owns one work area, so transforms enqueued on different
    # streams (which may run concurrently) must not share a plan
    key = (torch.cuda.current_device(), tuple(int(n) for n in meshsize), int(batch), int(direction),
           torch.cuda.current_stream().cuda_stream)
    plan = _PLANS.pop(key, None)
    if plan is None:
        plan = _Plan()
        _lib.call('pk_fft_plan_create', _lib.i32(meshsize), int(batch), int(direction),
                  _lib.ctypes.byref(plan))
        n0, n1, n2 = key[1]
        plan.nbytes = 8 * int(batch) * n0 * n1 * (n2 // 2 + 1)
        limit = _PLAN_CACHE_BYTES_FRACTION * torch.cuda.get_device_properties(key[0]).total_memory
        while _PLANS and (len(_PLANS) >= _PLAN_CACHE_MAX
                          or sum(p.nbytes for p in _PLANS.values()) + plan.nbytes > limit):
            _PLANS.pop(next(iter(_PLANS)))  # oldest use first
    _PLANS[key] = plan  # most recent last
    return plan


def _r2c(value, meshsize):
    """Batched out-of-place R2C of contiguous real meshes (..., N0, N1, N2)."""
    shape = tuple(int(n) for n in meshsize)
    value = value.contiguous()
    batch = value.numel() // int(np.prod(shape))
    out = torch.empty(value.shape[:-3] + shape[:2] + (shape[2] // 2 + 1,), dtype=torch.complex64,
                      device=value.device)
    _lib.call('pk_fft_exec', _plan(shape, batch, 0), _lib.stream_handle(), _lib.ptr(value), _lib.ptr(out))
    return out


def _c2r(value, meshsize, scale=True, destroy_input=False):
    """Batched C2R; ``scale`` applies jnp.fft.irfftn's 1 / N; the input is preserved unless destroy_input."""
    shape = tuple(int(n) for n in meshsize)
    if not destroy_input:
        value = value.clone()
    value = value.contiguous()
    batch = value.numel() // (shape[0] * shape[1] * (shape[2] // 2 + 1))
    out = torch.empty(value.shape[:-3] + shape, dtype=torch.float32, device=value.device)
    _lib.call('pk_fft_exec', _plan(shape, batch, 1), _lib.stream_handle(), _lib.ptr(value), _lib.ptr(out))
    if scale:
        _lib.call('pk_scale_real', _lib.stream_handle(), _lib.ptr(out), out.numel(),
                  float(np.float32(1. / np.prod(shape))))
    return out


def _backend_code(backend):
    return _lib.PK_BACKEND_JAXDECOMP if backend == 'jaxdecomp' else _lib.PK_BACKEND_JAX


# ---------------------------------------------------------------------- MeshAttrs

class MeshAttrs:
    """Mesh attributes (``mesh.py:1455-1719``).

    Parameters
    ----------
    meshsize : int or (3,) ints
    boxsize : float or (3,), default meshsize
    boxcenter : float or (3,), default 0
    dtype : only float32 is supported ('float', 'f4', np.float32)
    fft_backend : 'auto' (= 'jax'), 'jax' or 'jaxdecomp' (semantics of the reference's backends)
    """

    def __init__(self, meshsize=None, boxsize=None, boxcenter=0., dtype=float, fft_backend='auto'):
        if meshsize is not None:
            meshsize = _fill3(meshsize, 'i4')
            if boxsize is None:
                boxsize = 1. * meshsize
        if dtype not in (float, None) and np.dtype(dtype) != np.float32:
            raise NotImplementedError('only float32 meshes are supported, got {}'.format(dtype))
        if fft_backend == 'auto':
            fft_backend = 'jax'
        if fft_backend not in ('jax', 'jaxdecomp'):
            raise ValueError('fft_backend must be auto, jax or jaxdecomp')
        self.meshsize = meshsize
        self.boxsize = None if boxsize is None else _fill3(boxsize, 'f4')
        self.boxcenter = None if boxcenter is None else _fill3(boxcenter, 'f4')
        self.dtype = np.dtype('f4')
        self.fft_backend = fft_backend

    # mapping interface, as the reference's dataclass
    def keys(self):
        return ['meshsize', 'boxsize', 'boxcenter', 'dtype', 'fft_backend']

    def __getitem__(self, key):
        return getattr(self, key)

    def clone(self, **kwargs):
        state = {name: getattr(self, name) for name in self.keys()}
        state.update(kwargs)
        if state['dtype'] is not None and np.dtype(state['dtype']) == np.float32:
            state['dtype'] = float
        return MeshAttrs(**state)

    def __repr__(self):
        return 'MeshAttrs(meshsize={}, boxsize={}, boxcenter={}, fft_backend={!r})'.format(
            self.meshsize.tolist(), self.boxsize.tolist(), self.boxcenter.tolist(), self.fft_backend)

    def __eq__(self, other):
        return (isinstance(other, MeshAttrs) and np.array_equal(self.meshsize, other.meshsize)
                and np.array_equal(self.boxsize, other.boxsize)
                and np.array_equal(self.boxcenter, other.boxcenter) and self.fft_backend == other.fft_backend)

    __hash__ = None

    @property
    def rdtype(self):
        return np.dtype('f4')

    @property
    def cdtype(self):
        return np.dtype('c8')

    @property
    def ndim(self):
        return 3

    @property
    def is_hermitian(self):
        return True

    @property
    def cellsize(self):
        """boxsize / meshsize in float32 (``mesh.py:1575``)."""
        return (self.boxsize / self.meshsize.astype('f4')).astype('f4')

    @property
    def kfun(self):
        """2 pi / boxsize in float32 (``mesh.py:1580``)."""
        return (np.float32(2. * np.pi) / self.boxsize).astype('f4')

    @property
    def knyq(self):
        return (np.pi * self.meshsize / self.boxsize.astype('f8')).astype('f4')

    @property
    def backend_code(self):
        return _backend_code(self.fft_backend)

    def _freq(self, axis, kind, hermitian):
        n = int(self.meshsize[axis])
        if hermitian and self.fft_backend == 'jax':
            k = np.arange(0, n // 2 + 1, dtype='f4')
        else:
            idx = np.arange(n // 2 + 1 if hermitian else n)
            k = np.where(idx < (n + 1) // 2, idx, idx - n).astype('f4')
        f = (k / np.float32(n)).astype('f4')
        if kind == 'wavenumber':
            spacing = self.kfun[axis]
        elif kind == 'circular':
            spacing = np.float32(2. * np.pi / n)
        elif kind == 'index':
            spacing = np.float32(1.)
        else:
            raise ValueError('unknown kind {}'.format(kind))
        return ((f * spacing).astype('f4') * np.float32(n)).astype('f4')

    def kcoords(self, kind='wavenumber', sparse=None):
        """Fourier coordinates of the Hermitian grid (``mesh.py:1605-1636``), torch float32."""
        if kind == 'separation':
            kind = 'wavenumber'
        toret = [self._freq(axis, kind, hermitian=(axis == 2)) for axis in range(3)]
        return _meshgrid(toret, sparse)

    ccoords = kcoords

    def rcoords(self, kind='position', sparse=None):
        """Cell-corner positions, indices or separations (``mesh.py:1594-1603``), torch float32."""
        toret = []
        for axis in range(3):
            n = int(self.meshsize[axis])
            if kind == 'index':
                toret.append(np.arange(n, dtype='i4'))
                continue
            if kind == 'separation':  # fftfreq(n) * cellsize * n (mesh.py:392-394), float32
                sf = np.where(np.arange(n) < (n + 1) // 2, np.arange(n), np.arange(n) - n).astype('f4')
                x = ((sf / np.float32(n)).astype('f4') * np.float32(self.cellsize[axis])).astype('f4') * np.float32(n)
                toret.append(x.astype('f4'))
                continue
            x = (np.arange(n, dtype='f4') * self.cellsize[axis]).astype('f4')
            if kind == 'position':
                off = np.float32(self.boxcenter[axis] - np.float32(self.boxsize[axis] / np.float32(2.)))
                x = (x + off).astype('f4')
            else:
                raise ValueError('unknown kind {}'.format(kind))
            toret.append(x)
        return _meshgrid(toret, sparse)

    xcoords = rcoords

    def create(self, kind='real', fill=None):
        """Create a mesh (``mesh.py:1641-1677``)."""
        kind = {'real': RealMeshField, 'complex': ComplexMeshField}.get(kind, kind)
        shape = tuple(int(n) for n in self.meshsize)
        if kind is ComplexMeshField:
            shape = shape[:2] + (shape[2] // 2 + 1,)
            dtype = torch.complex64
        else:
            dtype = torch.float32
        if callable(fill):
            value = torch.as_tensor(fill(shape), device=_device()).to(dtype)
        elif fill is None:
            value = torch.empty(shape, dtype=dtype, device=_device())
        elif isinstance(fill, torch.Tensor) and tuple(fill.shape) == shape:
            value = fill.to(device=_device(), dtype=dtype)
        else:
            value = torch.full(shape, fill, dtype=dtype, device=_device())
        return kind(value, attrs=self)

    def r2c(self, value):
        return _r2c(value, self.meshsize)

    def c2r(self, value):
        return _c2r(value, self.meshsize)


def _meshgrid(arrays, sparse):
    dev = _device()
    ts = [torch.as_tensor(a, device=dev) for a in arrays]
    if sparse is None:
        return tuple(ts)
    if sparse:
        out = []
        for i, t in enumerate(ts):
            shape = [1, 1, 1]
            shape[i] = t.numel()
            out.append(t.reshape(shape))
        return tuple(out)
    return tuple(torch.meshgrid(*ts, indexing='ij'))


# ---------------------------------------------------------------------- fields

class BaseMeshField:
    """A mesh value (torch tensor) with its ``MeshAttrs`` (``mesh.py:1724-1918``)."""

    def __init__(self, value, attrs=None, **kwargs):
        if not isinstance(value, torch.Tensor):
            value = torch.as_tensor(np.asarray(value))
        value = value.to(_device())
        if attrs is None:
            meshsize = kwargs.pop('meshsize', None)
            if meshsize is None:
                meshsize = value.shape
                if isinstance(self, ComplexMeshField):
                    raise ValueError('provide attrs for a complex mesh')
            attrs = MeshAttrs(meshsize=meshsize, **kwargs)
        elif not isinstance(attrs, MeshAttrs):
            attrs = MeshAttrs(**dict(attrs))
        if kwargs:
            attrs = attrs.clone(**kwargs)
        self.value = value
        self.attrs = attrs

    def clone(self, **kwargs):
        value = kwargs.pop('value', self.value)
        attrs = kwargs.pop('attrs', self.attrs)
        if kwargs:
            attrs = attrs.clone(**kwargs)
        return self.__class__(value, attrs=attrs)

    def __getitem__(self, item):
        return self.value[item]

    def __array__(self, dtype=None, copy=None):
        a = self.value.detach().cpu().numpy()
        return a.astype(dtype) if dtype is not None else a

    @property
    def shape(self):
        return tuple(self.value.shape)

    @property
    def size(self):
        return self.value.numel()

    @property
    def ndim(self):
        return self.value.ndim

    @property
    def dtype(self):
        return self.value.dtype

    @property
    def real(self):
        return self.value.real

    @property
    def imag(self):
        return self.value.imag

    meshsize = property(lambda self: self.attrs.meshsize)
    boxsize = property(lambda self: self.attrs.boxsize)
    boxcenter = property(lambda self: self.attrs.boxcenter)
    cellsize = property(lambda self: self.attrs.cellsize)

    def sum(self, *args, **kwargs):
        return self.value.sum(*args, **kwargs)

    def mean(self, *args, **kwargs):
        return self.value.mean(*args, **kwargs)

    def std(self):
        return self.value.std(unbiased=False)

    def var(self):
        return self.value.var(unbiased=False)

    def min(self):
        return self.value.min()

    def max(self):
        return self.value.max()

    def ravel(self):
        return self.value.reshape(-1)

    def conj(self):
        return self.clone(value=torch.conj(self.value).resolve_conj())


def _binary(op, reverse=False):
    def fn(self, other):
        o = other.value if isinstance(other, BaseMeshField) else other
        v = op(o, self.value) if reverse else op(self.value, o)
        return self.clone(value=v)
    return fn


for _name, _op in [('__add__', operator.add), ('__sub__', operator.sub), ('__mul__', operator.mul),
                   ('__truediv__', operator.truediv), ('__pow__', operator.pow)]:
    setattr(BaseMeshField, _name, _binary(_op))
    setattr(BaseMeshField, '__r' + _name[2:], _binary(_op, reverse=True))
BaseMeshField.__neg__ = lambda self: self.clone(value=-self.value)
BaseMeshField.__abs__ = lambda self: self.clone(value=self.value.abs())


class RealMeshField(BaseMeshField):
    """Real-space mesh (``mesh.py:1962-2110``)."""

    @property
    def spacing(self):
        return self.cellsize

    def coords(self, kind='position', sparse=None):
        return self.attrs.rcoords(kind=kind, sparse=sparse)

    def r2c(self):
        return ComplexMeshField(_r2c(self.value, self.attrs.meshsize), attrs=self.attrs)

    def apply(self, fn, kind=Ellipsis, sparse=False):
        if kind is Ellipsis:
            kind = getattr(fn, 'kind', None)
        args = [self.value]
        if kind in ('index', 'position'):
            args.append(self.coords(kind=kind, sparse=sparse))
        elif kind is not None:
            raise ValueError('do not recognize kind = {}'.format(kind))
        value = fn(*args)
        return self.clone(value=value)

    def read(self, positions, resampler='cic', compensate=False, exchange=False, **kwargs):
        """Read the mesh at ``positions`` (``mesh.py:2030-2061``)."""
        if isinstance(positions, ParticleField):
            positions = positions.positions
        return _read(self, positions, resampler=resampler, compensate=compensate)


class ComplexMeshField(BaseMeshField):
    """Fourier-space mesh on the Hermitian layout (``mesh.py:2120-2196``)."""

    @property
    def spacing(self):
        return self.attrs.kfun

    @property
    def kfun(self):
        return self.attrs.kfun

    @property
    def knyq(self):
        return self.attrs.knyq

    def coords(self, kind='wavenumber', sparse=None):
        return self.attrs.kcoords(kind=kind, sparse=sparse)

    def c2r(self):
        return RealMeshField(_c2r(self.value, self.attrs.meshsize), attrs=self.attrs)

    def apply(self, fn, sparse=False, kind=Ellipsis):
        if kind is Ellipsis:
            kind = getattr(fn, 'kind', None)
        compensate_order = getattr(fn, 'compensate_order', None)
        if compensate_order is not None and kind == 'circular':
            # a resampler compensation window: fused CUDA pass
            out = torch.empty_like(self.value)
            _lib.call('pk_interlace_compensate', _lib.stream_handle(), _lib.ptr(self.value.contiguous()), 1,
                      _lib.i32(self.attrs.meshsize), int(compensate_order), self.attrs.backend_code, 0,
                      1., _lib.ptr(out))
            return self.clone(value=out)
        args = [self.value]
        if kind in ('circular', 'wavenumber'):
            args.append(self.coords(kind=kind, sparse=sparse))
        elif kind is not None:
            raise ValueError('do not recognize kind = {}'.format(kind))
        return self.clone(value=fn(*args))


def r2c(mesh):
    return mesh.r2c()


def c2r(mesh):
    return mesh.c2r()


def apply(mesh, fn, sparse=False, **kwargs):
    return mesh.apply(fn, sparse=sparse, **kwargs)


def read(mesh, positions, *args, **kwargs):
    return mesh.read(positions, *args, **kwargs)


def paint(particles, *args, **kwargs):
    return particles.paint(*args, **kwargs)


# ---------------------------------------------------------------------- particles

def _same_order(value, *args, **kwargs):
    return value


def _uniform_per_particle(seed, size, device):
    """Uniform [0, 1) float64 per particle for ``seed`` = int, (key, ids) or (key, 'index'), as
    ``create_sharded_random(jax.random.uniform, seed, size)`` draws them with x64 on
    (``mesh.py:237-329``), through ``pk_uniform_ids``."""
    key, ids = seed if isinstance(seed, tuple) else (seed, None)
    if key is None or not isinstance(key, (int, np.integer)):
        raise NotImplementedError('split seeds must be an integer key, optionally with ids')
    if isinstance(ids, str):
        if ids != 'index':
            raise ValueError('ids must be an array or \'index\'')
        ids = torch.arange(size, dtype=torch.int64, device=device)
    elif ids is not None:
        ids = ids if isinstance(ids, torch.Tensor) else torch.as_tensor(np.asarray(ids))
        ids = ids.to(device=device, dtype=torch.int64).reshape(-1).contiguous()
        if ids.numel() != size:
            raise ValueError('expected {} ids, got {}'.format(size, ids.numel()))
    out = torch.empty(size, dtype=torch.float64, device=device)
    _lib.call('pk_uniform_ids', _lib.stream_handle(), int(key) & 0xFFFFFFFFFFFFFFFF, _lib.ptr(ids), int(size),
              _lib.ptr(out))
    return out


def split_particles(*particles, seed=0, fields=None, return_masks=False):
    """Disjoint random subsamples for the normalisation (``split_particles``, ``mesh.py:3160-3204``).

    Particles sharing a field id (``fields``; a ``None`` entry repeats the previous particles)
    are split by one uniform draw per particle: subsample ``i`` of ``n`` keeps
    ``i / n <= x < (i + 1) / n`` (its weights multiplied by the mask).  ``seed``: one per unique
    field, each an integer or ``(integer, ids)`` with per-particle ids or ``'index'``.
    """
    if len(particles) == 1 and isinstance(particles[0], (tuple, list)):
        particles = tuple(particles[0])
    particles = list(particles)
    fields = [0] if fields is None else list(fields)
    for p in particles[len(fields):]:
        fields.append(fields[-1] if p is None else fields[-1] + 1)
    for i, (p, f) in enumerate(zip(particles, fields)):
        if p is None:
            particles[i] = particles[fields.index(f)]
    unique = []
    for f in fields:
        if f not in unique:
            unique.append(f)
    seeds = seed if isinstance(seed, list) else [seed]
    if len(seeds) != len(unique):
        raise ValueError('provide as many seeds as unique fields')
    out = [None] * len(particles) if return_masks else list(particles)
    for f, sd in zip(unique, seeds):
        idx = [i for i, ff in enumerate(fields) if ff == f]
        first = particles[idx[0]]
        x = _uniform_per_particle(sd, first.size, first.positions.device)
        nsplits = len(idx)
        for isplit, i in enumerate(idx):
            mask = (x >= isplit * 1. / nsplits) & (x < (isplit + 1) * 1. / nsplits)
            if return_masks:
                out[i] = mask
            else:
                out[i] = particles[i].clone(weights=(particles[i].weights * mask).to(torch.float32))
    return out


class ParticleField:
    """Particles with weights (``mesh.py:2398-2670``).

    ``exchange`` / ``backend`` are accepted for signature compatibility; a single
    GPU holds the whole catalog, so there is nothing to exchange.
    """

    def __init__(self, positions, weights=None, attrs=None, extra=None, exchange=False, backend='auto', **kwargs):
        if attrs is None:
            attrs = kwargs.pop('mattrs', None)
        if attrs is None:
            raise ValueError('attrs must be provided')
        if not isinstance(attrs, MeshAttrs):
            attrs = MeshAttrs(**dict(attrs))
        self.positions = _as_positions(positions)
        self._weights = _as_weights(weights, self.positions.shape[0])
        self.attrs = attrs
        self.extra = {k: torch.as_tensor(np.asarray(v) if not isinstance(v, torch.Tensor) else v).to(_device())
                      for k, v in (extra or {}).items()}
        # one GPU holds the whole catalog: particle-ordered arrays need no exchange
        self.exchange_direct = self.exchange_inverse = _same_order

    @property
    def weights(self):
        if self._weights is None:
            self._weights = torch.ones(self.positions.shape[0], dtype=torch.float32, device=self.positions.device)
        return self._weights

    @property
    def size(self):
        return self.positions.shape[0]

    def __repr__(self):
        return '{}(size={}, extra={})'.format(self.__class__.__name__, self.size, list(self.extra))

    def sum(self, *args, **kwargs):
        """Sum of weights."""
        if self._weights is None and not args and not kwargs:
            return torch.tensor(float(self.size), dtype=torch.float32, device=self.positions.device)
        return self.weights.sum(*args, **kwargs)

    def clone(self, **kwargs):
        kwargs.pop('exchange', None)
        kwargs.pop('backend', None)
        state = dict(positions=self.positions, weights=self._weights, attrs=self.attrs, extra=self.extra)
        state.update(kwargs)
        return self.__class__(**state)

    def exchange(self, **kwargs):
        return self.clone(**kwargs)

    def __getitem__(self, item):
        return self.clone(positions=self.positions[item], weights=self.weights[item],
                          extra={k: v[item] for k, v in self.extra.items()})

    @classmethod
    def concatenate(cls, others, weights=None, local=True, extra_weights=None, **kwargs):
        """Concatenate fields with factors on their weights (``mesh.py:2544-2578``)."""
        if weights is None:
            weights = [1] * len(others)
        positions = torch.cat([o.positions for o in others], dim=0)
        ws = []
        for o, f in zip(others, weights):
            fw = f if isinstance(f, torch.Tensor) else torch.tensor(float(f), device=o.positions.device)
            ws.append((fw.to(torch.float32) * o.weights).to(torch.float32))
        w = torch.cat(ws, dim=0)
        names = [n for n in others[0].extra if all(n in o.extra for o in others[1:])]
        extra = {n: torch.cat([o.extra[n] for o in others], dim=0) for n in names}
        return cls(positions, weights=w, attrs=others[0].attrs, extra=extra)

    def __add__(self, other):
        return self.concatenate([self, other], [1, 1])

    def __sub__(self, other):
        return self.concatenate([self, other], [1, -1])

    def __mul__(self, other):
        return self.concatenate([self], [other])

    __rmul__ = __mul__

    def __truediv__(self, other):
        return self.concatenate([self], [1. / other])

    def paint(self, resampler='cic', interlacing=0, compensate=False, out='real', dtype=None, **kwargs):
        """Paint to a mesh (``mesh.py:2604-2644`` → ``_paint``)."""
        attrs = self.attrs
        if dtype is not None:
            attrs = attrs.clone(dtype=dtype)
        return _paint(attrs, self.positions, self._weights, resampler=resampler, interlacing=interlacing,
                      compensate=compensate, out=out)


def _paint_call(attrs, positions, weights, order, interlacing, begin, count, out, status, config):
    """One pk_paint_batch launch sequence (a single catalog) with tile configuration ``config``."""
    n = positions.shape[0]
    shape = _lib.i32(attrs.meshsize)
    nbytes = _lib.c_size_t()
    _lib.call('pk_paint_batch_workspace_size', n, 1, shape, order, count, config, _lib.ctypes.byref(nbytes))
    ws = _workspace(nbytes.value)
    _lib.call('pk_paint_batch', _lib.stream_handle(), _lib.ptr(positions), _lib.ptr(weights), None, n, 1, shape,
              _lib.f32(attrs.boxsize), _lib.f32(attrs.boxcenter), _lib.f32(attrs.cellsize), order, interlacing, begin,
              count, config, _lib.ptr(out), _lib.ptr(ws), nbytes.value, _lib.ptr(status))


def _paint_config(attrs, positions, weights, order, interlacing, group, out, status):
    """Tile configuration of the paint pass, autotuned once per (mesh, order, shifts, N octave).

    Every configuration paints the same bits (the fixed-point scale depends on the catalog
    only), so the choice affects the speed alone.  Under CUDA graph capture nothing is timed:
    a tuned value is used when there is one, else configuration 0.
    """
    from .autotune import best_tile_config, make_key, cached_tile_config
    n = positions.shape[0]
    key = make_key('paint', tuple(int(s) for s in attrs.meshsize), order, group,
                   int(round(2. * math.log2(max(n, 2)))))
    if torch.cuda.is_current_stream_capturing():
        return cached_tile_config(key, default=0)
    return best_tile_config(key, lambda config: _paint_call(attrs, positions, weights, order, interlacing, 0, group,
                                                            out, status, config))


def _paint_shifts(attrs, positions, weights, order, interlacing, status=None):
    """All shifted real meshes, (I, N0, N1, N2) float32, through pk_paint_batch (≤ 4 shifts per launch)."""
    interlacing = max(int(interlacing), 1)
    shape = tuple(int(s) for s in attrs.meshsize)
    meshes = torch.empty((interlacing,) + shape, dtype=torch.float32, device=positions.device)
    group = min(interlacing, 4)
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=positions.device)
    config = _paint_config(attrs, positions, weights, order, interlacing, group, meshes[:group], status)
    for begin in range(0, interlacing, group):
        count = min(group, interlacing - begin)
        _paint_call(attrs, positions, weights, order, interlacing, begin, count, meshes[begin:begin + count], status,
                    config)
    return meshes, status


def _paint(attrs, positions, weights=None, resampler='cic', interlacing=0, compensate=False, out='real',
           halo_add=0, check=False):
    """``_paint`` (``mesh.py:2673-2754``) on the GPU.

    Paint every interlacing shift in one tiled pass, batched R2C, then one fused
    interlacing + compensation pass (which also folds the C2R normalisation).  With
    ``out='complex'`` that pass is deferred until the mesh's value is needed (a spectrum
    of the mesh is binned from the shifted meshes directly).
    """
    order = resamplers.get_resampler(resampler).order
    interlacing = max(int(interlacing), 1)
    positions = _as_positions(positions)
    weights = _as_weights(weights, positions.shape[0])
    meshsize = attrs.meshsize
    meshes, status = _paint_shifts(attrs, positions, weights, order, interlacing)
    if check and int(status.item()):
        raise ValueError('non-finite positions / weights, or positions far outside the box')
    if interlacing == 1 and not compensate:
        if out == 'real':
            return RealMeshField(meshes[0], attrs=attrs)
        return ComplexMeshField(_r2c(meshes[0], meshsize), attrs=attrs)
    cmeshes = _r2c(meshes, meshsize)
    del meshes
    if out != 'real':
        return _InterlacedComplexMeshField(cmeshes, attrs, order if compensate else 0)
    for_c2r = out == 'real'
    scale = float(np.float32(1. / np.prod(meshsize))) if for_c2r else 1.
    combined = torch.empty(cmeshes.shape[1:], dtype=torch.complex64, device=positions.device)
    _lib.call('pk_interlace_compensate', _lib.stream_handle(), _lib.ptr(cmeshes), interlacing,
              _lib.i32(meshsize), order if compensate else 0, attrs.backend_code, int(for_c2r),
              scale, _lib.ptr(combined))
    del cmeshes
    if for_c2r:
        return RealMeshField(_c2r(combined, meshsize, scale=False, destroy_input=True), attrs=attrs)
    return ComplexMeshField(combined, attrs=attrs)


class _InterlacedComplexMeshField(ComplexMeshField):
    """The complex mesh of ``paint(..., out='complex')`` with interlacing or compensation,
    kept as its interlaced, uncompensated shifted meshes until its value is needed.

    ``value`` forms the combined mesh (``pk_interlace_compensate``) on first access and
    keeps it; ``compute_mesh2_spectrum`` bins an untouched field straight from the shifted
    meshes (``pk_bin_global_interlaced``: the same numbers, without writing the combined
    mesh and reading it back).  Everything else sees an ordinary ``ComplexMeshField``.
    """

    def __init__(self, shifted, attrs, comp_order):
        self._shifted = shifted
        self._comp_order = int(comp_order)
        self._value = None
        self.attrs = attrs

    @property
    def value(self):
        if self._value is None:
            meshsize = self.attrs.meshsize
            combined = torch.empty(self._shifted.shape[1:], dtype=torch.complex64, device=self._shifted.device)
            _lib.call('pk_interlace_compensate', _lib.stream_handle(), _lib.ptr(self._shifted),
                      self._shifted.shape[0], _lib.i32(meshsize), self._comp_order, self.attrs.backend_code, 0,
                      1., _lib.ptr(combined))
            self._value = combined
            self._shifted = None
        return self._value

    @value.setter
    def value(self, v):
        self._value = v
        self._shifted = None

    @property
    def lazy(self):
        """(shifted meshes, compensation order) while the combined mesh is not formed, else None."""
        return None if self._shifted is None else (self._shifted, self._comp_order)

    def clone(self, **kwargs):
        if not kwargs or (set(kwargs) == {'attrs'} and kwargs['attrs'] is self.attrs):
            return self
        return ComplexMeshField(kwargs.pop('value', self.value), attrs=kwargs.pop('attrs', self.attrs)).clone(**kwargs)


def _read(mesh, positions, resampler='cic', compensate=False, halo_add=0):
    """``_read`` (``mesh.py:2064-2110``) on the GPU."""
    res = resamplers.get_resampler(resampler)
    if compensate:
        mesh = mesh.r2c().apply(res.compensate).c2r()
    attrs = mesh.attrs
    positions = _as_positions(positions)
    out = torch.empty(positions.shape[0], dtype=torch.float32, device=positions.device)
    value = mesh.value.contiguous()
    _lib.call('pk_read', _lib.stream_handle(), _lib.ptr(value), _lib.ptr(positions), None, positions.shape[0],
              _lib.i32(attrs.meshsize), _lib.f32(attrs.boxsize), _lib.f32(attrs.boxcenter),
              _lib.f32(attrs.cellsize), res.order, 0., 1., _lib.ptr(out), None, 0)
    return out


class FKPField:
    """FKP field: data minus alpha * randoms (``mesh.py:2913-2999``)."""

    def __init__(self, data, randoms, attrs=None):
        if attrs is not None:
            data = data.clone(attrs=attrs)
            randoms = randoms.clone(attrs=attrs)
        self.data = data
        self.randoms = randoms
        self._particles = None

    def clone(self, **kwargs):
        state = dict(data=self.data, randoms=self.randoms)
        state.update(kwargs)
        return self.__class__(**state)

    def exchange(self, **kwargs):
        return self.clone()

    @property
    def attrs(self):
        return self.data.attrs

    @property
    def alpha(self):
        return self.data.sum() / self.randoms.sum()

    @property
    def particles(self):
        if self._particles is None:
            self._particles = (self.data - self.alpha * self.randoms).clone(attrs=self.data.attrs)
        return self._particles

    def paint(self, resampler='cic', interlacing=1, compensate=False, dtype=None, out='real', **kwargs):
        return self.particles.paint(resampler=resampler, interlacing=interlacing, compensate=compensate,
                                    dtype=dtype, out=out, **kwargs)


# ---------------------------------------------------------------------- box helpers

@lru_cache(maxsize=32)
def next_fft_size(n, primes=(2, 3, 5, 7), divisors=()):
    """Smallest m >= n with prime factors in ``primes``, divisible by ``divisors`` (``mesh.py:2304-2340``)."""
    n = int(n)
    primes = tuple(p for p in primes if p > 1)
    divisors = tuple(int(d) for d in divisors if d > 1)
    D = 1
    for d in divisors:
        D = abs(D * d) // math.gcd(D, d)
    m = ((n + D - 1) // D) * D
    if not primes:
        return m
    while True:
        x = m
        for p in primes:
            while x % p == 0:
                x //= p
        if x == 1:
            return m
        m += D


def _extent(*positions):
    nonempty = [p for p in positions if p.shape[0]]
    if not nonempty:
        raise ValueError('<= 1 particles found; cannot infer boxsize')
    pmin = torch.stack([p.amin(dim=0) for p in nonempty]).amin(dim=0).cpu().numpy().astype('f4')
    pmax = torch.stack([p.amax(dim=0) for p in nonempty]).amax(dim=0).cpu().numpy().astype('f4')
    return pmin, pmax


def get_mesh_attrs(*positions, meshsize=None, boxsize=None, boxcenter=None, cellsize=None, boxpad=2.,
                   check=False, approximate=False, dtype=None, primes=None, divisors=None, **kwargs):
    """Enclosing box for positions (``mesh.py:2271-2381``)."""
    positions = [_as_positions(p) for p in positions]
    if cellsize is not None and meshsize is not None:
        if boxsize is not None:
            raise ValueError('cannot specify boxsize, cellsize and meshsize simultaneously')
        boxsize = _fill3(meshsize, 'i4') * _fill3(cellsize, 'f4')
    if boxsize is None or boxcenter is None or (positions and check):
        if not positions:
            raise ValueError('positions must be provided if boxsize and boxcenter are not specified, or check is True')
        pmin, pmax = _extent(*positions)
        delta = np.abs(pmax - pmin)
        if boxcenter is None:
            boxcenter = (np.float32(0.5) * (pmin + pmax)).astype('f4')
        if boxsize is None:
            boxsize = np.float32(delta.max() * np.float32(boxpad))
        if check and np.any(_fill3(boxsize, 'f4') < delta):
            raise ValueError('boxsize {} too small to contain all data (max {})'.format(boxsize, delta))
    boxsize = _fill3(boxsize, 'f4')
    if meshsize is None:
        if cellsize is None:
            raise ValueError('meshsize (or cellsize) must be specified')
        cellsize = _fill3(cellsize, 'f4')
        meshsize = np.ceil((boxsize / cellsize).astype('f4')).astype('i4')
        primes = tuple(primes or ())
        if not divisors or np.ndim(divisors[0]) == 0:
            divisors = [tuple(divisors or ())] * 3
        meshsize = np.array([next_fft_size(m, primes=primes, divisors=tuple(d)) for m, d in zip(meshsize, divisors)])
        newbox = (meshsize * cellsize).astype('f4')
        if not positions and not approximate and not np.allclose(newbox, boxsize):
            raise ValueError('cannot enforce cellsize = {} with meshsize = {}, as it would lead to boxsize = {} != '
                             'input boxsize = {}'.format(cellsize, meshsize, newbox, boxsize))
        boxsize = newbox
    kwargs.pop('sharding_mesh', None)
    return MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=boxcenter, **kwargs)
