"""Power-spectrum result containers (the layout of lsstypes' ``Mesh2SpectrumPole(s)``).

jax-power returns lsstypes objects (``types.py:93-94``); lsstypes is an external,
unpinned dependency.  This module keeps the fields the estimator fills
(``mesh2.py:341-344, 371-374``) — ``k``, ``k_edges``, ``nmodes``, ``num_raw``,
``num_shotnoise``, ``norm``, ``volume``, ``ell``, ``attrs`` — and the methods the
reference's tests use: ``value()`` = (num_raw - num_shotnoise) / norm (the
normalisation that reproduces the reference's golden ``value().std()``),
``clone(norm=..., num_shotnoise=...)``, ``get(ells=...)``, ``values(name)``,
``coords('k')``, ``ells``.  Arrays are NumPy float64 on the host.  ``num_raw`` may be given
as a deferred value (``DeferredRows``): the estimator's per-bin sums stay on the device and
are read back, once for all multipoles, when ``num_raw`` is first used, so that computing a
spectrum does not wait for the GPU (as JAX arrays do not).  ``Mesh2SpectrumPoles.prefetch()``
starts that read-back on a side stream, so that reading a spectrum after enqueuing the next
one waits only for the first.

On disk (``write`` / ``read``, the names lsstypes exports and ``types.py:5-7`` re-exports):
lsstypes' own HDF5 layout is not available here (neither lsstypes nor h5py is installed),
so an observable is stored as one NumPy ``.npz`` archive of its state: the class name, the
multipoles, and per pole every field, ``ell`` and ``attrs`` (as JSON).  ``read`` gives back
an object equal field for field.
"""
import json

import numpy as np

__all__ = ['Mesh2SpectrumPole', 'Mesh2SpectrumPoles', 'Mesh2CorrelationPole', 'Mesh2CorrelationPoles',
           'WindowMatrix', 'DeferredRows', 'read', 'write']


class DeferredRows:
    """Rows of a device tensor of per-bin sums, read back to the host on first use.

    ``row(i)`` gives a deferred row: ``scale[i] * sums[i] / divisor`` in float64, computed
    on the host from the one read-back of the whole tensor that all rows share.
    """

    def __init__(self, sums, divisor, scales):
        self._sums = sums
        self._host = None
        self._pending = None
        self._divisor = np.asarray(divisor, dtype='f8')
        self._scales = list(scales)
        self.shape = tuple(sums.shape[1:])

    def prefetch(self):
        """Start the read-back now: a copy into pinned host memory on a side stream that waits
        only for the sums, so that a later read waits for that copy, not for the work the caller
        has enqueued since (e.g. the next spectrum)."""
        if self._host is not None or self._pending is not None or not getattr(self._sums, 'is_cuda', False):
            return
        import torch
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream(self._sums.device))  # the sums' device, whichever is current
        stream = _readback_stream(self._sums.device)
        host = torch.empty(self._sums.shape, dtype=self._sums.dtype, pin_memory=True)
        with torch.cuda.stream(stream):
            stream.wait_event(ready)
            host.copy_(self._sums, non_blocking=True)
            done = torch.cuda.Event()
            done.record(stream)
        self._sums.record_stream(stream)
        self._pending = (host, done)

    def _read(self):
        if self._host is None:
            if self._pending is not None:
                host, done = self._pending
                done.synchronize()
                self._host = host.numpy()
                self._pending = None
            else:
                self._host = self._sums.cpu().numpy()
            self._sums = None
        return self._host

    def row(self, i):
        return _DeferredRow(self, i)


_READBACK_STREAMS = {}


def _readback_stream(device):
    import torch
    key = torch.device(device).index
    if key not in _READBACK_STREAMS:
        _READBACK_STREAMS[key] = torch.cuda.Stream(device=device)
    return _READBACK_STREAMS[key]


class _DeferredRow:

    def __init__(self, rows, i):
        self.rows, self.i, self.shape = rows, i, rows.shape

    def get(self):
        r = self.rows
        return r._read()[self.i] / r._divisor * r._scales[self.i]


class Mesh2SpectrumPole:

    _fields = ('k', 'k_edges', 'nmodes', 'num_raw', 'num_shotnoise', 'norm', 'volume')

    def __init__(self, k, k_edges, nmodes, num_raw, num_shotnoise=None, norm=None, volume=None, ell=0,
                 attrs=None):
        self.k = np.asarray(k, dtype='f8')
        self.k_edges = np.asarray(k_edges, dtype='f8')
        self.nmodes = np.asarray(nmodes, dtype='f8')
        if isinstance(num_raw, _DeferredRow):
            self._num_raw, self._deferred = None, num_raw
            shape = num_raw.shape
            if num_shotnoise is None or norm is None:
                shape = self.num_raw.shape  # zeros_like / ones_like need the values' type
        else:
            self._num_raw, self._deferred = np.asarray(num_raw), None
            shape = self._num_raw.shape
        self.num_shotnoise = np.zeros_like(self.num_raw) if num_shotnoise is None else \
            np.broadcast_to(np.asarray(num_shotnoise), shape).copy()
        self.norm = np.ones_like(self.num_raw, dtype='f8') if norm is None else \
            np.broadcast_to(np.asarray(norm, dtype='f8'), shape).copy()
        self.volume = volume
        self.ell = int(ell)
        self.attrs = dict(attrs or {})

    @property
    def num_raw(self):
        if self._num_raw is None:
            self._num_raw = np.asarray(self._deferred.get())
            self._deferred = None
        return self._num_raw

    @num_raw.setter
    def num_raw(self, value):
        self._num_raw, self._deferred = np.asarray(value), None

    def value(self):
        return (self.num_raw - self.num_shotnoise) / self.norm

    def coords(self, name='k'):
        return getattr(self, name)

    def values(self, name='value'):
        if name == 'value':
            return self.value()
        if name == 'shotnoise':
            return self.num_shotnoise / self.norm
        return getattr(self, name)

    def clone(self, **kwargs):
        state = {name: getattr(self, name) for name in self._fields}
        state.update(ell=self.ell, attrs=self.attrs)
        state.update(kwargs)
        return self.__class__(**state)

    def __repr__(self):
        return 'Mesh2SpectrumPole(ell={}, nbins={})'.format(self.ell, self.k.size)

    def state(self):
        state = {name: getattr(self, name) for name in self._fields}
        state.update(ell=self.ell, attrs=self.attrs)
        return state

    @classmethod
    def from_state(cls, state):
        return cls(**state)

    def write(self, filename):
        write(filename, self)


class Mesh2SpectrumPoles:

    def __init__(self, poles):
        self.poles = list(poles)

    @property
    def ells(self):
        return tuple(p.ell for p in self.poles)

    @property
    def wa_orders(self):
        """Wide-angle order of each pole (``attrs['wa_order']``, 0 when absent): the theory side
        of a first-point window matrix (the reference's ``wa_orders`` label)."""
        return tuple(int(p.attrs.get('wa_order', 0)) for p in self.poles)

    def __iter__(self):
        return iter(self.poles)

    def __len__(self):
        return len(self.poles)

    def _index(self, ell, wa_order):
        keys = list(zip(self.ells, self.wa_orders))
        if wa_order is None:
            return self.ells.index(int(ell))
        return keys.index((int(ell), int(wa_order)))

    def get(self, ells=None, ell=None, wa_orders=None):
        if ells is None:
            ells = ell
        if ells is None:
            return self
        if np.ndim(ells) == 0:
            return self.poles[self._index(ells, wa_orders)]
        was = [None] * len(ells) if wa_orders is None else (list(wa_orders) if np.ndim(wa_orders) else
                                                            [wa_orders] * len(ells))
        return self.__class__([self.poles[self._index(e, w)] for e, w in zip(ells, was)])

    def value(self):
        return np.concatenate([p.value() for p in self.poles])

    def prefetch(self):
        """Start reading back the multipoles still on the device (see ``DeferredRows.prefetch``);
        returns self."""
        for p in self.poles:
            deferred = getattr(p, '_deferred', None)
            if deferred is not None:
                deferred.rows.prefetch()
        return self

    def clone(self, **kwargs):
        """Per-pole update; list values (one per ell) are dispatched, scalars broadcast."""
        poles = []
        for i, p in enumerate(self.poles):
            kw = {k: (v[i] if isinstance(v, (list, tuple)) else v) for k, v in kwargs.items()}
            poles.append(p.clone(**kw))
        return self.__class__(poles)

    def __repr__(self):
        return 'Mesh2SpectrumPoles(ells={})'.format(self.ells)

    def write(self, filename):
        write(filename, self)


class Mesh2CorrelationPole(Mesh2SpectrumPole):
    """Correlation-function multipole: ``s``, ``s_edges`` in place of ``k``, ``k_edges``."""

    _fields = ('s', 's_edges', 'nmodes', 'num_raw', 'num_shotnoise', 'norm', 'volume')

    def __init__(self, s, s_edges, nmodes, num_raw, num_shotnoise=None, norm=None, volume=None, ell=0,
                 attrs=None):
        super().__init__(s, s_edges, nmodes, num_raw, num_shotnoise=num_shotnoise, norm=norm, volume=volume,
                         ell=ell, attrs=attrs)
        self.s, self.s_edges = self.k, self.k_edges

    def coords(self, name='s'):
        return getattr(self, name)

    def __repr__(self):
        return 'Mesh2CorrelationPole(ell={}, nbins={})'.format(self.ell, self.s.size)


class Mesh2CorrelationPoles(Mesh2SpectrumPoles):

    def __repr__(self):
        return 'Mesh2CorrelationPoles(ells={})'.format(self.ells)


class WindowMatrix:
    """Window matrix (the lsstypes ``WindowMatrix`` built at ``mesh2.py:1462-1482``).

    ``value`` (observable size, theory size) maps the theory multipoles, flattened ell by ell,
    to the binned multipoles: ``observable`` (``Mesh2SpectrumPoles`` on the output k bins,
    ``norm`` the window's normalisation, ``num_raw`` zero) and ``theory`` (one
    ``Mesh2SpectrumPole`` per input ell on the input k edges, ``k`` their mid-points).
    """

    def __init__(self, observable, theory, value):
        self.observable = observable
        self.theory = theory
        self.value = np.asarray(value)

    @property
    def shape(self):
        return self.value.shape

    def dot(self, theory):
        """``value @ theory``, the theory given as a flat vector or one array per input ell."""
        if not isinstance(theory, np.ndarray) or theory.ndim != 1:
            theory = np.concatenate([np.ravel(t) for t in theory])
        return self.value.dot(theory)

    def write(self, filename):
        write(filename, self)

    def __repr__(self):
        return 'WindowMatrix(shape={}, ells={}, ellsin={})'.format(self.shape, self.observable.ells,
                                                                   self.theory.ells)


_CLASSES = {cls.__name__: cls for cls in (Mesh2SpectrumPole, Mesh2SpectrumPoles, Mesh2CorrelationPole,
                                          Mesh2CorrelationPoles, WindowMatrix)}
_POLE_OF = {'Mesh2SpectrumPoles': Mesh2SpectrumPole, 'Mesh2CorrelationPoles': Mesh2CorrelationPole}


def _pole_arrays(prefix, pole):
    out = {}
    for name, value in pole.state().items():
        if name == 'attrs':
            out[prefix + 'attrs'] = np.array(json.dumps(value, default=lambda o: np.asarray(o).tolist()))
        elif value is None:
            out[prefix + name + '.none'] = np.array(True)
        else:
            out[prefix + name] = np.asarray(value)
    return out


def _pole_state(prefix, archive):
    state = {}
    for key in archive.files:
        if not key.startswith(prefix):
            continue
        name = key[len(prefix):]
        if name == 'attrs':
            state['attrs'] = json.loads(str(archive[key]))
        elif name.endswith('.none'):
            state[name[:-len('.none')]] = None
        elif name == 'ell':
            state['ell'] = int(archive[key])
        elif name == 'volume':
            state['volume'] = archive[key][()] if archive[key].ndim == 0 else archive[key]
        else:
            state[name] = archive[key]
    return state


def write(filename, observable):
    """Save a (list of) multipole(s) to ``filename`` (NumPy ``.npz``)."""
    name = type(observable).__name__
    if name not in _CLASSES:
        raise TypeError('cannot write {}'.format(type(observable)))
    arrays = {'__class__': np.array(name)}
    if isinstance(observable, WindowMatrix):
        arrays['value'] = observable.value
        for part in ('observable', 'theory'):
            poles = getattr(observable, part)
            arrays['{}/npoles'.format(part)] = np.array(len(poles))
            for i, pole in enumerate(poles):
                arrays.update(_pole_arrays('{}/pole{:d}/'.format(part, i), pole))
    elif isinstance(observable, Mesh2SpectrumPoles):
        arrays['__npoles__'] = np.array(len(observable))
        for i, pole in enumerate(observable):
            arrays.update(_pole_arrays('pole{:d}/'.format(i), pole))
    else:
        arrays.update(_pole_arrays('pole/', observable))
    with open(filename, 'wb') as f:
        np.savez(f, **arrays)


def read(filename):
    """Load what ``write`` saved."""
    with np.load(filename, allow_pickle=False) as archive:
        name = str(archive['__class__'])
        if name == 'WindowMatrix':
            parts = [Mesh2SpectrumPoles([Mesh2SpectrumPole.from_state(_pole_state('{}/pole{:d}/'.format(part, i), archive))
                                         for i in range(int(archive['{}/npoles'.format(part)]))])
                     for part in ('observable', 'theory')]
            return WindowMatrix(*parts, value=archive['value'])
        if name in _POLE_OF:
            pole_cls = _POLE_OF[name]
            poles = [pole_cls.from_state(_pole_state('pole{:d}/'.format(i), archive))
                     for i in range(int(archive['__npoles__']))]
            return _CLASSES[name](poles)
        return _CLASSES[name].from_state(_pole_state('pole/', archive))
