"""Power-spectrum binning and estimators (host side of the CUDA library).

Mirrors ``jaxpower/mesh2.py``:

- ``BinMesh2SpectrumPoles`` (``mesh2.py:25-119``): k edges (``np.arange(0, k_Nyq, step)``
  in float64, compared in float32), nmodes and xavg computed on the GPU by
  ``pk_bin_modes``; the per-mode bin index is never materialised;
- ``compute_mesh2_spectrum`` (``mesh2.py:253-374``): global line of sight through
  ``pk_bin_global``; first-point / endpoint through ``pk_ylm_premultiply`` +
  batched cuFFT R2C + ``pk_bin_firstpoint`` (sum over m done inside the binning
  pass: bin is linear, so sum_m bin(.) = bin(sum_m .));
- ``compute_fkp2_normalization`` / ``compute_fkp2_shotnoise`` /
  ``compute_box2_normalization`` (``mesh2.py:508-621``).
"""
import functools
import itertools
import math

import numpy as np
import torch

from . import _lib
from .mesh import (MeshAttrs, BaseMeshField, RealMeshField, ComplexMeshField, ParticleField, FKPField,
                   _r2c, _c2r, _workspace, _device, _paint, get_mesh_attrs, split_particles)
from .types import Mesh2SpectrumPole, Mesh2SpectrumPoles, Mesh2CorrelationPole, Mesh2CorrelationPoles, DeferredRows

__all__ = ['BinMesh2SpectrumPoles', 'compute_mesh2_spectrum', 'compute_mesh2', 'compute_fkp2_normalization',
           'compute_fkp2_shotnoise', 'compute_box2_normalization', 'compute_normalization',
           'compute_box_normalization', 'compute_mesh2_spectrum_window', 'compute_mesh2_spectrum_mean',
           'compute_smooth2_spectrum_window']


def _plain_bins(bin, what):
    """Paths whose fused kernels bin each mode once (the fixed line-of-sight window and mean
    spectrum, the batched runner) reject mode oversampling."""
    if getattr(bin, '_kshifts', None):
        raise NotImplementedError('{} does not support mode_oversampling > 0'.format(what))


def _format_ells(ells):
    if np.ndim(ells) == 0:
        ells = (ells,)
    return tuple(sorted(int(e) for e in ells))


def _uniform_step(edges):
    if len(edges) < 2:
        return 0.
    d = np.diff(edges)
    if np.all(d > 0) and np.max(np.abs(d - d.mean())) <= 1e-3 * d.mean():
        return float(d.mean())
    return 0.


class BinMesh2SpectrumPoles:
    """Binning operator for mesh to power spectrum (``mesh2.py:67-119``).

    Parameters
    ----------
    mattrs : MeshAttrs or mesh field
    edges : array, dict ('min', 'max', 'step') or None
    ells : int or tuple
    mode_oversampling : int s >= 0; s > 0 bins the modes once per integer shift in [-s, s]^3
        by |k + shift| (the shift added to each k coordinate as the reference adds it,
        ``mesh2.py:48-61``) and averages: nmodes is the mean over the shifts, xavg the sum of
        the per-shift sums of |k + shift| divided by that mean (the reference's expression),
        and binned values the mean of the per-shift sums over nmodes (``mesh.py:2876-2910``).
    """

    def __init__(self, mattrs, edges=None, ells=0, mode_oversampling=0):
        if not isinstance(mattrs, MeshAttrs):
            mattrs = mattrs.attrs
        mode_oversampling = int(mode_oversampling)
        if mode_oversampling < 0:
            raise ValueError('mode_oversampling must be >= 0')
        self.mode_oversampling = mode_oversampling
        r = range(-mode_oversampling, mode_oversampling + 1)
        self._kshifts = [tuple(float(v) for v in sh) for sh in itertools.product(r, r, r)] if mode_oversampling else []
        self.mattrs = mattrs
        self.ells = _format_ells(ells)
        vec0 = np.float32(mattrs.kfun.min())
        if edges is None:
            edges = {}
        if isinstance(edges, dict):
            step = edges.get('step', None)
            vecmax = np.float32(np.float32(vec0 * np.float32(np.min(mattrs.meshsize))) / np.float32(2.))
            if step is None:
                edges = self._find_unique_edges(vec0, edges.get('min', 0.), edges.get('max', np.inf))
            else:
                edges = np.arange(edges.get('min', 0.), edges.get('max', float(vecmax)), step)
        edges = np.asarray(edges, dtype='f8')
        if edges.ndim == 2:
            edges = np.append(edges[:, 0], edges[-1, 1])
        self._edges1d = edges
        self.edges = np.column_stack([edges[:-1], edges[1:]])
        self._step = _uniform_step(edges.astype('f4'))
        self.d_edges = torch.as_tensor(edges.astype('f4'), device=_device())
        nbins = len(edges) - 1
        nmodes = torch.empty(nbins, dtype=torch.float64, device=_device())
        ksum = torch.empty(nbins, dtype=torch.float64, device=_device())
        ws = self._workspace()
        if self._kshifts:
            for ish, sh in enumerate(self._kshifts):
                _lib.call('pk_bin_modes_shifted', _lib.stream_handle(), _lib.i32(mattrs.meshsize),
                          _lib.f32(mattrs.kfun), _lib.f32(sh), _lib.ptr(self.d_edges), len(edges), self._step,
                          mattrs.backend_code, int(ish > 0), _lib.ptr(nmodes), _lib.ptr(ksum), _lib.ptr(ws),
                          ws.numel())
        else:
            _lib.call('pk_bin_modes', _lib.stream_handle(), _lib.i32(mattrs.meshsize), _lib.f32(mattrs.kfun),
                      _lib.ptr(self.d_edges), len(edges), self._step, mattrs.backend_code, _lib.ptr(nmodes),
                      _lib.ptr(ksum), _lib.ptr(ws), ws.numel())
        self.nmodes = nmodes.cpu().numpy() / max(len(self._kshifts), 1)  # mean over the shifts, an IEEE division
        with np.errstate(invalid='ignore', divide='ignore'):
            self.xavg = ksum.cpu().numpy() / self.nmodes

    def _workspace(self):
        nbytes = _lib.c_size_t()
        _lib.call('pk_bin_workspace_size', _lib.i32(self.mattrs.meshsize), len(self._edges1d), 9,
                  _lib.ctypes.byref(nbytes))
        return _workspace(nbytes.value)

    def _find_unique_edges(self, x0, xmin=0., xmax=np.inf):
        """``_find_unique_edges`` (``mesh.py:2789-2811``): mid-points between unique |k|."""
        kx, ky, kz = self.mattrs.kcoords(sparse=True)
        x2 = ((kx * kx + ky * ky) + kz * kz).reshape(-1)
        x2 = x2[(x2 >= xmin**2) & (x2 <= xmax**2)]
        key = (x2.double() / (0.5 * float(x0))**2 + 0.5).to(torch.int64)
        _, inverse = torch.unique(key, return_inverse=True)
        first = torch.full((int(inverse.max()) + 1,), x2.numel(), dtype=torch.int64, device=x2.device)
        first.scatter_reduce_(0, inverse, torch.arange(x2.numel(), device=x2.device), reduce='amin')
        x = torch.sqrt(x2[first]).cpu().numpy().astype('f8')
        tmp = (x[:-1] + x[1:]) / 2.
        return np.concatenate([[tmp[0] - (x[1] - x[0])], tmp, [tmp[-1] + (x[-1] - x[-2])]])

    @property
    def nbins(self):
        return len(self._edges1d) - 1

    @property
    def wmodes(self):
        kz = self.mattrs.kcoords(sparse=True)[2]
        n2 = int(self.mattrs.meshsize[2])
        if self.mattrs.fft_backend == 'jax':
            w = 1 + (kz > 0).to(torch.int32)
        else:
            z = torch.arange(kz.numel(), device=kz.device).reshape(kz.shape)
            w = 2 - ((z == 0) | ((n2 % 2 == 0) & (z == n2 // 2))).to(torch.int32)
        return w.expand(tuple(self.mattrs.meshsize[:2]) + (n2 // 2 + 1,))

    def __call__(self, mesh, remove_zero=False):
        """Per-bin mean of a complex mesh with Hermitian weights (``mesh2.py:100-119``)."""
        value = mesh.value if isinstance(mesh, BaseMeshField) else mesh
        if not isinstance(value, torch.Tensor):
            value = torch.as_tensor(np.asarray(value))
        value = value.to(device=_device(), dtype=torch.complex64).contiguous()
        out = torch.empty(2 * self.nbins, dtype=torch.float64, device=value.device)
        ws = self._workspace()
        if self._kshifts:
            for ish, sh in enumerate(self._kshifts):
                _lib.call('pk_bin_mesh_shifted', _lib.stream_handle(), _lib.ptr(value), _lib.i32(self.mattrs.meshsize),
                          _lib.f32(self.mattrs.kfun), _lib.f32(sh), _lib.ptr(self.d_edges), len(self._edges1d),
                          self._step, self.mattrs.backend_code, int(bool(remove_zero)), int(ish > 0), _lib.ptr(out),
                          _lib.ptr(ws), ws.numel())
            out /= len(self._kshifts)
        else:
            _lib.call('pk_bin_mesh', _lib.stream_handle(), _lib.ptr(value), _lib.i32(self.mattrs.meshsize),
                      _lib.f32(self.mattrs.kfun), _lib.ptr(self.d_edges), len(self._edges1d), self._step,
                      self.mattrs.backend_code, int(bool(remove_zero)), _lib.ptr(out), _lib.ptr(ws), ws.numel())
        out = out.cpu().numpy()
        return (out[:self.nbins] + 1j * out[self.nbins:]) / self.nmodes


class BinMesh2CorrelationPoles:
    """Binning operator for mesh to correlation function (``mesh2.py:124-192``).

    Separations are the real-space grid ``fftfreq(n) * cellsize * n`` of the full mesh
    (``mesh.py:1590-1603``, kind 'separation'), every cell with unit weight; bins of |s|
    (exact |s|^2 thresholds on the GPU).

    Parameters
    ----------
    mattrs : MeshAttrs or mesh field
    edges : array, dict ('min', 'max' (default cellsize * min(meshsize) / 2), 'step') or None
    ells : int or tuple
    mode_oversampling : int s >= 0; s > 0 bins the separations once per integer shift in
        [-s, s]^3 by |s + shift| and averages, as ``BinMesh2SpectrumPoles`` does for k
    basis : None (bins of |s| on the separation grid) or 'bessel': the estimator's Fourier-space
        mode values projected on j_ell(|k| s) at each bin's mean separation (``mesh2.py:169-181``;
        ``pk_bin_bessel``)
    klimit : None, True ((0, k_Nyq)) or (kmin, kmax): modes kept in the Bessel projection
    batch_size : accepted for the reference's signature (its ``lax.map`` batching); unused
    """

    def __init__(self, mattrs, edges=None, ells=0, mode_oversampling=0, basis=None, klimit=None, batch_size=None):
        if not isinstance(mattrs, MeshAttrs):
            mattrs = mattrs.attrs
        mode_oversampling = int(mode_oversampling)
        if mode_oversampling < 0:
            raise ValueError('mode_oversampling must be >= 0')
        r = range(-mode_oversampling, mode_oversampling + 1)
        self._sshifts = [tuple(float(v) for v in sh) for sh in itertools.product(r, r, r)] if mode_oversampling else []
        if self._sshifts and basis == 'bessel':
            raise NotImplementedError("mode_oversampling > 0 with basis='bessel' is not supported")
        if basis not in (None, 'bessel'):
            raise ValueError('unknown basis {}'.format(basis))
        self.mattrs = mattrs
        self.ells = _format_ells(ells)
        self.basis = basis
        if isinstance(klimit, bool):
            klimit = (0., float(np.min(mattrs.knyq))) if klimit else None
        self.klimit = None if klimit is None else tuple(float(k) for k in klimit)
        self.batch_size = batch_size
        vec0 = np.float32(mattrs.cellsize.min())
        if edges is None:
            edges = {}
        if isinstance(edges, dict):
            step = edges.get('step', None)
            vecmax = np.float32(np.float32(vec0 * np.float32(np.min(mattrs.meshsize))) / np.float32(2.))
            if step is None:
                edges = self._find_unique_edges(vec0, edges.get('min', 0.), edges.get('max', np.inf))
            else:
                edges = np.arange(edges.get('min', 0.), edges.get('max', float(vecmax)), step)
        edges = np.asarray(edges, dtype='f8')
        if edges.ndim == 2:
            edges = np.append(edges[:, 0], edges[-1, 1])
        self._edges1d = edges
        self.edges = np.column_stack([edges[:-1], edges[1:]])
        self._step = _uniform_step(edges.astype('f4'))
        self.d_edges = torch.as_tensor(edges.astype('f4'), device=_device())
        nbins = len(edges) - 1
        nmodes = torch.empty(nbins, dtype=torch.float64, device=_device())
        ssum = torch.empty(nbins, dtype=torch.float64, device=_device())
        ws = self._workspace()
        if self._sshifts:  # mesh2.py:48-61: nmodes averaged over the shifts, xavg the summed |s + shift| over it
            for ish, sh in enumerate(self._sshifts):
                _lib.call('pk_bin_separation_modes_shifted', _lib.stream_handle(), _lib.i32(mattrs.meshsize),
                          _lib.f32(mattrs.cellsize), _lib.f32(sh), _lib.ptr(self.d_edges), len(edges), self._step,
                          int(ish > 0), _lib.ptr(nmodes), _lib.ptr(ssum), _lib.ptr(ws), ws.numel())
        else:
            _lib.call('pk_bin_separation_modes', _lib.stream_handle(), _lib.i32(mattrs.meshsize),
                      _lib.f32(mattrs.cellsize), _lib.ptr(self.d_edges), len(edges), self._step, _lib.ptr(nmodes),
                      _lib.ptr(ssum), _lib.ptr(ws), ws.numel())
        self.nmodes = nmodes.cpu().numpy() / max(len(self._sshifts), 1)  # mean over the shifts, an IEEE division
        with np.errstate(invalid='ignore', divide='ignore'):
            self.xavg = ssum.cpu().numpy() / self.nmodes

    def _workspace(self):
        nbytes = _lib.c_size_t()
        _lib.call('pk_bin_separation_workspace_size', _lib.i32(self.mattrs.meshsize), len(self._edges1d), 3,
                  _lib.ctypes.byref(nbytes))
        return _workspace(nbytes.value)

    def _find_unique_edges(self, x0, xmin=0., xmax=np.inf):
        """``_find_unique_edges`` (``mesh.py:2789-2811``): mid-points between unique |s|."""
        sx, sy, sz = self.mattrs.rcoords(kind='separation', sparse=True)
        x2 = ((sx * sx + sy * sy) + sz * sz).reshape(-1)
        x2 = x2[(x2 >= xmin**2) & (x2 <= xmax**2)]
        key = (x2.double() / (0.5 * float(x0))**2 + 0.5).to(torch.int64)
        _, inverse = torch.unique(key, return_inverse=True)
        first = torch.full((int(inverse.max()) + 1,), x2.numel(), dtype=torch.int64, device=x2.device)
        first.scatter_reduce_(0, inverse, torch.arange(x2.numel(), device=x2.device), reduce='amin')
        x = torch.sqrt(x2[first]).cpu().numpy().astype('f8')
        tmp = (x[:-1] + x[1:]) / 2.
        return np.concatenate([[tmp[0] - (x[1] - x[0])], tmp, [tmp[-1] + (x[-1] - x[-2])]])

    @property
    def nbins(self):
        return len(self._edges1d) - 1

    def _sums(self, value, ells, los=(0., 0., 1.)):
        value = value.to(device=_device(), dtype=torch.float32).contiguous()
        out = torch.empty(len(ells) * self.nbins, dtype=torch.float64, device=value.device)
        ws = self._workspace()
        if self._sshifts:  # the mean over the shifted binnings (mesh.py:2894-2895)
            for ish, sh in enumerate(self._sshifts):
                _lib.call('pk_bin_separation_global_shifted', _lib.stream_handle(), _lib.ptr(value),
                          _lib.i32(self.mattrs.meshsize), _lib.f32(self.mattrs.cellsize), _lib.f32(sh), _lib.f32(los),
                          _lib.ptr(self.d_edges), len(self._edges1d), self._step, len(ells), _lib.i32(ells),
                          int(ish > 0), _lib.ptr(out), _lib.ptr(ws), ws.numel())
            return out.reshape(len(ells), self.nbins) / len(self._sshifts)
        _lib.call('pk_bin_separation_global', _lib.stream_handle(), _lib.ptr(value), _lib.i32(self.mattrs.meshsize),
                  _lib.f32(self.mattrs.cellsize), _lib.f32(los), _lib.ptr(self.d_edges), len(self._edges1d),
                  self._step, len(ells), _lib.i32(ells), _lib.ptr(out), _lib.ptr(ws), ws.numel())
        return out.reshape(len(ells), self.nbins)

    def __call__(self, mesh, ell=0, remove_zero=False):
        """Per-bin mean of a real mesh (``mesh2.py:162-192``, configuration-space basis)."""
        value = mesh.value if isinstance(mesh, BaseMeshField) else mesh
        if not isinstance(value, torch.Tensor):
            value = torch.as_tensor(np.asarray(value))
        if remove_zero:
            value = value.clone()
            value.view(-1)[0] = 0.
        return self._sums(value, (0,))[0].cpu().numpy() / self.nmodes


def compute_mesh2_correlation(*meshes, bin=None, los='z'):
    """Correlation-function multipoles from mesh(es) (``mesh2.py:377-504``).

    Fixed line of sight: A = c2r(|delta_k|^2) (or c2r(conj(delta1_k) delta2_k));
    xi_ell = (2 ell + 1) <A L_ell(mu)> per |s| bin (the s = 0 cell dropped for ell > 0).
    First point: xi_0 = <c2r(|A0|^2)>, xi_ell = 4 pi <sum_m c2r(conj(r2c(rho Y_lm(xhat))) A0)
    Y_lm(shat)> (s = 0 dropped).  num_raw = xi_ell / V_cell.
    """
    meshes, fields = _format_meshes(*meshes)
    mattrs = meshes[0].attrs
    norm_value = np.float32(np.prod(mattrs.meshsize.astype('f4'))) / np.float32(np.prod(mattrs.cellsize))
    los_name, vlos, swap = _los(los)
    ells = bin.ells
    meshsize = mattrs.meshsize
    auto = fields[1] == fields[0]

    def _c(mesh):
        return mesh.value if isinstance(mesh, ComplexMeshField) else _r2c(mesh.value, meshsize)

    def _r(mesh):
        return mesh.value if isinstance(mesh, RealMeshField) else _c2r(mesh.value, meshsize)

    if bin.basis == 'bessel':
        return _bessel_correlation(meshes, auto, bin, los_name, vlos, swap, norm_value)

    if vlos is None:  # first point (end point: the meshes swapped), mesh2.py:414-463
        if swap and not auto:
            meshes = meshes[::-1]
        A0 = _c(meshes[0] if auto else meshes[1]).contiguous()
        sums = {}
        if 0 in ells:
            if auto:
                prod = (A0.real * A0.real + A0.imag * A0.imag).to(torch.complex64)
            else:
                prod = torch.conj(_c(meshes[0])) * A0
            sums[0] = bin._sums(_c2r(prod.contiguous(), meshsize), (0,))[0]
            del prod
        nonzero = [ell for ell in ells if ell != 0]
        if nonzero:
            rho = _r(meshes[0]).contiguous()
            offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
            stream = _lib.stream_handle()
            for ell in nonzero:
                terms = [(ell, m) for m in range(-ell, ell + 1)]
                carry = torch.zeros_like(rho)
                batch = _term_batch(mattrs, len(terms))
                for start in range(0, len(terms), batch):
                    chunk = terms[start:start + batch]
                    nt = len(chunk)
                    t_ell, t_m = [t[0] for t in chunk], [t[1] for t in chunk]
                    real = torch.empty((nt,) + tuple(int(n) for n in meshsize), dtype=torch.float32, device=rho.device)
                    _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rho), _lib.i32(meshsize),
                              _lib.f32(mattrs.cellsize), _lib.f32(offset), nt, _lib.i32(t_ell), _lib.i32(t_m),
                              _lib.ptr(real))
                    F = _r2c(real, meshsize)
                    _lib.call('pk_conj_multiply', stream, _lib.ptr(F), _lib.ptr(A0), nt, A0.numel(), _lib.ptr(F))
                    real = _c2r(F, meshsize, destroy_input=True)
                    del F
                    _lib.call('pk_ylm_separation_accumulate', stream, _lib.ptr(real), _lib.i32(meshsize),
                              _lib.f32(mattrs.cellsize), nt, _lib.i32(t_ell), _lib.i32(t_m), _lib.ptr(carry))
                    del real
                carry.view(-1)[0] = 0.  # remove_zero
                sums[ell] = 4. * np.pi * bin._sums(carry, (0,))[0]
                del carry
        raw = torch.stack([sums[ell] for ell in ells]).cpu().numpy()
        factors = [1.] * len(ells)
        attrs = dict(los=los_name)
    else:
        c1 = _c(meshes[0])
        if auto:
            prod = (c1.real * c1.real + c1.imag * c1.imag).to(torch.complex64)
        else:
            prod = torch.conj(c1) * _c(meshes[1])
        A = _c2r(prod.contiguous(), meshsize)
        del prod
        raw = bin._sums(A, ells, los=vlos).cpu().numpy()
        factors = [1. if ell == 0 else 2. * ell + 1. for ell in ells]
        attrs = dict(los=vlos)
    cellvol = float(np.prod(mattrs.cellsize.astype('f8')))
    norm = np.full(bin.nbins, norm_value, dtype='f8')
    poles = []
    for i, ell in enumerate(ells):
        num = raw[i] / bin.nmodes * factors[i]
        poles.append(Mesh2CorrelationPole(s=bin.xavg, s_edges=bin.edges, nmodes=bin.nmodes, num_raw=num / cellvol,
                                          norm=norm, volume=cellvol * bin.nmodes, ell=ell, attrs=attrs))
    return Mesh2CorrelationPoles(poles)


def _bessel_correlation(meshes, auto, bin, los_name, vlos, swap, norm_value):
    """compute_mesh2_correlation with ``bin.basis == 'bessel'`` (``mesh2.py:414-500``).

    The estimator's mode values stay in Fourier space: |delta|^2 (or conj(delta1) delta2)
    times L_ell(mu_k) for a fixed line of sight, |A0|^2 and conj(sum_m F_lm Y_lm(khat)) A0
    for the first point; ``pk_bin_bessel`` projects their real parts on j_ell(|k| s) at
    each bin's ``xavg`` (``mesh2.py:169-177``).  num_raw = factor (-1)^(ell/2) sums / N / V_cell,
    factor 1 for ell = 0, 2 ell + 1 (fixed los) or 4 pi (first point) otherwise; no division
    by the bin counts.
    """
    mattrs = bin.mattrs
    meshsize = mattrs.meshsize
    ells = bin.ells
    stream = _lib.stream_handle()

    def _c(mesh):
        return mesh.value if isinstance(mesh, ComplexMeshField) else _r2c(mesh.value, meshsize)

    def _r(mesh):
        return mesh.value if isinstance(mesh, RealMeshField) else _c2r(mesh.value, meshsize)

    nbins = bin.nbins
    sep = torch.as_tensor(np.asarray(bin.xavg, dtype='f8'), device=_device())
    nbytes = _lib.c_size_t()
    _lib.call('pk_bin_bessel_workspace_size', _lib.i32(meshsize), nbins, len(ells), _lib.ctypes.byref(nbytes))
    ws = _workspace(nbytes.value)
    out = torch.zeros(len(ells) * nbins, dtype=torch.float64, device=_device())
    klimit = None if bin.klimit is None else _lib.f32(bin.klimit)
    common = (_lib.i32(meshsize), _lib.f32(mattrs.kfun), mattrs.backend_code)

    def project(d1, d2, F, terms, los, include_ell0, accumulate):
        t_ell = _lib.i32([t[0] for t in terms]) if terms else None
        t_m = _lib.i32([t[1] for t in terms]) if terms else None
        _lib.call('pk_bin_bessel', stream, _lib.ptr(d1), _lib.ptr(d2), _lib.ptr(F), len(terms), t_ell, t_m, *common,
                  None if los is None else _lib.f32(los), _lib.ptr(sep), nbins, klimit, len(ells), _lib.i32(ells),
                  int(include_ell0), int(accumulate), _lib.ptr(out), _lib.ptr(ws), ws.numel())

    if vlos is None:
        if swap and not auto:
            meshes = meshes[::-1]
        A0 = _c(meshes[0] if auto else meshes[1]).contiguous()
        B0 = None if auto else _c(meshes[0]).contiguous()
        project(A0, B0, None, [], None, 0 in ells, False)
        terms = _firstpoint_terms(ells)
        if terms:
            rho = _r(meshes[0]).contiguous()
            offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
            batch = _term_batch(mattrs, len(terms))
            for start in range(0, len(terms), batch):
                chunk = terms[start:start + batch]
                nt = len(chunk)
                real = torch.empty((nt,) + tuple(int(n) for n in meshsize), dtype=torch.float32, device=rho.device)
                _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rho), _lib.i32(meshsize), _lib.f32(mattrs.cellsize),
                          _lib.f32(offset), nt, _lib.i32([t[0] for t in chunk]), _lib.i32([t[1] for t in chunk]),
                          _lib.ptr(real))
                F = _r2c(real, meshsize)
                del real
                project(A0, None, F, chunk, None, False, True)
                del F
        factors = [1. if ell == 0 else 4. * np.pi for ell in ells]
        attrs = dict(los=los_name)
    else:
        d1 = _c(meshes[0]).contiguous()
        d2 = None if auto else _c(meshes[1]).contiguous()
        project(d1, d2, None, [], vlos, True, False)
        factors = [1. if ell == 0 else 2. * ell + 1. for ell in ells]
        attrs = dict(los=vlos)
    raw = out.reshape(len(ells), nbins).cpu().numpy()
    cellvol = float(np.prod(mattrs.cellsize.astype('f8')))
    nmesh = float(np.prod(meshsize.astype('f8')))
    norm = np.full(nbins, norm_value, dtype='f8')
    poles = []
    for i, ell in enumerate(ells):
        num = raw[i] * factors[i] * (-1.) ** (ell // 2) / nmesh
        poles.append(Mesh2CorrelationPole(s=bin.xavg, s_edges=bin.edges, nmodes=bin.nmodes, num_raw=num / cellvol,
                                          norm=norm, volume=cellvol * bin.nmodes, ell=ell, attrs=attrs))
    return Mesh2CorrelationPoles(poles)


def _format_meshes(*meshes, fields=None):
    if len(meshes) == 1 and isinstance(meshes[0], (tuple, list)):
        meshes = tuple(meshes[0])
    meshes = list(meshes)
    assert 1 <= len(meshes) <= 2
    if fields is None:
        fields = [0]
    else:
        fields = list(fields)
    meshes = meshes + [None] * (2 - len(meshes))
    for mesh in meshes[len(fields):]:
        fields.append(fields[-1] if mesh is None else fields[-1] + 1)
    for i, (mesh, field) in enumerate(zip(meshes, fields)):
        if mesh is None:
            meshes[i] = meshes[fields.index(field)]
    return meshes, tuple(fields)


def _2c(mesh):
    return mesh if isinstance(mesh, ComplexMeshField) else mesh.r2c()


def _2r(mesh):
    return mesh if isinstance(mesh, RealMeshField) else mesh.c2r()


def _los(los):
    if isinstance(los, str) and los in ('firstpoint', 'local', 'endpoint'):
        return ('firstpoint' if los == 'local' else los), None, los == 'endpoint'
    if isinstance(los, str):
        vlos = np.zeros(3)
        vlos['xyz'.index(los)] = 1.
    else:
        vlos = np.asarray(los, dtype='f8')
    return los, vlos, False


def _firstpoint_terms(ells):
    return [(ell, m) for ell in ells if ell > 0 for m in range(-ell, ell + 1)]


def _free_device_memory():
    """Bytes free on the device plus those torch's caching allocator holds unused."""
    free, _ = torch.cuda.mem_get_info()
    return free + torch.cuda.memory_reserved() - torch.cuda.memory_allocated()


def _term_batch(mattrs, nterms):
    """How many (ell, m) terms to transform at once, given free device memory."""
    nr = int(np.prod(mattrs.meshsize))
    nc = int(mattrs.meshsize[0]) * int(mattrs.meshsize[1]) * (int(mattrs.meshsize[2]) // 2 + 1)
    per_term = 4 * nr + 8 * nc
    return int(max(1, min(nterms, 32, (0.4 * _free_device_memory()) // per_term)))


def _term_batches(mattrs, ells):
    """First-point terms grouped into transforms that fit in memory, whole ells kept together.

    Ells are taken in ascending order, every m of an ell in one batch when it fits (the
    kernels have compiled forms for whole-ell term lists); an ell larger than a batch is
    split.
    """
    terms = _firstpoint_terms(sorted(ells))
    if not terms:
        return []
    batch = _term_batch(mattrs, len(terms))
    out, cur = [], []
    for ell in sorted(ell for ell in ells if ell > 0):
        block = [(ell, m) for m in range(-ell, ell + 1)]
        if len(cur) + len(block) > batch and cur:
            out.append(cur)
            cur = []
        if len(block) > batch:
            out += [block[i:i + batch] for i in range(0, len(block), batch)]
        else:
            cur = cur + block
    if cur:
        out.append(cur)
    return out


def _ell_factors(ells, vlos):
    """Per-multipole factor of the binned sums: (2 ell + 1) global, 4 pi first point (1 for ell 0)."""
    if vlos is None:
        return [1. if ell == 0 else 4. * np.pi for ell in ells]
    return [2. * ell + 1. for ell in ells]


def _spectrum_sums(mattrs, bin, los, rmesh=None, cmesh=None, cmesh2=None, rmesh2=None, keep=None):
    """Raw per-bin sums (nells, nbins) float64 on the device (no host synchronisation).

    Global los: sum of w Re/Im(conj(d1) d2) L_ell(mu) over each bin.  First point: the
    sums of ``pk_bin_firstpoint`` over all (ell, m) terms.  ``rmesh`` / ``cmesh`` are the
    real / Hermitian-complex values of the first mesh (either may be None), likewise for
    the second mesh of a cross spectrum.  ``keep`` (a dict, first point only): receives
    A0 and the transformed Y_lm-weighted meshes of every term batch, ``keep['F']`` a list of
    (terms, F), when they fit in a third of the free device memory (the backward pass
    then reuses them instead of transforming again).
    """
    meshsize = mattrs.meshsize
    los, vlos, swap = _los(los)
    ells = bin.ells
    nbins = bin.nbins
    ws = bin._workspace()
    stream = _lib.stream_handle()
    raw = torch.zeros(len(ells) * nbins, dtype=torch.float64, device=_device())
    cross = cmesh2 is not None or rmesh2 is not None
    if vlos is None:
        if swap and cross:
            rmesh, cmesh, rmesh2, cmesh2 = rmesh2, cmesh2, rmesh, cmesh
        if rmesh is None:
            rmesh = _c2r(cmesh, meshsize)
        if cross:
            A0 = cmesh2 if cmesh2 is not None else _r2c(rmesh2, meshsize)
            B0 = cmesh if cmesh is not None else _r2c(rmesh, meshsize)
        else:
            A0 = cmesh if cmesh is not None else _r2c(rmesh, meshsize)
            B0 = None
        A0 = A0.contiguous()
        terms = _firstpoint_terms(ells)
        kshifts = getattr(bin, '_kshifts', [])

        def bin_firstpoint(F, nt, t_ell, t_m, include_ell0):
            if not kshifts:
                _lib.call('pk_bin_firstpoint', stream, _lib.ptr(A0), _lib.ptr(B0), _lib.ptr(F), nt, t_ell, t_m,
                          _lib.i32(meshsize), _lib.f32(mattrs.kfun), _lib.ptr(bin.d_edges), len(bin._edges1d),
                          bin._step, mattrs.backend_code, len(ells), _lib.i32(ells), include_ell0, 1, _lib.ptr(raw),
                          _lib.ptr(ws), ws.numel())
                return
            for sh in kshifts:  # mode oversampling: the per-shift sums, averaged below
                _lib.call('pk_bin_firstpoint_shifted', stream, _lib.ptr(A0), _lib.ptr(B0), _lib.ptr(F), nt, t_ell, t_m,
                          _lib.i32(meshsize), _lib.f32(mattrs.kfun), _lib.f32(sh), _lib.ptr(bin.d_edges),
                          len(bin._edges1d), bin._step, mattrs.backend_code, len(ells), _lib.i32(ells), include_ell0,
                          1, _lib.ptr(raw), _lib.ptr(ws), ws.numel())

        if not terms:
            bin_firstpoint(None, 0, None, None, 1)
        else:
            rho = rmesh.contiguous()
            offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
            batches = _term_batches(mattrs, ells)
            real = torch.empty((max(map(len, batches)),) + tuple(int(n) for n in meshsize), dtype=torch.float32,
                               device=rho.device)
            if keep is not None:
                per_term = 8 * A0.numel()
                if len(terms) * per_term < _free_device_memory() / 3:
                    keep['A0'], keep['F'] = A0, []
                else:
                    keep = None
            for ib, chunk in enumerate(batches):
                nt = len(chunk)
                t_ell, t_m = [t[0] for t in chunk], [t[1] for t in chunk]
                _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rho), _lib.i32(meshsize), _lib.f32(mattrs.cellsize),
                          _lib.f32(offset), nt, _lib.i32(t_ell), _lib.i32(t_m), _lib.ptr(real))
                F = _r2c(real[:nt], meshsize)
                include_ell0 = int(ib == 0 and 0 in ells)  # ell = 0 rides on the first batch
                bin_firstpoint(F, nt, _lib.i32(t_ell), _lib.i32(t_m), include_ell0)
                if keep is not None:
                    keep['F'].append((chunk, F))
                del F
        raw = raw.reshape(len(ells), nbins)
        if kshifts:
            raw = raw / len(kshifts)
        if swap:  # conj: odd multipoles (imaginary parts) change sign
            sign = torch.tensor([-1. if ell % 2 else 1. for ell in ells], dtype=raw.dtype, device=raw.device)
            raw = raw * sign[:, None]
        return raw
    d1 = (cmesh if cmesh is not None else _r2c(rmesh, meshsize)).contiguous()
    d2 = None
    if cross:
        d2 = (cmesh2 if cmesh2 is not None else _r2c(rmesh2, meshsize)).contiguous()
    kshifts = getattr(bin, '_kshifts', [])
    if kshifts:  # mode oversampling: mean of the per-shift sums
        for ish, sh in enumerate(kshifts):
            _lib.call('pk_bin_global_shifted', stream, _lib.ptr(d1), _lib.ptr(d2), _lib.i32(meshsize),
                      _lib.f32(mattrs.kfun), _lib.f32(sh), _lib.f32(vlos), _lib.ptr(bin.d_edges), len(bin._edges1d),
                      bin._step, mattrs.backend_code, len(ells), _lib.i32(ells), int(ish > 0), _lib.ptr(raw),
                      _lib.ptr(ws), ws.numel())
        return raw.reshape(len(ells), nbins) / len(kshifts)
    _lib.call('pk_bin_global', stream, _lib.ptr(d1), _lib.ptr(d2), _lib.i32(meshsize), _lib.f32(mattrs.kfun),
              _lib.f32(vlos), _lib.ptr(bin.d_edges), len(bin._edges1d), bin._step, mattrs.backend_code,
              len(ells), _lib.i32(ells), _lib.ptr(raw), _lib.ptr(ws), ws.numel())
    return raw.reshape(len(ells), nbins)


def _fusable(ells):
    """Multipoles the fused interlace + binning pass takes (up to 3 even ells <= 4)."""
    return len(ells) <= 3 and all(ell % 2 == 0 and ell <= 4 for ell in ells)


def _interlaced_sums(mattrs, bin, vlos, shifted, comp_order):
    """Global-los raw sums (nells, nbins) float64 of the mesh that interlacing ``shifted``
    ((nshifts, N0, N1, N2/2+1) R2C meshes) with compensation order ``comp_order`` would give,
    without forming it (``pk_bin_global_interlaced``)."""
    nbytes = _lib.c_size_t()
    _lib.call('pk_bin_batch_workspace_size', _lib.i32(mattrs.meshsize), len(bin._edges1d), len(bin.ells), 1,
              _lib.ctypes.byref(nbytes))
    ws = _workspace(nbytes.value)
    out = torch.zeros(len(bin.ells) * bin.nbins, dtype=torch.float64, device=shifted.device)
    _lib.call('pk_bin_global_interlaced', _lib.stream_handle(), _lib.ptr(shifted), 1, shifted.shape[0],
              int(comp_order), _lib.i32(mattrs.meshsize), _lib.f32(mattrs.kfun), _lib.f32(vlos), _lib.ptr(bin.d_edges),
              len(bin._edges1d), bin._step, mattrs.backend_code, len(bin.ells), _lib.i32(bin.ells), _lib.ptr(out),
              _lib.ptr(ws), ws.numel())
    return out.reshape(len(bin.ells), bin.nbins)


def _split(mesh):
    if mesh is None:
        return None, None
    if isinstance(mesh, ComplexMeshField):
        return None, mesh.value
    return mesh.value, None


def compute_mesh2_spectrum(*meshes, bin=None, los='z'):
    """Power-spectrum multipoles from mesh(es) (``mesh2.py:253-374``)."""
    meshes, fields = _format_meshes(*meshes)
    mattrs = meshes[0].attrs
    norm_value = np.float32(np.prod(mattrs.meshsize.astype('f4'))) / np.float32(np.prod(mattrs.cellsize))
    los_name, vlos, swap = _los(los)
    attrs = dict(los=vlos if vlos is not None else los_name)
    ells = bin.ells
    nbins = bin.nbins
    lazy = getattr(meshes[0], 'lazy', None) if fields[1] == fields[0] else None
    if lazy is not None and vlos is not None and _fusable(ells) and not getattr(bin, '_kshifts', []):
        raw = _interlaced_sums(mattrs, bin, vlos, *lazy)
    else:
        r1, c1 = _split(meshes[0])
        r2, c2 = (None, None) if fields[1] == fields[0] else _split(meshes[1])
        raw = _spectrum_sums(mattrs, bin, los, rmesh=r1, cmesh=c1, rmesh2=r2, cmesh2=c2)
    # the sums stay on the device until num_raw is first read (one read-back for all poles)
    num = DeferredRows(raw, bin.nmodes, _ell_factors(ells, vlos))
    norm = np.full(nbins, norm_value, dtype='f8')
    poles = [Mesh2SpectrumPole(k=bin.xavg, k_edges=bin.edges, nmodes=bin.nmodes, num_raw=num.row(i),
                               num_shotnoise=np.zeros(nbins), norm=norm,
                               volume=float(np.prod(mattrs.kfun.astype('f8'))) * bin.nmodes, ell=ell, attrs=attrs)
             for i, ell in enumerate(ells)]
    return Mesh2SpectrumPoles(poles)


def compute_mesh2(*meshes, bin=None, los='z'):
    """``compute_mesh2`` (``mesh2.py:225-250``): dispatch on the binning operator."""
    if isinstance(bin, BinMesh2SpectrumPoles):
        return compute_mesh2_spectrum(*meshes, bin=bin, los=los)
    if isinstance(bin, BinMesh2CorrelationPoles):
        return compute_mesh2_correlation(*meshes, bin=bin, los=los)
    raise NotImplementedError('bin must be a BinMesh2SpectrumPoles or BinMesh2CorrelationPoles')


# ---------------------------------------------------------------------- normalisation

def _norm_attrs(mattrs, cellsize):
    """``get_halo_for_new_mattrs(mattrs, cellsize=...)`` without sharding (``mesh.py:3002-3039``)."""
    cs = np.broadcast_to(np.asarray(cellsize, 'f4'), (3,))
    meshsize = np.ceil((mattrs.boxsize / cs).astype('f4')).astype('i4')
    boxsize = (meshsize * cs.astype('f8')).astype('f4')
    if np.any((meshsize - mattrs.meshsize) % 2):
        cell = (boxsize / meshsize.astype('f4')).astype('f4')
        meshsize = meshsize + 1
        boxsize = (cell * meshsize.astype('f4')).astype('f4')
    return MeshAttrs(meshsize=meshsize, boxsize=boxsize, boxcenter=mattrs.boxcenter, fft_backend=mattrs.fft_backend)


def _iter_meshes(*inputs, resampler='cic', interlacing=0, compensate=False, **kwargs):
    attrs = {k: v for k, v in kwargs.items() if v is not None}
    for inp in inputs:
        if isinstance(inp, RealMeshField):
            yield inp
            continue
        mattrs = inp.attrs
        if 'cellsize' in attrs:
            mattrs = _norm_attrs(mattrs, attrs['cellsize'])
        elif attrs:
            mattrs = mattrs.clone(**attrs)
        yield _paint(mattrs, inp.positions, inp._weights, resampler=resampler, interlacing=interlacing,
                     compensate=compensate, out='real')


def compute_normalization(*inputs, resampler='cic', start=1., **kwargs):
    """sum(prod meshes) * cell volume^(1 - n) (``mesh.py:3092-3118``), accumulated in float64."""
    product = None
    cellsize = None
    for mesh in _iter_meshes(*inputs, resampler=resampler, **kwargs):
        v = mesh.value.double()
        product = v if product is None else product * v
        cellsize = mesh.attrs.cellsize
    return float(start) * float(product.sum()) * float(np.prod(cellsize.astype('f8')))**(1 - len(inputs))


def compute_box_normalization(*inputs):
    mattrs = inputs[0].attrs
    size = float(np.prod(mattrs.meshsize.astype('f8')))
    normalization = 1.
    for mesh in inputs:
        normalization *= float(mesh.sum()) / size
    return normalization * size * float(np.prod(mattrs.cellsize.astype('f8')))**(1 - len(inputs))


def compute_box2_normalization(*inputs, bin=None):
    meshes = _format_meshes(*inputs)[0]
    norm = compute_box_normalization(*meshes)
    if bin is not None:
        return [norm] * len(bin.ells)
    return norm


def compute_fkp2_normalization(*fkps, bin=None, cellsize=10., split=None, fields=None, **kwargs):
    """FKP normalisation (``mesh2.py:516-574``): alpha * sum(rho_d rho_r) / V_cell, CIC at ``cellsize``.

    With ``split`` (a seed as ``split_particles`` takes it), the two randoms fields are
    disjoint random subsamples of the randoms instead (``mesh2.py:543-553``), alpha rescaled
    by each subsample's share of the weights.
    """
    kwargs.update(cellsize=cellsize)
    if split is not None:

        def randoms_of(f):
            return f.randoms if isinstance(f, FKPField) else f

        fkps, fields = _format_meshes(*fkps, fields=fields)
        def wsum(p):
            return float(p.weights.double().sum())

        alpha = 1.
        for f in fkps:
            if isinstance(f, FKPField):
                alpha *= wsum(f.data) / wsum(f.randoms)
        randoms = split_particles(*[randoms_of(f) for f in fkps], seed=split, fields=fields)
        for f, r in zip(fkps, randoms):
            alpha *= wsum(randoms_of(f)) / wsum(r)
        norm = alpha * compute_normalization(*randoms, **kwargs)
        if bin is not None:
            return [norm] * len(bin.ells)
        return norm
    fkps, fields = _format_meshes(*fkps)
    if fields[1] == fields[0]:
        fkp = fkps[0]
        alpha = float(fkp.data.sum()) / float(fkp.randoms.sum())
        norm = alpha * compute_normalization(fkp.data, fkp.randoms, **kwargs)
    else:
        alpha2 = float(fkps[1].data.sum()) / float(fkps[1].randoms.sum())
        norm = alpha2 * compute_normalization(fkps[0].data, fkps[1].randoms, **kwargs)
        alpha2 = float(fkps[0].data.sum()) / float(fkps[0].randoms.sum())
        norm += alpha2 * compute_normalization(fkps[1].data, fkps[0].randoms, **kwargs)
        norm = norm / 2
    if bin is not None:
        return [norm] * len(bin.ells)
    return norm


def compute_fkp2_shotnoise(*fkps, bin=None, fields=None):
    """FKP shot noise (``mesh2.py:577-621``): sum of w1 w2 for the same positions, else 0."""
    fkps, fields = _format_meshes(*fkps, fields=fields)

    def particles(f):
        return f.particles if isinstance(f, FKPField) else f

    if fields[1] == fields[0]:
        p = [particles(f) for f in fkps]
        shotnoise = float((p[0].weights.double() * p[1].weights.double()).sum())
    else:
        shotnoise = 0.
    if bin is not None:
        return [shotnoise * (ell == 0) * np.ones(bin.nbins) for ell in bin.ells]
    return shotnoise


def _window_edges(edgesin, ellsin):
    """Input k edges as (n, 2) and input multipoles: ints, or (ell, wide-angle order) pairs when
    any is given as a pair or the container carries wide-angle orders (``mesh2.py:826-836``)."""
    if hasattr(edgesin, 'ells') and hasattr(edgesin, 'poles'):  # a multipole container: its ells and k edges
        ellsin = list(zip(edgesin.ells, edgesin.wa_orders)) if any(edgesin.wa_orders) else edgesin.ells
        edgesin = next(iter(edgesin)).k_edges
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    if isinstance(ellsin, (int, np.integer)):
        ellsin = (ellsin,)
    if any(isinstance(e, tuple) for e in ellsin):
        return edgesin, [(int(e[0]), int(e[1])) if isinstance(e, tuple) else (int(e), 0) for e in ellsin]
    return edgesin, [int(ell) for ell in ellsin]


def _no_wide_angle(ellsin):
    """Wide-angle orders > 0 are built for the 'firstpoint' theory line of sight only."""
    if any(isinstance(e, tuple) and e[1] != 0 for e in ellsin):
        raise NotImplementedError("wide-angle orders > 0 with the 'local' theory line of sight are not supported")


def _plain_ells(ellsin):
    """Input multipoles of a fixed line of sight: wide-angle order 0 only (``mesh2.py:850-851``)."""
    if any(isinstance(e, tuple) and e[1] != 0 for e in ellsin):
        raise ValueError('wide-angle orders > 0 need a local (first-point) line of sight')
    return [e[0] if isinstance(e, tuple) else e for e in ellsin]


def _wide_angle_terms(ellsin):
    """Input multipoles as (ell, wide-angle order) pairs."""
    return [e if isinstance(e, tuple) else (int(e), 0) for e in ellsin]


def _wide_angle_rho(rmesh1, wa, mattrs, offset, cache):
    """W1 |x|^-wa (``mesh2.py:1214``), W1 itself for wa = 0; cached per order."""
    if wa == 0:
        return rmesh1
    if wa not in cache:
        rho = rmesh1.clone()
        _lib.call('pk_radial_power', _lib.stream_handle(), _lib.ptr(rho), 1, _lib.i32(mattrs.meshsize),
                  _lib.f32(mattrs.cellsize), _lib.f32(offset), 0, -int(wa))
        cache[wa] = rho
    return cache[wa]


def _wide_angle_s(meshes, nmeshes, wa, mattrs):
    """meshes *= |s|^wa on the separation grid (``mesh2.py:1214``: Q s^wa), in place."""
    if wa != 0:
        _lib.call('pk_radial_power', _lib.stream_handle(), _lib.ptr(meshes), nmeshes, _lib.i32(mattrs.meshsize),
                  _lib.f32(mattrs.cellsize), None, 1, int(wa))


def _window_batch(mattrs, batch_size):
    """Columns per pass of the selection-function window: B half-complex inputs, their real
    transforms and the transformed products must fit (about 16 N bytes per column)."""
    n = int(np.prod(mattrs.meshsize))
    fit = max(int(_free_device_memory() // (20 * n)), 1)
    limit = 16 if batch_size is None else max(int(batch_size), 1)
    return max(min(fit, limit, 16), 1)


def _window_merged(mattrs, bin, vlos, ells, ellsin, klo, khi, N):
    """Periodic window columns of disjoint, ascending input bins [klo, khi) in one binning
    pass per 9 (ell, ell_in) pairs, on the union of the output and input edges (float32, as
    |k| is compared): each merged interval lies in one output bin b and at most one input
    bin e, and its sums are added to column e, row b.  Returns (len(ellsin), nin, nells, nbins)."""
    eout = bin._edges1d.astype('f4')
    merged = np.unique(np.concatenate([eout, klo, khi]).astype('f4'))
    merged = merged[(merged >= eout[0]) & (merged <= eout[-1])]
    m0 = merged[:-1]
    b = np.searchsorted(eout, m0, side='right') - 1
    e = np.searchsorted(klo, m0, side='right') - 1
    inside = (e >= 0) & (merged[1:] <= khi[np.maximum(e, 0)]) & (b >= 0) & (b < bin.nbins)
    pairs = [(ill, iin) for iin in range(len(ellsin)) for ill, ell in enumerate(ells) if ell % 2 == 0]
    nm = len(merged) - 1
    out = np.zeros((len(ellsin), len(klo), len(ells), bin.nbins), dtype='f8')
    if not pairs or nm < 1:
        return out
    d_edges = torch.as_tensor(merged, device=_device())
    nbytes = _lib.c_size_t()
    _lib.call('pk_bin_workspace_size', _lib.i32(mattrs.meshsize), len(merged), 9, _lib.ctypes.byref(nbytes))
    ws = _workspace(nbytes.value)
    raw = torch.empty((len(pairs), nm), dtype=torch.float64, device=_device())
    for p0 in range(0, len(pairs), 9):
        chunk = pairs[p0:p0 + 9]
        _lib.call('pk_bin_window_pairs', _lib.stream_handle(), _lib.i32(mattrs.meshsize), _lib.f32(mattrs.kfun),
                  _lib.f32(vlos), _lib.ptr(d_edges), len(merged), _uniform_step(merged), mattrs.backend_code,
                  len(chunk), _lib.i32([ells[ill] for ill, _ in chunk]), _lib.i32([ellsin[iin] for _, iin in chunk]),
                  float(N), _lib.ptr(raw[p0:p0 + len(chunk)]), _lib.ptr(ws), ws.numel())
    raw = raw.cpu().numpy()
    for q, (ill, iin) in enumerate(pairs):
        np.add.at(out[iin, :, ill], (e[inside], b[inside]), raw[q, inside])
    return out


def compute_mesh2_spectrum_window(*meshes, edgesin, ellsin=None, bin=None, los='z', buffer=None, batch_size=None,
                                  pbar=False, norm=None, flags=tuple()):
    """Window matrix of the power-spectrum multipoles (``mesh2.py:921-1482``).

    Global line of sight ('x', 'y', 'z' or a 3-vector) with the input power defined on the
    mesh (no 'smooth' / 'infinite' flag).  Column (ell_in, [k_lo, k_hi)) is the estimator
    applied to ``A = N 1{k_lo <= |k| < k_hi} L_ell_in(mu)``:

    - periodic box (a ``MeshAttrs`` given): A is binned as it is, formed per mode inside the
      binning kernel; when the input edges are the output bins one pass per ell_in fills the
      diagonal, as the reference does (mesh2.py:1113-1118); disjoint ascending input bins take
      one pass for all columns on the merged edges (``pk_bin_window_pairs``), other input
      edges one pass per column (``pk_bin_window`` without a mesh);
    - selection function (one or two meshes W): ``Q = c2r(W1 W2*) / N`` and
      ``A <- r2c(Q c2r(A))``, up to 16 columns per batched FFT pair (``pk_window_fill``,
      cuFFT C2R, ``pk_window_multiply`` with the C2R's 1 / N folded into Q, cuFFT R2C,
      ``pk_bin_window_batch``: the fused binning pass, linear in A, over the batch).

    Row (ell, k bin) is ``(2 ell + 1) / (1 + ell % 2) rnorm bin(A (L_ell(mu) + L_ell(-mu)))``,
    k = 0 dropped, with ``rnorm = (N / V_cell) / norm / N``; odd ell rows are 0 (the
    reference's Legendre sum vanishes for odd ell).  Returns a ``WindowMatrix`` of shape
    (len(ells) nbins, len(ellsin) len(edgesin)).  ``buffer`` and ``pbar`` are accepted and
    have no effect; ``batch_size`` caps the columns per FFT batch.  The first-point /
    end-point line of sight (theory line of sight 'firstpoint', inputs ell_in or (ell_in,
    wide-angle order)) goes through ``_firstpoint_window``, the 'local' theory line of sight (``ellsin=(ells, 'local')``)
    through ``_local_window``.  ``flags=('smooth',)`` with a global line of sight goes through
    ``_smooth_window`` (first point: ``_firstpoint_smooth_window``), ``flags=('infinite',)``
    through ``_infinite_window`` (first point: ``_firstpoint_infinite_window``); 'smooth' with
    the 'local' theory line of sight through ``_local_smooth_window``, 'infinite' through
    ``_local_infinite_window``.  The 'jaxdecomp' backend raises ``NotImplementedError``.
    """
    from .types import WindowMatrix
    flags = tuple(flags)
    meshes, fields = _format_meshes(*meshes)
    periodic = isinstance(meshes[0], MeshAttrs)
    if periodic:
        assert fields[1] == fields[0]
        mattrs = meshes[0]
    else:
        mattrs = meshes[0].attrs
    if mattrs.fft_backend != 'jax':
        raise NotImplementedError("the window matrix takes the 'jax' FFT backend")
    los, vlos, swap = _los(los)
    f4 = np.float32
    ells = bin.ells
    nbins, nells = bin.nbins, len(ells)
    meshsize = mattrs.meshsize
    N = f4(np.prod(meshsize.astype('f4'), dtype='f4'))
    _norm = f4(N / f4(np.prod(mattrs.cellsize, dtype='f4')))
    norm = np.asarray(_norm if norm is None else norm, dtype='f4')
    if norm.ndim <= 1:
        norm = norm * np.ones(nells, dtype='f4')
    rnorm = (_norm / norm / N).astype('f4')
    if ('smooth' in flags or 'infinite' in flags) and vlos is None:
        if isinstance(ellsin, (tuple, list)) and len(ellsin) == 2 and isinstance(ellsin[1], str):
            ellsin, theory_los = ellsin
            if theory_los not in ('firstpoint', 'local'):
                raise NotImplementedError("theory line of sight '{}' with these flags is not supported".format(theory_los))
        else:
            theory_los = 'firstpoint'
        if isinstance(ellsin, (int, np.integer)):
            ellsin = (ellsin,)
        edgesin, ellsin = _window_edges(edgesin, ellsin)
        if theory_los == 'local':
            _no_wide_angle(ellsin)
            ellsin = _plain_ells(ellsin)
        if 'smooth' in flags and theory_los == 'local':
            wmat = _local_smooth_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm)
        elif 'smooth' in flags:
            wmat = _firstpoint_smooth_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm)
        elif theory_los == 'local':
            wmat = _local_infinite_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm)
        else:
            wmat = _firstpoint_infinite_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm)
        return _window_matrix(bin, norm, edgesin, ellsin, wmat)
    # a fixed line of sight bins with the fused window kernels, which take each mode once; the
    # local lines of sight bin through bin(...), which takes mode oversampling
    if vlos is not None:
        _plain_bins(bin, 'compute_mesh2_spectrum_window with a fixed line of sight')
    if 'infinite' in flags and 'smooth' not in flags:
        edgesin, ellsin = _window_edges(edgesin, ellsin)
        ellsin = _plain_ells(ellsin)
        Q = None if periodic else _selection_q(meshes, fields, mattrs, N)
        wmat = _infinite_window(mattrs, bin, Q, vlos, ellsin, edgesin, rnorm, batch_size)
        return _window_matrix(bin, norm, edgesin, ellsin, wmat)
    if 'smooth' in flags:
        edgesin, ellsin = _window_edges(edgesin, ellsin)
        ellsin = _plain_ells(ellsin)
        Q = None if periodic else _selection_q(meshes, fields, mattrs, N)
        wmat = _smooth_window(mattrs, bin, Q, vlos, ellsin, edgesin, rnorm)
        return _window_matrix(bin, norm, edgesin, ellsin, wmat)
    if vlos is None:
        theory_los = 'firstpoint'
        if isinstance(ellsin, (tuple, list)) and len(ellsin) == 2 and isinstance(ellsin[1], str):
            ellsin, theory_los = ellsin
        if theory_los not in ('firstpoint', 'local'):
            raise NotImplementedError("theory line of sight '{}' is not supported for the window".format(theory_los))
        if isinstance(ellsin, (int, np.integer)):
            ellsin = (ellsin,)
        edgesin, ellsin = _window_edges(edgesin, ellsin)
        if theory_los == 'local':
            _no_wide_angle(ellsin)
            ellsin = _plain_ells(ellsin)
            wmat = _local_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm)
        else:
            wmat = _firstpoint_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm, batch_size)
        return _window_matrix(bin, norm, edgesin, ellsin, wmat)
    edgesin, ellsin = _window_edges(edgesin, ellsin)
    ellsin = _plain_ells(ellsin)
    nin = len(edgesin)
    klo, khi = edgesin[:, 0].astype('f4'), edgesin[:, -1].astype('f4')

    stream = _lib.stream_handle()
    ws = bin._workspace()
    args_geom = (_lib.i32(meshsize), _lib.f32(mattrs.kfun), _lib.f32(vlos))
    args_bins = (_lib.ptr(bin.d_edges), len(bin._edges1d), bin._step, mattrs.backend_code, nells, _lib.i32(ells))

    def bin_window(out, value, ellin, lo, hi):
        _lib.call('pk_bin_window', stream, _lib.ptr(value) if value is not None else None, *args_geom, *args_bins,
                  int(ellin), float(lo), float(hi), float(N), _lib.ptr(out), _lib.ptr(ws), ws.numel())

    common = False
    if periodic:
        bedges = bin.edges
        mask_in = np.all(edgesin >= bedges[0], axis=-1) & np.all(edgesin <= bedges[-1], axis=-1)
        mask_edges = np.all(bedges >= edgesin[0], axis=-1) & np.all(bedges <= edgesin[-1], axis=-1)
        common = mask_edges.sum() == mask_in.sum() and np.allclose(edgesin[mask_in], bedges[mask_edges])

    if common:
        sums = torch.empty((len(ellsin), nells, nbins), dtype=torch.float64, device=_device())
        for iin, ellin in enumerate(ellsin):
            bin_window(sums[iin], None, ellin, -np.inf, np.inf)
    else:
        sums = torch.empty((len(ellsin), nin, nells, nbins), dtype=torch.float64, device=_device())
        if periodic and nin > 1 and np.all(khi > klo) and np.all(klo[1:] >= khi[:-1]):
            sums = _window_merged(mattrs, bin, vlos, ells, ellsin, klo, khi, N)
        elif periodic:
            for iin, ellin in enumerate(ellsin):
                for e in range(nin):
                    bin_window(sums[iin, e], None, ellin, klo[e], khi[e])
        else:
            A1 = _2c(meshes[0]).value.contiguous()
            A2 = A1 if fields[1] == fields[0] else _2c(meshes[1]).value.contiguous()
            prod = torch.empty_like(A1)
            _lib.call('pk_conj_multiply', stream, _lib.ptr(A2), _lib.ptr(A1), 1, A1.numel(), _lib.ptr(prod))
            # Q = c2r(W1 W2*) / N, times the 1 / N of every column's c2r (taken unscaled)
            Q = _c2r(prod, meshsize, scale=False, destroy_input=True)
            del prod, A1, A2
            _lib.call('pk_scale_real', stream, _lib.ptr(Q), Q.numel(), float(np.float64(f4(1.) / N) ** 3))
            nreal = Q.numel()
            B = _window_batch(mattrs, batch_size)
            cshape = tuple(int(n) for n in meshsize[:2]) + (int(meshsize[2]) // 2 + 1,)
            even = [ill for ill, ell in enumerate(ells) if ell % 2 == 0]
            sums.zero_()
            if even:
                nbytes = _lib.c_size_t()
                _lib.call('pk_bin_batch_workspace_size', _lib.i32(meshsize), len(bin._edges1d), len(even), B,
                          _lib.ctypes.byref(nbytes))
                wsb = _workspace(nbytes.value)
                raw = torch.empty((B, len(even), nbins), dtype=torch.float64, device=_device())
            for iin, ellin in enumerate(ellsin):
                for e0 in range(0, nin if even else 0, B):
                    nb = min(B, nin - e0)
                    cols = torch.empty((nb,) + cshape, dtype=torch.complex64, device=_device())
                    _lib.call('pk_window_fill', stream, *args_geom[:2], mattrs.backend_code, args_geom[2], int(ellin),
                              float(N), nb, _lib.f32(klo[e0:e0 + nb]), _lib.f32(khi[e0:e0 + nb]), _lib.ptr(cols))
                    real = _c2r(cols, meshsize, scale=False, destroy_input=True)
                    del cols
                    _lib.call('pk_window_multiply', stream, _lib.ptr(real), nb, _lib.ptr(Q), nreal)
                    cols = _r2c(real, meshsize)
                    del real
                    _lib.call('pk_bin_window_batch', stream, _lib.ptr(cols), nb, *args_geom, _lib.ptr(bin.d_edges),
                              len(bin._edges1d), bin._step, mattrs.backend_code, len(even),
                              _lib.i32([ells[ill] for ill in even]), 1, _lib.ptr(raw), _lib.ptr(wsb), wsb.numel())
                    sums[iin, e0:e0 + nb, even] = raw[:nb]
                    del cols
    sums = sums.cpu().numpy() if isinstance(sums, torch.Tensor) else sums
    with np.errstate(invalid='ignore', divide='ignore'):
        factor = np.array([(2 * ell + 1) / (1 + ell % 2) * rnorm[ill] for ill, ell in enumerate(ells)])
        spectra = sums / bin.nmodes * factor[:, None]  # (..., nells, nbins)
    if common:
        wmat = []
        rows = np.flatnonzero(mask_in)
        for iin in range(len(ellsin)):
            w = np.zeros((nin, nells, nbins), dtype='f8')
            for ill in range(nells):
                w[rows, ill, np.flatnonzero(mask_edges)] = spectra[iin, ill][mask_edges]
            wmat.append(w.reshape(nin, -1))
    else:
        wmat = [spectra[iin].reshape(nin, -1) for iin in range(len(ellsin))]
    wmat = np.concatenate(wmat, axis=0).T
    return _window_matrix(bin, norm, edgesin, ellsin, wmat)


def _window_matrix(bin, norm, edgesin, ellsin, wmat):
    """The ``WindowMatrix`` of ``mesh2.py:1462-1482``: output multipoles on ``bin`` with
    ``norm`` per ell, theory multipoles on the input edges (``k`` their mid-points)."""
    from .types import WindowMatrix
    nbins, nin = bin.nbins, len(edgesin)
    observable = Mesh2SpectrumPoles([Mesh2SpectrumPole(k=bin.xavg, k_edges=bin.edges, nmodes=bin.nmodes,
                                                       num_raw=np.zeros(nbins), num_shotnoise=np.zeros(nbins),
                                                       norm=np.ones(nbins) * norm[ill], ell=ell)
                                     for ill, ell in enumerate(bin.ells)])
    kin = np.mean(edgesin, axis=-1)
    terms = _wide_angle_terms(ellsin)
    theory = Mesh2SpectrumPoles([Mesh2SpectrumPole(k=kin, k_edges=edgesin, nmodes=np.ones(nin), num_raw=np.zeros(nin),
                                                   ell=ellin, attrs=dict(wa_order=wa) if wa else None)
                                 for ellin, wa in terms])
    return WindowMatrix(observable=observable, theory=theory, value=wmat)


def _selection_q(meshes, fields, mattrs, N):
    """``Q = c2r(W1 W2*) / N`` (``mesh2.py:1019-1026``), a real device mesh."""
    A1 = _2c(meshes[0]).value.contiguous()
    A2 = A1 if fields[1] == fields[0] else _2c(meshes[1]).value.contiguous()
    prod = torch.empty_like(A1)
    _lib.call('pk_conj_multiply', _lib.stream_handle(), _lib.ptr(A2), _lib.ptr(A1), 1, A1.numel(), _lib.ptr(prod))
    Q = _c2r(prod, mattrs.meshsize, destroy_input=True)
    _lib.call('pk_scale_real', _lib.stream_handle(), _lib.ptr(Q), Q.numel(), float(np.float32(1.) / N))
    return Q


def _bessel_primitive(ell, x, h=0.05):
    """``F(x) = int_0^x t^2 j_ell(t) dt`` (float64) for x >= 0: 8-point Gauss-Legendre panels
    of width h summed cumulatively, plus one 8-point panel from the last node to x."""
    from scipy.special import spherical_jn
    x = np.asarray(x, dtype='f8')
    xg, wg = np.polynomial.legendre.leggauss(8)
    n = int(np.ceil(float(x.max(initial=0.)) / h)) + 1
    nodes = np.arange(n + 1) * h
    t = ((nodes[1:] + nodes[:-1]) / 2.)[:, None] + (h / 2.) * xg
    Fn = np.concatenate([[0.], np.cumsum((h / 2.) * np.sum(wg * t ** 2 * spherical_jn(ell, t), axis=-1))])
    i = np.minimum((x / h).astype(np.int64), n)
    a = nodes[i]
    half = (x - a) / 2.
    t = ((x + a) / 2.)[..., None] + half[..., None] * xg
    return Fn[i] + half * np.sum(wg * t ** 2 * spherical_jn(ell, t), axis=-1)


def _bessel_shell(ell, lo, hi, s):
    """``4 pi int_lo^hi k^2 j_ell(k s) dk`` for separations s: ``4 pi (F(hi s) - F(lo s)) / s^3``;
    at s = 0, ``4 pi (hi^3 - lo^3) / 3`` for ell = 0, else 0 (the tophat integral of
    ``utils.py:453-462``)."""
    s = np.asarray(s, dtype='f8')
    out = np.zeros_like(s)
    nz = s > 0
    if nz.any():
        sz = s[nz]
        out[nz] = 4. * np.pi * (_bessel_primitive(ell, hi * sz) - _bessel_primitive(ell, lo * sz)) / sz ** 3
    if ell == 0:
        out[~nz] = 4. * np.pi * (hi ** 3 - lo ** 3) / 3.
    return out


def _smooth_window(mattrs, bin, Q, vlos, ellsin, edgesin, rnorm):
    """'smooth' window of the global line of sight (``mesh2.py:1061-1093``): the mesh enters only
    through the correlation-space multipoles ``Qs = sbin(Q L_ell(mu_s) L_ell_in(mu_s))`` on the
    separation grid with default (unique |s|) bins, one binning pass per 3 Legendre orders: the
    product ``L_ell L_ell_in`` is expanded on ``L_p`` and each ``sbin(Q L_p)`` comes from
    ``pk_bin_separation_global`` (the s = 0 cell, which that pass drops for p > 0, is added back:
    the reference's bin keeps it).  Each column is then a 1D transform on the host:
    ``(2 ell + 1) rnorm (-1)^(ell / 2) sum_s n_s j_ell(k s) W_in(s) V Qs`` with
    ``W_in = (-1)^(ell_in / 2) / (2 pi)^3 4 pi int k^2 j_ell_in(k s) dk`` over the input bin."""
    from numpy.polynomial import legendre as npleg
    from scipy.special import spherical_jn
    sbin = BinMesh2CorrelationPoles(mattrs, edges=None)
    value = Q if Q is not None else torch.ones(tuple(int(n) for n in mattrs.meshsize), dtype=torch.float32,
                                               device=_device())
    q0 = float(value.reshape(-1)[0])
    ells = bin.ells

    def product(a, b):
        return npleg.legmul([0.] * a + [1.], [0.] * b + [1.])

    orders = sorted({p for ell in ells for ellin in ellsin for p, c in enumerate(product(ell, ellin)) if c != 0})
    sums = {}
    for p0 in range(0, len(orders), 3):
        chunk = orders[p0:p0 + 3]
        got = sbin._sums(value, chunk, los=vlos).cpu().numpy()
        for i, p in enumerate(chunk):
            sums[p] = got[i].copy()
            if p > 0:  # the s = 0 cell, mu = 0
                sums[p][0] += q0 * npleg.legval(0., [0.] * p + [1.])
    snmodes = sbin.nmodes
    with np.errstate(invalid='ignore', divide='ignore'):
        savg = np.where(snmodes == 0, 0., sbin.xavg)
    kout = np.where(bin.nmodes == 0, 0., bin.xavg)
    volume = float(np.prod(mattrs.boxsize.astype('f8')))
    wmat = []
    for ellin in ellsin:
        shells = [_bessel_shell(ellin, float(lo), float(hi), savg) * (-1) ** (ellin // 2) / (2. * np.pi) ** 3
                  for lo, hi in edgesin]
        blocks = []
        for ill, ell in enumerate(ells):
            with np.errstate(invalid='ignore', divide='ignore'):
                Qs = sum(c * sums[p] for p, c in enumerate(product(ell, ellin)) if c != 0) / snmodes
            if ell != 0:
                Qs[0] = 0.
            Qs = np.where(snmodes == 0, 0., Qs)
            jk = spherical_jn(ell, kout[:, None] * savg[None, :]) * snmodes[None, :]
            cols = [(2 * ell + 1) * float(rnorm[ill]) * (-1) ** (ell // 2) * jk.dot(w * volume * Qs) for w in shells]
            blocks.append(np.array(cols))
        wmat.append(np.concatenate(blocks, axis=-1))
    return np.concatenate(wmat, axis=0).T


def _firstpoint_smooth_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm):
    """'smooth' window of the first-point line of sight (``mesh2.py:1196-1238``; a wide-angle
    order n > 0 takes W1 |x|^-n and Q |s|^n, ``mesh2.py:1214``): for each ell_in and output ell,
    ``Qs = 4 pi V_cell sbin(sum_{m, m1} Q_{ell m m1} Y_lm(shat) Y_{ell_in m1}(shat))`` with
    ``Q_{ell m m1} = 4 pi / (2 ell_in + 1) c2r(conj(r2c(W1 Y_lm Y_{ell_in m1})) A0)`` (first bin 0
    for ell > 0), then ``rnorm (-1)^(ell/2) sum_s n_s j_ell(k s) W_in(s) Qs`` per input bin (no
    2 ell + 1 factor on this path).  The Y_lm(shat) weights go through
    ``pk_ylm_separation_accumulate`` (twice: the m1 sum, then the Y_lm factor)."""
    from scipy.special import spherical_jn
    meshsize = mattrs.meshsize
    stream = _lib.stream_handle()
    if swap:
        meshes = meshes[::-1]
    if periodic:
        rmesh1 = torch.ones(tuple(int(n) for n in meshsize), dtype=torch.float32, device=_device())
        A0 = _r2c(rmesh1, meshsize)
    else:
        rmesh1 = _2r(meshes[0]).value.contiguous()
        A0 = _2c(meshes[0] if fields[1] == fields[0] else meshes[1]).value.contiguous()
    offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
    geo = (_lib.i32(meshsize), _lib.f32(mattrs.cellsize), _lib.f32(offset))
    rshape = tuple(int(n) for n in meshsize)
    sbin = BinMesh2CorrelationPoles(mattrs, edges=None)
    snmodes = sbin.nmodes
    with np.errstate(invalid='ignore', divide='ignore'):
        savg = np.where(snmodes == 0, 0., sbin.xavg)
    kout = np.where(bin.nmodes == 0, 0., bin.xavg)
    cellvol = float(np.prod(mattrs.cellsize.astype('f8')))
    ells = bin.ells
    nb = bin.nbins
    r1 = torch.empty((1,) + rshape, dtype=torch.float32, device=_device())
    blocks = []
    rhos = {}
    for ellin, wa in _wide_angle_terms(ellsin):
        n1 = 2 * ellin + 1
        in_ell, in_m = _lib.i32([ellin] * n1), _lib.i32(list(range(-ellin, ellin + 1)))
        rho = _wide_angle_rho(rmesh1, wa, mattrs, offset, rhos)
        R = torch.empty((n1,) + rshape, dtype=torch.float32, device=_device())
        block = np.zeros((len(edgesin), len(ells) * nb))
        shells = [_bessel_shell(ellin, float(lo), float(hi), savg) * (-1) ** (ellin // 2) / (2. * np.pi) ** 3
                  for lo, hi in edgesin.astype('f4')]
        for ill, ell in enumerate(ells):
            carry2 = torch.zeros(rshape, dtype=torch.float32, device=_device())
            for m in range(-ell, ell + 1):
                _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rho), *geo, 1, _lib.i32([ell]), _lib.i32([m]),
                          _lib.ptr(r1))
                _lib.call('pk_ylm_premultiply', stream, _lib.ptr(r1), *geo, n1, in_ell, in_m, _lib.ptr(R))
                F = _r2c(R, meshsize)
                _lib.call('pk_conj_multiply', stream, _lib.ptr(F), _lib.ptr(A0), n1, A0.numel(), _lib.ptr(F))
                G = _c2r(F, meshsize, destroy_input=True)
                del F
                _lib.call('pk_scale_real', stream, _lib.ptr(G), G.numel(), float(4. * np.pi / (2 * ellin + 1)))
                _wide_angle_s(G, n1, wa, mattrs)
                carry1 = torch.zeros(rshape, dtype=torch.float32, device=_device())
                _lib.call('pk_ylm_separation_accumulate', stream, _lib.ptr(G), _lib.i32(meshsize),
                          _lib.f32(mattrs.cellsize), n1, in_ell, in_m, _lib.ptr(carry1))
                _lib.call('pk_ylm_separation_accumulate', stream, _lib.ptr(carry1), _lib.i32(meshsize),
                          _lib.f32(mattrs.cellsize), 1, _lib.i32([ell]), _lib.i32([m]), _lib.ptr(carry2))
                del G, carry1
            Qs = 4. * np.pi * sbin(carry2) * cellvol
            if ell != 0:
                Qs[0] = 0.
            Qs = np.where(snmodes == 0, 0., Qs)
            jk = spherical_jn(ell, kout[:, None] * savg[None, :]) * snmodes[None, :]
            for e, w in enumerate(shells):
                block[e, ill * nb:(ill + 1) * nb] = (-1) ** (ell // 2) * jk.dot(w * Qs) * float(rnorm[ill])
        blocks.append(block)
        del R
    wmat = np.concatenate(blocks, axis=0).T
    if ells[0] % 2:  # the reference keeps the imaginary part of the first multipole's rows: 0 here
        wmat[:nb] = 0.
    return wmat


@functools.lru_cache(maxsize=None)
def _real_gaunt(lm1, lm2, lm3):
    """Integral over the sphere of three real spherical harmonics (the ``real_gaunt`` table of
    ``utils.py:540-622``), by Gauss-Legendre quadrature in cos(theta) and a uniform phi grid
    (exact for these polynomial degrees).  The harmonics follow the library's definition
    (associated Legendre functions with the Condon-Shortley phase, cos(m phi) / sin(|m| phi));
    a (-1)^m convention change leaves every nonzero coefficient unchanged."""
    from scipy.special import lpmv
    x, wx = np.polynomial.legendre.leggauss(16)
    phi = 2. * np.pi * np.arange(48) / 48.

    def Y(ell, m):
        amp = np.sqrt((2 * ell + 1) / (4. * np.pi))
        if m != 0:
            amp *= np.sqrt(2. * math.factorial(ell - abs(m)) / math.factorial(ell + abs(m))) * (-1) ** m
        trig = np.cos(m * phi) if m > 0 else (np.sin(-m * phi) if m < 0 else np.ones_like(phi))
        return amp * lpmv(abs(m), ell, x)[:, None] * trig[None, :]

    return float(np.sum(wx[:, None] * (2. * np.pi / 48.) * Y(*lm1) * Y(*lm2) * Y(*lm3)))


def _local_smooth_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm):
    """'smooth' window with the 'local' theory line of sight (``mesh2.py:1319-1361``, combined into
    the input multipoles as ``:1447-1455``).  For each (ell1, ell2) in {2, 0}^2, output ell and
    p in (0, 2, 4) with a nonzero Gaunt (p 0, ell1 0, ell2 0):
    ``Qs_p = 4 pi V_cell sbin(sum_{m, m1, m2, mp} G(p mp, l1 m1, l2 m2) Y_lm(shat) Y_p mp(shat) Q)``,
    ``Q = (4 pi)^2 / ((2 l1 + 1)(2 l2 + 1)) c2r(conj(r2c(W1 Y_lm Y_l1m1)) r2c(W2 Y_l2m2))``.  The
    Gaunt sums are one small matrix product over the pair meshes (torch); the Y(shat) weights go
    through ``pk_ylm_separation_accumulate``; then host Bessel transforms with the tophat of
    order p."""
    from scipy.special import spherical_jn
    meshsize = mattrs.meshsize
    stream = _lib.stream_handle()
    if any(ell not in (0, 2, 4) for ell in ellsin):
        raise ValueError("the 'local' theory line of sight takes input multipoles among (0, 2, 4)")
    if swap:
        meshes = meshes[::-1]
    if periodic:
        rmesh1 = torch.ones(tuple(int(n) for n in meshsize), dtype=torch.float32, device=_device())
        rmesh2 = rmesh1
    else:
        rmesh1 = _2r(meshes[0]).value.contiguous()
        rmesh2 = rmesh1 if fields[1] == fields[0] else _2r(meshes[1]).value.contiguous()
    offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
    geo = (_lib.i32(meshsize), _lib.f32(mattrs.cellsize), _lib.f32(offset))
    cs = _lib.f32(mattrs.cellsize)
    rshape = tuple(int(n) for n in meshsize)
    cshape = rshape[:2] + (rshape[2] // 2 + 1,)
    nreal = int(np.prod(rshape))
    t2 = [(0, 0)] + [(2, m) for m in range(-2, 3)]
    R2 = torch.empty((len(t2),) + rshape, dtype=torch.float32, device=_device())
    _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rmesh2), *geo, len(t2), _lib.i32([t[0] for t in t2]),
              _lib.i32([t[1] for t in t2]), _lib.ptr(R2))
    B = _r2c(R2, meshsize)
    del R2
    index2 = {t: i for i, t in enumerate(t2)}
    sbin = BinMesh2CorrelationPoles(mattrs, edges=None)
    snmodes = sbin.nmodes
    with np.errstate(invalid='ignore', divide='ignore'):
        savg = np.where(snmodes == 0, 0., sbin.xavg)
    kout = np.where(bin.nmodes == 0, 0., bin.xavg)
    cellvol = float(np.prod(mattrs.cellsize.astype('f8')))
    ells, nb, nin = bin.ells, bin.nbins, len(edgesin)
    coeff2 = {(0, 0): [(0, 1.), (4, -7. / 18.)], (0, 2): [(2, 1. / 2.), (4, -5. / 18.)], (2, 2): [(4, 35. / 18.)]}
    coeff2[2, 0] = coeff2[0, 2]
    r1 = torch.empty((1,) + rshape, dtype=torch.float32, device=_device())
    wmat = np.zeros((len(ellsin), nin, len(ells) * nb))
    for ell1 in (2, 0):
        for ell2 in (2, 0):
            pairs = [(m1, m2) for m1 in range(-ell1, ell1 + 1) for m2 in range(-ell2, ell2 + 1)]
            weight = (4. * np.pi) ** 2 / ((2 * ell1 + 1) * (2 * ell2 + 1))
            n1 = 2 * ell1 + 1
            in_ell, in_m = _lib.i32([ell1] * n1), _lib.i32(list(range(-ell1, ell1 + 1)))
            R = torch.empty((n1,) + rshape, dtype=torch.float32, device=_device())
            P = torch.empty((len(pairs),) + cshape, dtype=torch.complex64, device=_device())
            ps = [p for p in (0, 2, 4) if abs(_real_gaunt((p, 0), (ell1, 0), (ell2, 0))) > 1e-10]
            gaunt = {p: torch.as_tensor(np.array([[_real_gaunt((p, mp), (ell1, m1), (ell2, m2)) for m1, m2 in pairs]
                                                   for mp in range(-p, p + 1)], dtype='f4'), device=_device())
                     for p in ps}
            block = np.zeros((nin, len(ells) * nb))
            for ill, ell in enumerate(ells):
                carry3 = {p: torch.zeros(rshape, dtype=torch.float32, device=_device()) for p in ps}
                for m in range(-ell, ell + 1):
                    _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rmesh1), *geo, 1, _lib.i32([ell]), _lib.i32([m]),
                              _lib.ptr(r1))
                    _lib.call('pk_ylm_premultiply', stream, _lib.ptr(r1), *geo, n1, in_ell, in_m, _lib.ptr(R))
                    F = _r2c(R, meshsize)
                    for q, (m1, m2) in enumerate(pairs):
                        _lib.call('pk_conj_multiply', stream, _lib.ptr(F[m1 + ell1]), _lib.ptr(B[index2[ell2, m2]]), 1,
                                  B[0].numel(), _lib.ptr(P[q]))
                    G = _c2r(P, meshsize) * weight
                    for p in ps:
                        H = torch.tensordot(gaunt[p], G.reshape(len(pairs), nreal), dims=1).contiguous()
                        carry = torch.zeros(rshape, dtype=torch.float32, device=_device())
                        _lib.call('pk_ylm_separation_accumulate', stream, _lib.ptr(H), _lib.i32(meshsize), cs, 2 * p + 1,
                                  _lib.i32([p] * (2 * p + 1)), _lib.i32(list(range(-p, p + 1))), _lib.ptr(carry))
                        _lib.call('pk_ylm_separation_accumulate', stream, _lib.ptr(carry), _lib.i32(meshsize), cs, 1,
                                  _lib.i32([ell]), _lib.i32([m]), _lib.ptr(carry3[p]))
                    del F, G
                jk = (-1) ** (ell // 2) * spherical_jn(ell, kout[:, None] * savg[None, :]) * snmodes[None, :]
                for p in ps:
                    Qp = 4. * np.pi * sbin(carry3[p]) * cellvol
                    if ell != 0:
                        Qp[0] = 0.
                    Qp = np.where(snmodes == 0, 0., Qp)
                    for e, (lo, hi) in enumerate(edgesin.astype('f4')):
                        w = _bessel_shell(p, float(lo), float(hi), savg) * (-1) ** (p // 2) / (2. * np.pi) ** 3
                        block[e, ill * nb:(ill + 1) * nb] += jk.dot(w * Qp) * float(rnorm[ill])
            for illin, ellin in enumerate(ellsin):
                wmat[illin] += sum(c * (ell == ellin) for ell, c in coeff2[ell1, ell2]) * block
    wmat = wmat.reshape(-1, wmat.shape[-1]).T
    if ells[0] % 2:
        wmat[:nb] = 0.
    return wmat


def _local_infinite_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm):
    """'infinite' window with the 'local' theory line of sight (``mesh2.py:1363-1396``, combined
    into the input multipoles as ``:1447-1455``).  For each (ell1, ell2) in {2, 0}^2 and output
    (ell, m): ``C_p = V_cell sum_{m1, m2, mp} G(p mp, l1 m1, l2 m2) Y_p mp(shat) Q`` (the pair
    meshes of the 'local' window, Gaunt sums by one matrix product, ``pk_ylm_separation_accumulate``),
    then per input bin ``4 pi rnorm bin(Y_lm(khat) r2c(sum_p W_p(|s|) C_p))`` with k = 0 dropped
    for ell = 0 only, ``W_p`` the tophat Bessel profile of order p tabulated on the distinct |s|."""
    meshsize = mattrs.meshsize
    stream = _lib.stream_handle()
    if any(ell not in (0, 2, 4) for ell in ellsin):
        raise ValueError("the 'local' theory line of sight takes input multipoles among (0, 2, 4)")
    if swap:
        meshes = meshes[::-1]
    if periodic:
        rmesh1 = torch.ones(tuple(int(n) for n in meshsize), dtype=torch.float32, device=_device())
        rmesh2 = rmesh1
    else:
        rmesh1 = _2r(meshes[0]).value.contiguous()
        rmesh2 = rmesh1 if fields[1] == fields[0] else _2r(meshes[1]).value.contiguous()
    offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
    geo = (_lib.i32(meshsize), _lib.f32(mattrs.cellsize), _lib.f32(offset))
    cs, kf = _lib.f32(mattrs.cellsize), _lib.f32(mattrs.kfun)
    rshape = tuple(int(n) for n in meshsize)
    cshape = rshape[:2] + (rshape[2] // 2 + 1,)
    nreal = int(np.prod(rshape))
    t2 = [(0, 0)] + [(2, m) for m in range(-2, 3)]
    R2 = torch.empty((len(t2),) + rshape, dtype=torch.float32, device=_device())
    _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rmesh2), *geo, len(t2), _lib.i32([t[0] for t in t2]),
              _lib.i32([t[1] for t in t2]), _lib.ptr(R2))
    B = _r2c(R2, meshsize)
    del R2
    index2 = {t: i for i, t in enumerate(t2)}
    sx, sy, sz = mattrs.rcoords(kind='separation', sparse=True)
    snorm = torch.sqrt((sx * sx + sy * sy) + sz * sz)
    uniq, inverse = torch.unique(snorm.reshape(-1), return_inverse=True)
    uniq_h = uniq.cpu().numpy().astype('f8')
    profiles = {}
    for p in (0, 2, 4):
        profiles[p] = [torch.as_tensor((_bessel_shell(p, float(lo), float(hi), uniq_h) * (-1) ** (p // 2)
                                        / (2. * np.pi) ** 3).astype('f4'), device=_device())[inverse].reshape(rshape)
                       for lo, hi in edgesin.astype('f4')]
    cellvol = float(np.prod(mattrs.cellsize.astype('f8')))
    ells, nb, nin = bin.ells, bin.nbins, len(edgesin)
    coeff2 = {(0, 0): [(0, 1.), (4, -7. / 18.)], (0, 2): [(2, 1. / 2.), (4, -5. / 18.)], (2, 2): [(4, 35. / 18.)]}
    coeff2[2, 0] = coeff2[0, 2]
    r1 = torch.empty((1,) + rshape, dtype=torch.float32, device=_device())
    xi = torch.empty(rshape, dtype=torch.float32, device=_device())
    wmat = np.zeros((len(ellsin), nin, len(ells) * nb), dtype='c16')
    for ell1 in (2, 0):
        for ell2 in (2, 0):
            pairs = [(m1, m2) for m1 in range(-ell1, ell1 + 1) for m2 in range(-ell2, ell2 + 1)]
            weight = (4. * np.pi) ** 2 / ((2 * ell1 + 1) * (2 * ell2 + 1))
            n1 = 2 * ell1 + 1
            in_ell, in_m = _lib.i32([ell1] * n1), _lib.i32(list(range(-ell1, ell1 + 1)))
            R = torch.empty((n1,) + rshape, dtype=torch.float32, device=_device())
            P = torch.empty((len(pairs),) + cshape, dtype=torch.complex64, device=_device())
            ps = [p for p in (0, 2, 4) if abs(_real_gaunt((p, 0), (ell1, 0), (ell2, 0))) > 1e-10]
            gaunt = {p: torch.as_tensor(np.array([[_real_gaunt((p, mp), (ell1, m1), (ell2, m2)) for m1, m2 in pairs]
                                                   for mp in range(-p, p + 1)], dtype='f4'), device=_device())
                     for p in ps}
            block = np.zeros((nin, len(ells) * nb), dtype='c16')
            for ill, ell in enumerate(ells):
                for m in range(-ell, ell + 1):
                    _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rmesh1), *geo, 1, _lib.i32([ell]), _lib.i32([m]),
                              _lib.ptr(r1))
                    _lib.call('pk_ylm_premultiply', stream, _lib.ptr(r1), *geo, n1, in_ell, in_m, _lib.ptr(R))
                    F = _r2c(R, meshsize)
                    for q, (m1, m2) in enumerate(pairs):
                        _lib.call('pk_conj_multiply', stream, _lib.ptr(F[m1 + ell1]), _lib.ptr(B[index2[ell2, m2]]), 1,
                                  B[0].numel(), _lib.ptr(P[q]))
                    G = _c2r(P, meshsize) * (weight * cellvol)
                    C = {}
                    for p in ps:
                        H = torch.tensordot(gaunt[p], G.reshape(len(pairs), nreal), dims=1).contiguous()
                        C[p] = torch.zeros(rshape, dtype=torch.float32, device=_device())
                        _lib.call('pk_ylm_separation_accumulate', stream, _lib.ptr(H), _lib.i32(meshsize), cs, 2 * p + 1,
                                  _lib.i32([p] * (2 * p + 1)), _lib.i32(list(range(-p, p + 1))), _lib.ptr(C[p]))
                    del F, G
                    for e in range(nin):
                        xi.zero_()
                        for p in ps:
                            xi.add_(profiles[p][e] * C[p])
                        A = _r2c(xi, meshsize)
                        Aell = torch.zeros(cshape, dtype=torch.complex64, device=_device())
                        _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(A), _lib.i32(meshsize), kf, 1,
                                  _lib.i32([ell]), _lib.i32([m]), 1., 0, _lib.ptr(Aell))
                        block[e, ill * nb:(ill + 1) * nb] += 4. * np.pi * bin(Aell, remove_zero=ell == 0) * float(rnorm[ill])
            for illin, ellin in enumerate(ellsin):
                wmat[illin] += sum(c * (ell == ellin) for ell, c in coeff2[ell1, ell2]) * block
    wmat = wmat.reshape(-1, wmat.shape[-1]).T
    first = wmat[:nb].imag if ells[0] % 2 else wmat[:nb].real
    wmat = wmat.real.copy()
    wmat[:nb] = first
    return wmat


def _firstpoint_infinite_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm):
    """'infinite' window of the first-point line of sight (``mesh2.py:1240-1262``; a wide-angle
    order n > 0 takes W1 |x|^-n and Q |s|^n, ``mesh2.py:1249``): for each ell_in and output (ell, m),
    ``C_{ell m} = V_cell sum_m1 Y_{ell_in m1}(shat) Q_{ell m m1}`` (``pk_ylm_separation_accumulate``),
    then per input bin ``4 pi rnorm bin(sum_m r2c(W_in(|s|) C_{ell m}) Y_lm(khat))`` with k = 0
    dropped for ell = 0 only, ``W_in`` the tophat Bessel profile tabulated on the distinct |s|."""
    meshsize = mattrs.meshsize
    stream = _lib.stream_handle()
    if swap:
        meshes = meshes[::-1]
    if periodic:
        rmesh1 = torch.ones(tuple(int(n) for n in meshsize), dtype=torch.float32, device=_device())
        A0 = _r2c(rmesh1, meshsize)
    else:
        rmesh1 = _2r(meshes[0]).value.contiguous()
        A0 = _2c(meshes[0] if fields[1] == fields[0] else meshes[1]).value.contiguous()
    offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
    geo = (_lib.i32(meshsize), _lib.f32(mattrs.cellsize), _lib.f32(offset))
    kf = _lib.f32(mattrs.kfun)
    rshape = tuple(int(n) for n in meshsize)
    cshape = rshape[:2] + (rshape[2] // 2 + 1,)
    sx, sy, sz = mattrs.rcoords(kind='separation', sparse=True)
    snorm = torch.sqrt((sx * sx + sy * sy) + sz * sz)
    uniq, inverse = torch.unique(snorm.reshape(-1), return_inverse=True)
    uniq_h = uniq.cpu().numpy().astype('f8')
    cellvol = float(np.prod(mattrs.cellsize.astype('f8')))
    ells = bin.ells
    nb = bin.nbins
    out_terms = [(ell, m) for ell in ells for m in range(-ell, ell + 1)]
    r1 = torch.empty((1,) + rshape, dtype=torch.float32, device=_device())
    col = torch.empty(rshape, dtype=torch.float32, device=_device())
    blocks = []
    rhos = {}
    for ellin, wa in _wide_angle_terms(ellsin):
        n1 = 2 * ellin + 1
        in_ell, in_m = _lib.i32([ellin] * n1), _lib.i32(list(range(-ellin, ellin + 1)))
        rho = _wide_angle_rho(rmesh1, wa, mattrs, offset, rhos)
        R = torch.empty((n1,) + rshape, dtype=torch.float32, device=_device())
        C = torch.zeros((len(out_terms),) + rshape, dtype=torch.float32, device=_device())
        for t, (ell, m) in enumerate(out_terms):
            _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rho), *geo, 1, _lib.i32([ell]), _lib.i32([m]),
                      _lib.ptr(r1))
            _lib.call('pk_ylm_premultiply', stream, _lib.ptr(r1), *geo, n1, in_ell, in_m, _lib.ptr(R))
            F = _r2c(R, meshsize)
            _lib.call('pk_conj_multiply', stream, _lib.ptr(F), _lib.ptr(A0), n1, A0.numel(), _lib.ptr(F))
            G = _c2r(F, meshsize, destroy_input=True)
            del F
            _lib.call('pk_scale_real', stream, _lib.ptr(G), G.numel(), float(4. * np.pi / (2 * ellin + 1) * cellvol))
            _wide_angle_s(G, n1, wa, mattrs)
            _lib.call('pk_ylm_separation_accumulate', stream, _lib.ptr(G), _lib.i32(meshsize),
                      _lib.f32(mattrs.cellsize), n1, in_ell, in_m, _lib.ptr(C[t]))
            del G
        block = np.zeros((len(edgesin), len(ells) * nb))
        for e, (lo, hi) in enumerate(edgesin.astype('f4')):
            prof = _bessel_shell(ellin, float(lo), float(hi), uniq_h) * (-1) ** (ellin // 2) / (2. * np.pi) ** 3
            profile = torch.as_tensor(prof.astype('f4'), device=_device())[inverse].reshape(rshape)
            for ill, ell in enumerate(ells):
                Aell = torch.zeros(cshape, dtype=torch.complex64, device=_device())
                for m in range(-ell, ell + 1):
                    torch.mul(profile, C[out_terms.index((ell, m))], out=col)
                    Ft = _r2c(col, meshsize)
                    _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(Ft), _lib.i32(meshsize), kf, 1,
                              _lib.i32([ell]), _lib.i32([m]), 1., 1, _lib.ptr(Aell))
                value = 4. * np.pi * bin(Aell, remove_zero=ell == 0) * float(rnorm[ill])
                block[e, ill * nb:(ill + 1) * nb] = value.imag if (ill == 0 and ell % 2) else value.real
        blocks.append(block)
        del C, R
    return np.concatenate(blocks, axis=0).T


def _infinite_window(mattrs, bin, Q, vlos, ellsin, edgesin, rnorm, batch_size=None):
    """'infinite' window of the global line of sight (``mesh2.py:1095-1107``): column
    (ell_in, [k_lo, k_hi]) is the estimator applied to ``r2c(Q V W_in(|s|) L_ell_in(mu_s))``,
    ``W_in = (-1)^(ell_in / 2) / (2 pi)^3 4 pi int k^2 j_ell_in(k s) dk`` (the theory correlation
    function of a tophat power spectrum, no mesh resolution limit).  The radial profile is
    tabulated on the host on the distinct |s| of the separation grid and gathered onto the
    mesh with torch; the columns then go through one batched cuFFT R2C and the fused binning
    pass linear in the mesh (``pk_bin_window_batch``, k = 0 dropped)."""
    stream = _lib.stream_handle()
    meshsize = mattrs.meshsize
    sx, sy, sz = mattrs.rcoords(kind='separation', sparse=True)
    s2 = (sx * sx + sy * sy) + sz * sz
    snorm = torch.sqrt(s2)
    smu = (sx * float(vlos[0]) + sy * float(vlos[1]) + sz * float(vlos[2])) / \
        torch.where(snorm == 0., torch.ones_like(snorm), snorm)
    uniq, inverse = torch.unique(snorm.reshape(-1), return_inverse=True)
    uniq_h = uniq.cpu().numpy().astype('f8')
    volume = float(np.prod(mattrs.boxsize.astype('f8')))
    ells = bin.ells
    even = [ill for ill, ell in enumerate(ells) if ell % 2 == 0]
    nin, nb = len(edgesin), bin.nbins
    rshape = tuple(int(n) for n in meshsize)
    B = _window_batch(mattrs, batch_size)
    sums = np.zeros((len(ellsin), nin, len(ells), nb))
    if even:
        nbytes = _lib.c_size_t()
        _lib.call('pk_bin_batch_workspace_size', _lib.i32(meshsize), len(bin._edges1d), len(even), B,
                  _lib.ctypes.byref(nbytes))
        ws = _workspace(nbytes.value)
        raw = torch.empty((B, len(even), nb), dtype=torch.float64, device=_device())
    for iin, ellin in enumerate(ellsin):
        legin = _legendre(ellin, smu).reshape(-1) * volume
        if Q is not None:
            legin = legin * Q.reshape(-1)
        for e0 in range(0, nin if even else 0, B):
            n = min(B, nin - e0)
            cols = torch.empty((n,) + rshape, dtype=torch.float32, device=_device())
            for c in range(n):
                lo, hi = edgesin[e0 + c]
                prof = _bessel_shell(ellin, float(np.float32(lo)), float(np.float32(hi)), uniq_h)
                prof = prof * (-1) ** (ellin // 2) / (2. * np.pi) ** 3
                table = torch.as_tensor(prof.astype('f4'), device=_device())
                cols[c].view(-1).copy_(table[inverse] * legin)
            A = _r2c(cols, meshsize)
            del cols
            _lib.call('pk_bin_window_batch', stream, _lib.ptr(A), n, _lib.i32(meshsize), _lib.f32(mattrs.kfun),
                      _lib.f32(vlos), _lib.ptr(bin.d_edges), len(bin._edges1d), bin._step, mattrs.backend_code,
                      len(even), _lib.i32([ells[ill] for ill in even]), 1, _lib.ptr(raw), _lib.ptr(ws), ws.numel())
            sums[iin, e0:e0 + n][:, even] = raw[:n].cpu().numpy()
            del A
    with np.errstate(invalid='ignore', divide='ignore'):
        factor = np.array([(2 * ell + 1) / (1 + ell % 2) * float(rnorm[ill]) for ill, ell in enumerate(ells)])
        spectra = sums / bin.nmodes * factor[:, None]
    return np.concatenate([spectra[iin].reshape(nin, -1) for iin in range(len(ellsin))], axis=0).T


def _local_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm):
    """Window matrix with the 'local' theory line of sight (``mesh2.py:1398-1455``).  For each
    (ell1, ell2) in {2, 0}^2 and output (ell, m), the (m1, m2) pairs give
    ``Q = (4 pi)^2 / ((2 ell1 + 1) (2 ell2 + 1)) c2r(conj(r2c(W1 Y_lm Y_l1m1)) r2c(W2 Y_l2m2))``;
    each input bin [k_lo, k_hi] (ends included) gives
    ``xi = c2r(1{shell} Y_l1m1(khat) Y_l2m2(-khat))`` per pair and the block column
    ``4 pi rnorm bin(sum_m r2c(sum_pairs xi Q) Y_lm(khat))`` (k = 0 dropped for ell = 0).  The
    blocks combine into the input multipoles 0, 2, 4 with the coefficients of L_ell1 L_ell2 on
    L_0, L_2, L_4."""
    if any(ell not in (0, 2, 4) for ell in ellsin):
        raise ValueError("the 'local' theory line of sight takes input multipoles among (0, 2, 4)")
    meshsize = mattrs.meshsize
    stream = _lib.stream_handle()
    if swap:
        meshes = meshes[::-1]
    if periodic:
        rmesh1 = torch.ones(tuple(int(n) for n in meshsize), dtype=torch.float32, device=_device())
        rmesh2 = rmesh1
    else:
        rmesh1 = _2r(meshes[0]).value.contiguous()
        rmesh2 = rmesh1 if fields[1] == fields[0] else _2r(meshes[1]).value.contiguous()
    offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
    geo = (_lib.i32(meshsize), _lib.f32(mattrs.cellsize), _lib.f32(offset))
    kf = _lib.f32(mattrs.kfun)
    cshape = tuple(int(n) for n in meshsize[:2]) + (int(meshsize[2]) // 2 + 1,)
    rshape = tuple(int(n) for n in meshsize)
    nreal = int(np.prod(rshape))
    ells = bin.ells
    out_terms = [(ell, m) for ell in ells for m in range(-ell, ell + 1)]
    kvec = mattrs.kcoords(sparse=True)
    knorm = torch.sqrt(kvec[0] ** 2 + kvec[1] ** 2 + kvec[2] ** 2)
    # B_{l2 m2} = r2c(W2 Y_l2m2(xhat)), l2 in (0, 2)
    t2 = [(0, 0)] + [(2, m) for m in range(-2, 3)]
    R2 = torch.empty((len(t2),) + rshape, dtype=torch.float32, device=_device())
    _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rmesh2), *geo, len(t2), _lib.i32([t[0] for t in t2]),
              _lib.i32([t[1] for t in t2]), _lib.ptr(R2))
    B = _r2c(R2, meshsize)
    del R2
    index2 = {t: i for i, t in enumerate(t2)}
    coeff2 = {(0, 0): [(0, 1.), (4, -7. / 18.)], (0, 2): [(2, 1. / 2.), (4, -5. / 18.)], (2, 2): [(4, 35. / 18.)]}
    coeff2[2, 0] = coeff2[0, 2]
    r1 = torch.empty((1,) + rshape, dtype=torch.float32, device=_device())
    tmp = torch.empty(rshape, dtype=torch.float32, device=_device())
    one = torch.empty((1,) + cshape, dtype=torch.complex64, device=_device())
    nin, nb = len(edgesin), bin.nbins
    wmat = np.zeros((len(ellsin), nin, len(ells) * nb), dtype='c16')
    for ell1 in (2, 0):
        for ell2 in (2, 0):
            pairs = [((ell1, m1), (ell2, m2)) for m1 in range(-ell1, ell1 + 1) for m2 in range(-ell2, ell2 + 1)]
            npair = len(pairs)
            weight = np.full(npair, (4. * np.pi) ** 2 / ((2 * ell1 + 1) * (2 * ell2 + 1)), dtype='f4')
            n1 = 2 * ell1 + 1
            in_ell, in_m = _lib.i32([ell1] * n1), _lib.i32(list(range(-ell1, ell1 + 1)))
            R = torch.empty((n1,) + rshape, dtype=torch.float32, device=_device())
            Q = torch.empty((len(out_terms), npair) + rshape, dtype=torch.float32, device=_device())
            P = torch.empty((npair,) + cshape, dtype=torch.complex64, device=_device())
            for t, (ell, m) in enumerate(out_terms):
                _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rmesh1), *geo, 1, _lib.i32([ell]), _lib.i32([m]),
                          _lib.ptr(r1))
                _lib.call('pk_ylm_premultiply', stream, _lib.ptr(r1), *geo, n1, in_ell, in_m, _lib.ptr(R))
                F = _r2c(R, meshsize)
                for p, ((_, m1), t2p) in enumerate(pairs):
                    _lib.call('pk_conj_multiply', stream, _lib.ptr(F[m1 + ell1]), _lib.ptr(B[index2[t2p]]), 1,
                              B[0].numel(), _lib.ptr(P[p]))
                Q[t] = _c2r(P, meshsize, destroy_input=True)
                del F
            block = np.zeros((nin, len(ells) * nb), dtype='c16')
            for e, (lo, hi) in enumerate(edgesin.astype('f4')):
                tophat = ((knorm >= float(lo)) & (knorm <= float(hi))).to(torch.complex64)
                xi_c = torch.empty((npair,) + cshape, dtype=torch.complex64, device=_device())
                for p, ((l1, m1), (l2, m2)) in enumerate(pairs):
                    _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(tophat), _lib.i32(meshsize), kf, 1,
                              _lib.i32([l1]), _lib.i32([m1]), 1., 0, _lib.ptr(one))
                    _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(one), _lib.i32(meshsize), kf, 1,
                              _lib.i32([l2]), _lib.i32([m2]), 1., 0, _lib.ptr(xi_c[p]))
                xi = _c2r(xi_c, meshsize, destroy_input=True)
                del xi_c
                spectrum = []
                for ill, ell in enumerate(ells):
                    Aell = torch.zeros(cshape, dtype=torch.complex64, device=_device())
                    for m in range(-ell, ell + 1):
                        t = out_terms.index((ell, m))
                        _lib.call('pk_sum_products', stream, _lib.ptr(tmp), _lib.ptr(xi), _lib.ptr(Q[t]), npair,
                                  _lib.f32(weight), nreal, 0)
                        Ft = _r2c(tmp, meshsize)
                        _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(Ft), _lib.i32(meshsize), kf, 1,
                                  _lib.i32([ell]), _lib.i32([m]), 1., 1, _lib.ptr(Aell))
                    spectrum.append(4. * np.pi * bin(Aell, remove_zero=ell == 0) * float(rnorm[ill]))
                block[e] = np.concatenate(spectrum)
            del Q, R, P
            for illin, ellin in enumerate(ellsin):
                coeff = sum(c * (ell == ellin) for ell, c in coeff2[ell1, ell2])
                wmat[illin] += coeff * block
    wmat = wmat.reshape(-1, wmat.shape[-1]).T
    first = wmat[:nb].imag if ells[0] % 2 else wmat[:nb].real
    wmat = wmat.real.copy()
    wmat[:nb] = first
    return wmat


def _firstpoint_window(meshes, fields, periodic, mattrs, bin, edgesin, ellsin, swap, rnorm, batch_size=None):
    """First-point window matrix, input power on the mesh (``mesh2.py:1264-1304``,
    ``1462-1470``).  For each input (ell_in, wide-angle order n) (n = 0 for a plain ell_in; for
    n > 0 W1 is W1 |x|^-n and each Q is multiplied by |s|^n, ``mesh2.py:1273``):

        Q_{ell m m1} = 4 pi / (2 ell_in + 1) c2r(conj(r2c(W1 Y_lm(xhat) Y_{ell_in m1}(xhat))) A0),

    kept for every output (ell, m); then per input bin [k_lo, k_hi] (both ends included),
    ``xi_m1 = c2r(1{k_lo <= |k| <= k_hi} Y_{ell_in m1}(khat))``,
    ``A_ell = sum_m r2c(sum_m1 xi_m1 Q_{ell m m1}) Y_lm(khat)`` and the column is
    ``4 pi rnorm bin(A_ell)`` with k = 0 dropped for ell = 0 only (``remove_zero=ell == 0``).
    The real part is kept, but the first multipole's rows take the imaginary part when that
    multipole is odd (``mesh2.py:1464-1469`` advances only over the first multipole)."""
    meshsize = mattrs.meshsize
    stream = _lib.stream_handle()
    if swap:
        meshes = meshes[::-1]
    if periodic:
        rmesh1 = torch.ones(tuple(int(n) for n in meshsize), dtype=torch.float32, device=_device())
        A0 = _r2c(rmesh1, meshsize)
    else:
        rmesh1 = _2r(meshes[0]).value.contiguous()
        A0 = _2c(meshes[0] if fields[1] == fields[0] else meshes[1]).value.contiguous()
    offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
    geo = (_lib.i32(meshsize), _lib.f32(mattrs.cellsize), _lib.f32(offset))
    kf = _lib.f32(mattrs.kfun)
    cshape = tuple(int(n) for n in meshsize[:2]) + (int(meshsize[2]) // 2 + 1,)
    rshape = tuple(int(n) for n in meshsize)
    nreal = int(np.prod(rshape))
    ells = bin.ells
    out_terms = [(ell, m) for ell in ells for m in range(-ell, ell + 1)]
    kvec = mattrs.kcoords(sparse=True)
    knorm = torch.sqrt(kvec[0] ** 2 + kvec[1] ** 2 + kvec[2] ** 2)
    r1 = torch.empty((1,) + rshape, dtype=torch.float32, device=_device())
    blocks = []
    rhos = {}
    for ellin, wa in _wide_angle_terms(ellsin):
        n1 = 2 * ellin + 1
        if n1 > 32:
            raise NotImplementedError('ell_in <= 15')
        in_ell, in_m = _lib.i32([ellin] * n1), _lib.i32(list(range(-ellin, ellin + 1)))
        rho = _wide_angle_rho(rmesh1, wa, mattrs, offset, rhos)
        # Q[t] for output term t: (n1, N) real meshes
        Q = torch.empty((len(out_terms), n1) + rshape, dtype=torch.float32, device=_device())
        R = torch.empty((n1,) + rshape, dtype=torch.float32, device=_device())
        for t, (ell, m) in enumerate(out_terms):
            _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rho), *geo, 1, _lib.i32([ell]), _lib.i32([m]),
                      _lib.ptr(r1))
            _lib.call('pk_ylm_premultiply', stream, _lib.ptr(r1), *geo, n1, in_ell, in_m, _lib.ptr(R))
            F = _r2c(R, meshsize)
            _lib.call('pk_conj_multiply', stream, _lib.ptr(F), _lib.ptr(A0), n1, A0.numel(), _lib.ptr(F))
            Q[t] = _c2r(F, meshsize, destroy_input=True)
            _wide_angle_s(Q[t], n1, wa, mattrs)
            del F
        coef = np.full(n1, 4. * np.pi / (2 * ellin + 1), dtype='f4')
        rows = []
        tmp = torch.empty(rshape, dtype=torch.float32, device=_device())
        for lo, hi in edgesin.astype('f4'):
            tophat = ((knorm >= float(lo)) & (knorm <= float(hi))).to(torch.complex64)
            xi_c = torch.empty((n1,) + cshape, dtype=torch.complex64, device=_device())
            _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(tophat), _lib.i32(meshsize), kf, n1, in_ell, in_m, 1.,
                      0, _lib.ptr(xi_c))
            xi = _c2r(xi_c, meshsize, destroy_input=True)
            del xi_c
            spectrum = []
            for ill, ell in enumerate(ells):
                Aell = torch.zeros(cshape, dtype=torch.complex64, device=_device())
                for m in range(-ell, ell + 1):
                    t = out_terms.index((ell, m))
                    _lib.call('pk_sum_products', stream, _lib.ptr(tmp), _lib.ptr(xi), _lib.ptr(Q[t]), n1,
                              _lib.f32(coef), nreal, 0)
                    Ft = _r2c(tmp, meshsize)
                    _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(Ft), _lib.i32(meshsize), kf, 1,
                              _lib.i32([ell]), _lib.i32([m]), 1., 1, _lib.ptr(Aell))
                spectrum.append(4. * np.pi * bin(Aell, remove_zero=ell == 0) * float(rnorm[ill]))
            rows.append(np.concatenate(spectrum))
        blocks.append(np.array(rows))
        del Q, R
    wmat = np.concatenate(blocks, axis=0).T
    nb = bin.nbins
    first = wmat[:nb].imag if ells[0] % 2 else wmat[:nb].real
    wmat = wmat.real.copy()
    wmat[:nb] = first
    return wmat


_LEGENDRE_COEFS = {0: (1.,), 1: (0., 1.), 2: (-1. / 2., 0., 3. / 2.), 3: (0., -3. / 2., 0., 5. / 2.),
                   4: (3. / 8., 0., -15. / 4., 0., 35. / 8.), 5: (0., 15. / 8., 0., -35. / 4., 0., 63. / 8.),
                   6: (-5. / 16., 0., 105. / 16., 0., -315. / 16., 0., 231. / 16.),
                   7: (0., -35. / 16., 0., 315. / 16., 0., -693. / 16., 0., 429. / 16.),
                   8: (35. / 128., 0., -315. / 32., 0., 3465. / 64., 0., -3003. / 32., 0., 6435. / 128.)}


def _legendre(ell, x):
    """L_ell(x) (``utils.py:341-352``) of a device tensor, for theory evaluation on the k grid."""
    out = torch.zeros_like(x)
    for c in reversed(_LEGENDRE_COEFS[ell]):
        out = out * x + c
    return out


def _theory_poles(theory):
    """Split the ``theory`` argument of compute_mesh2_spectrum_mean (``mesh2.py:1538-1566``)."""
    poles, kin, theory_los = theory, None, 'firstpoint'
    if isinstance(poles, tuple) and isinstance(poles[-1], str):
        theory_los = poles[-1]
        if theory_los not in ('firstpoint', 'local'):
            raise NotImplementedError("theory line of sight '{}' is not supported".format(theory_los))
        poles = poles[0] if len(poles) == 2 else poles[:-1]
    if isinstance(poles, tuple):
        kin, poles = poles
    if isinstance(poles, Mesh2SpectrumPoles):
        edges = np.asarray(next(iter(poles)).k_edges, dtype='f8')
        kin = np.append(edges[..., 0], edges[-1, 1])
        poles = {ell: poles.get(ell).value() for ell in poles.ells}
    if isinstance(poles, list):
        poles = {ell: pole for ell, pole in zip((0, 2, 4), poles)}
    return kin, poles, theory_los


def _local_theory_pairs(poles, get_theory, rnorm):
    """Kernels of the 'local' theory line of sight (``mesh2.py:1647-1661``): for (ell1, ell2) in
    {0, 2}^2, K = rnorm sum coeff P_ell (coefficients of L_ell1 L_ell2 on L_0, L_2, L_4), and every
    (ell1 m1, ell2 m2) pair with its weight (4 pi)^2 / ((2 ell1 + 1) (2 ell2 + 1))."""
    coeff2 = {(0, 0): [(0, 1.), (4, -7. / 18.)], (0, 2): [(2, 1. / 2.), (4, -5. / 18.)], (2, 2): [(4, 35. / 18.)]}
    coeff2[2, 0] = coeff2[0, 2]
    pairs = []
    for ell1 in (0, 2):
        for ell2 in (0, 2):
            kernel = sum(coeff * get_theory(poles[ell, 0]) for ell, coeff in coeff2[ell1, ell2]) * rnorm
            weight = (4. * np.pi) ** 2 / ((2 * ell1 + 1) * (2 * ell2 + 1))
            for m1 in range(-ell1, ell1 + 1):
                for m2 in range(-ell2, ell2 + 1):
                    pairs.append(((ell1, m1), (ell2, m2), kernel, weight))
    return pairs


def _firstpoint_mean(meshes, fields, periodic, mattrs, bin, poles, get_theory, swap, N, norm, rnorm,
                     theory_los='firstpoint'):
    """First-point branch of compute_mesh2_spectrum_mean (``mesh2.py:1607-1669``, theory line of
    sight 'firstpoint'; theory keys ell or (ell, wide-angle order)).  For each output (ell, m):

        Q = sum over theory (ell1, m1) of 4 pi / (2 ell1 + 1) xi_{ell1 m1} G,
        xi_{ell1 m1} = c2r(P_ell1(k) rnorm Y_{ell1 m1}(khat)),
        G = c2r(conj(r2c(W1 Y_{ell m}(xhat) Y_{ell1 m1}(xhat))) A0),   A0 = r2c(W2),
        A_ell += r2c(Q) Y_{ell m}(khat),

    then 4 pi bin(A_ell) (k = 0 kept), real part for even ell, imaginary for odd, conjugated
    for the end point.  W = 1 for a periodic box.  Kernels: pk_ylm_premultiply (twice, for
    the product of two Y_lm), cuFFT, pk_conj_multiply, pk_sum_products, pk_ylm_kgrid_multiply,
    pk_bin_mesh."""
    if not isinstance(poles, dict):
        raise NotImplementedError('the first-point mean spectrum takes theory multipoles, not a callable of k')
    poles = {(ell if isinstance(ell, tuple) else (ell, 0)): pole for ell, pole in poles.items()}
    if theory_los == 'local' and any(wa != 0 for _, wa in poles):
        raise NotImplementedError("wide-angle orders > 0 with the 'local' theory line of sight are not supported")
    meshsize = mattrs.meshsize
    stream = _lib.stream_handle()
    if swap:
        meshes = meshes[::-1]
    if periodic:
        rmesh1 = torch.ones(tuple(int(n) for n in meshsize), dtype=torch.float32, device=_device())
        A0 = _r2c(rmesh1, meshsize)
    else:
        rmesh1 = _2r(meshes[0]).value.contiguous()
        A0 = _2c(meshes[0] if fields[1] == fields[0] else meshes[1]).value.contiguous()
    offset = (mattrs.boxcenter - (mattrs.boxsize / np.float32(2.)).astype('f4')).astype('f4')
    cshape = tuple(int(n) for n in meshsize[:2]) + (int(meshsize[2]) // 2 + 1,)
    rshape = tuple(int(n) for n in meshsize)
    nreal = int(np.prod(rshape))
    geo = (_lib.i32(meshsize), _lib.f32(mattrs.cellsize), _lib.f32(offset))
    if theory_los == 'local':
        return _local_mean(rmesh1, A0, meshes, fields, periodic, mattrs, bin, poles, get_theory, swap, norm, rnorm,
                           geo)
    # per wide-angle order wa: the theory terms, their xi_{ell1 m1} = c2r(P rnorm Y(khat)) s^wa, and
    # the mesh W1 |x|^-wa that the Y_lm(xhat) products start from (mesh2.py:1641-1645)
    was = sorted({wa for _, wa in poles})
    rhos = {}
    groups = []
    for wa in was:
        terms1 = [(ell1, m1) for (ell1, w) in poles if w == wa for m1 in range(-ell1, ell1 + 1)]
        if len(terms1) > 32:
            raise NotImplementedError('at most 32 theory (ell, m) terms per wide-angle order')
        coef = np.array([4. * np.pi / (2 * ell1 + 1) for ell1, _ in terms1], dtype='f4')
        xi_c = torch.empty((len(terms1),) + cshape, dtype=torch.complex64, device=_device())
        t0 = 0
        for (ell1, w), pole in poles.items():
            if w != wa:
                continue
            kernel = torch.zeros(cshape, dtype=torch.complex64, device=_device())
            kernel.real.copy_((get_theory(pole) * rnorm).to(torch.float32).expand(cshape))
            n1 = 2 * ell1 + 1
            _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(kernel), _lib.i32(meshsize), _lib.f32(mattrs.kfun), n1,
                      _lib.i32([ell1] * n1), _lib.i32(list(range(-ell1, ell1 + 1))), 1., 0, _lib.ptr(xi_c[t0:t0 + n1]))
            t0 += n1
        xi = _c2r(xi_c, meshsize, destroy_input=True)
        del xi_c
        _wide_angle_s(xi, len(terms1), wa, mattrs)
        rho = _wide_angle_rho(rmesh1, wa, mattrs, offset, rhos)
        groups.append((rho, terms1, coef, xi,
                       torch.empty((len(terms1),) + rshape, dtype=torch.float32, device=_device())))
    num = []
    r1 = torch.empty((1,) + rshape, dtype=torch.float32, device=_device())
    Q = torch.empty(rshape, dtype=torch.float32, device=_device())
    for ell in bin.ells:
        Aell = torch.zeros(cshape, dtype=torch.complex64, device=_device())
        for m in range(-ell, ell + 1):
            for gi, (rho, terms1, coef, xi, R) in enumerate(groups):
                _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rho), *geo, 1, _lib.i32([ell]), _lib.i32([m]),
                          _lib.ptr(r1))
                _lib.call('pk_ylm_premultiply', stream, _lib.ptr(r1), *geo, len(terms1),
                          _lib.i32([t[0] for t in terms1]), _lib.i32([t[1] for t in terms1]), _lib.ptr(R))
                F = _r2c(R, meshsize)
                _lib.call('pk_conj_multiply', stream, _lib.ptr(F), _lib.ptr(A0), len(terms1), A0.numel(), _lib.ptr(F))
                G = _c2r(F, meshsize, destroy_input=True)
                del F
                _lib.call('pk_sum_products', stream, _lib.ptr(Q), _lib.ptr(xi), _lib.ptr(G), len(terms1),
                          _lib.f32(coef), nreal, int(gi > 0))
                del G
            FQ = _r2c(Q, meshsize)
            _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(FQ), _lib.i32(meshsize), _lib.f32(mattrs.kfun), 1,
                      _lib.i32([ell]), _lib.i32([m]), 1., 1, _lib.ptr(Aell))
            del FQ
        value = bin(Aell)  # per-bin mean, k = 0 kept
        value = 4. * np.pi * value
        if swap:
            value = np.conj(value)
        num.append(value.real if ell % 2 == 0 else value.imag)
    volume = float(np.prod(mattrs.kfun.astype('f8'))) * bin.nmodes
    return Mesh2SpectrumPoles([Mesh2SpectrumPole(k=bin.xavg, k_edges=bin.edges, nmodes=bin.nmodes, num_raw=num[ill],
                                                 norm=np.ones(bin.nbins) * norm, volume=volume, ell=ell,
                                                 attrs=dict(los='firstpoint' if not swap else 'endpoint'))
                               for ill, ell in enumerate(bin.ells)])


def _local_mean(rmesh1, A0, meshes, fields, periodic, mattrs, bin, poles, get_theory, swap, norm, rnorm, geo):
    """'local' theory line of sight of the first-point mean spectrum (``mesh2.py:1646-1661``):
    for each output (ell, m), Q = sum over pairs (l1 m1, l2 m2) of
    w xi_pair c2r(conj(r2c(W1 Y_lm Y_l1m1)) r2c(W2 Y_l2m2)), with
    xi_pair = c2r(K_l1l2(k) Y_l1m1(khat) Y_l2m2(-khat)) (ell2 even: Y_l2m2(-khat) = Y_l2m2(khat))."""
    meshsize = mattrs.meshsize
    stream = _lib.stream_handle()
    cshape = tuple(int(n) for n in meshsize[:2]) + (int(meshsize[2]) // 2 + 1,)
    rshape = tuple(int(n) for n in meshsize)
    nreal = int(np.prod(rshape))
    kf = _lib.f32(mattrs.kfun)
    if periodic:
        rmesh2 = rmesh1
    else:
        rmesh2 = rmesh1 if fields[1] == fields[0] else _2r(meshes[1]).value.contiguous()
    terms = [(0, 0)] + [(2, m) for m in range(-2, 3)]
    t_ell, t_m = _lib.i32([t[0] for t in terms]), _lib.i32([t[1] for t in terms])
    # B_{l2 m2} = r2c(W2 Y_l2m2(xhat))
    R = torch.empty((len(terms),) + rshape, dtype=torch.float32, device=_device())
    _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rmesh2), *geo, len(terms), t_ell, t_m, _lib.ptr(R))
    B = _r2c(R, meshsize)
    pairs = _local_theory_pairs(poles, get_theory, rnorm)
    # xi of every pair, in pair order
    xi_c = torch.empty((len(pairs),) + cshape, dtype=torch.complex64, device=_device())
    tmp = torch.empty((1,) + cshape, dtype=torch.complex64, device=_device())
    for p, ((l1, m1), (l2, m2), kernel, _) in enumerate(pairs):
        kc = torch.zeros(cshape, dtype=torch.complex64, device=_device())
        kc.real.copy_(torch.as_tensor(kernel, device=_device()).to(torch.float32).expand(cshape))
        _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(kc), _lib.i32(meshsize), kf, 1, _lib.i32([l1]),
                  _lib.i32([m1]), 1., 0, _lib.ptr(tmp))
        _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(tmp), _lib.i32(meshsize), kf, 1, _lib.i32([l2]),
                  _lib.i32([m2]), 1., 0, _lib.ptr(xi_c[p]))
    xi = _c2r(xi_c, meshsize, destroy_input=True)
    del xi_c, tmp
    weights = np.array([w for *_, w in pairs], dtype='f4')
    index = {t: i for i, t in enumerate(terms)}
    r1 = torch.empty((1,) + rshape, dtype=torch.float32, device=_device())
    P = torch.empty((len(pairs),) + cshape, dtype=torch.complex64, device=_device())
    Q = torch.empty(rshape, dtype=torch.float32, device=_device())
    num = []
    for ell in bin.ells:
        Aell = torch.zeros(cshape, dtype=torch.complex64, device=_device())
        for m in range(-ell, ell + 1):
            _lib.call('pk_ylm_premultiply', stream, _lib.ptr(rmesh1), *geo, 1, _lib.i32([ell]), _lib.i32([m]),
                      _lib.ptr(r1))
            _lib.call('pk_ylm_premultiply', stream, _lib.ptr(r1), *geo, len(terms), t_ell, t_m, _lib.ptr(R))
            F = _r2c(R, meshsize)
            for p, (t1, t2, _, _) in enumerate(pairs):
                _lib.call('pk_conj_multiply', stream, _lib.ptr(F[index[t1]]), _lib.ptr(B[index[t2]]), 1,
                          B[0].numel(), _lib.ptr(P[p]))
            G = _c2r(P, meshsize, destroy_input=True)
            for p0 in range(0, len(pairs), 32):
                nt = min(32, len(pairs) - p0)
                _lib.call('pk_sum_products', stream, _lib.ptr(Q), _lib.ptr(xi[p0:p0 + nt]), _lib.ptr(G[p0:p0 + nt]),
                          nt, _lib.f32(weights[p0:p0 + nt]), nreal, int(p0 > 0))
            del G, F
            FQ = _r2c(Q, meshsize)
            _lib.call('pk_ylm_kgrid_multiply', stream, _lib.ptr(FQ), _lib.i32(meshsize), kf, 1, _lib.i32([ell]),
                      _lib.i32([m]), 1., 1, _lib.ptr(Aell))
            del FQ
        value = 4. * np.pi * bin(Aell)
        if swap:
            value = np.conj(value)
        num.append(value.real if ell % 2 == 0 else value.imag)
    volume = float(np.prod(mattrs.kfun.astype('f8'))) * bin.nmodes
    return Mesh2SpectrumPoles([Mesh2SpectrumPole(k=bin.xavg, k_edges=bin.edges, nmodes=bin.nmodes, num_raw=num[ill],
                                                 norm=np.ones(bin.nbins) * norm, volume=volume, ell=ell,
                                                 attrs=dict(los='firstpoint' if not swap else 'endpoint'))
                               for ill, ell in enumerate(bin.ells)])


def compute_mesh2_spectrum_mean(*meshes, theory, bin=None, los='z'):
    """Mean power-spectrum multipoles from a theory (``mesh2.py:1485-1605``), global line of sight.

    ``theory``: a callable of the k vector (list of three broadcastable device tensors), a
    dict {ell: callable of |k| or array}, a list (ells 0, 2, 4), ``(kin, poles)`` with array
    poles, or a ``Mesh2SpectrumPoles``; arrays are read per mode from the bin containing |k|
    (order-0 ``Interpolator1D``, ``utils.py:507-537``: on ``kin`` as edges when it has one
    more entry than the poles, else on mid-point edges around ``kin``; 0 outside).
    ``A = P(k) N / V_cell`` on the half-complex grid (evaluated with torch: the theory is user
    code), then ``A <- r2c(Q c2r(A))`` with ``Q = c2r(W1 W2*)`` for a selection function, else
    ``A <- N A``; each even ell is ``(2 ell + 1) bin(A L_ell(mu))`` with k = 0 kept, in one
    fused binning pass (``pk_bin_window_batch``); odd ell is 0.  The first-point / end-point
    line of sight takes theory multipoles (keys ell or (ell, wide-angle order)) through ``_firstpoint_mean``.
    The 'jaxdecomp' layout raises ``NotImplementedError``.
    """
    meshes, fields = _format_meshes(*meshes)
    periodic = isinstance(meshes[0], MeshAttrs)
    if periodic:
        assert fields[1] == fields[0]
        mattrs = meshes[0]
    else:
        mattrs = meshes[0].attrs
    if mattrs.fft_backend != 'jax':
        raise NotImplementedError("the mean spectrum takes the 'jax' FFT backend")
    los, vlos, swap = _los(los)
    meshsize = mattrs.meshsize
    if periodic:
        N = float(np.prod(meshsize.astype('f8')))
        norm = N / float(np.prod(mattrs.cellsize.astype('f8')))
    else:
        N = np.float32(np.prod(meshsize.astype('f4'), dtype='f4'))
        norm = np.float32(N / np.float32(np.prod(mattrs.cellsize, dtype='f4')))
    rnorm = norm / N
    ells = bin.ells
    kin, poles, theory_los = _theory_poles(theory)
    kvec = mattrs.kcoords(sparse=True)
    knorm = torch.sqrt(kvec[0] ** 2 + kvec[1] ** 2 + kvec[2] ** 2)

    def get_theory(pole):
        if callable(pole):
            return pole(knorm)
        pole = np.asarray(pole, dtype='f8')
        kin_ = np.asarray(kin, dtype='f8')
        if len(kin_) == len(pole) + 1:
            edges = kin_
        else:
            tmp = (kin_[:-1] + kin_[1:]) / 2.
            edges = np.concatenate([[tmp[0] - (kin_[1] - kin_[0])], tmp, [tmp[-1] + (kin_[-1] - kin_[-2])]])
        d_edges = torch.as_tensor(edges.astype('f4'), device=knorm.device)
        idx = torch.bucketize(knorm, d_edges, right=True) - 1
        inside = (idx >= 0) & (idx <= len(edges) - 2)
        table = torch.as_tensor(pole.astype('f4'), device=knorm.device)
        return torch.where(inside, table[idx.clamp(0, len(pole) - 1)], torch.zeros_like(knorm))

    if vlos is None:  # binned through bin(...): mode oversampling is taken
        return _firstpoint_mean(meshes, fields, periodic, mattrs, bin, poles, get_theory, swap, N, norm, rnorm,
                                theory_los=theory_los)
    _plain_bins(bin, 'compute_mesh2_spectrum_mean with a fixed line of sight')
    mu = (kvec[0] * float(vlos[0]) + kvec[1] * float(vlos[1]) + kvec[2] * float(vlos[2])) / \
        torch.where(knorm == 0., torch.ones_like(knorm), knorm)
    if callable(poles):
        pk = poles(kvec)
    else:
        pk = 0.
        for ell, pole in poles.items():
            pk = pk + get_theory(pole) * _legendre(int(ell[0] if isinstance(ell, tuple) else ell), mu)
    cshape = tuple(int(n) for n in meshsize[:2]) + (int(meshsize[2]) // 2 + 1,)
    A = torch.zeros(cshape, dtype=torch.complex64, device=_device())
    A.real.copy_(torch.as_tensor(pk * rnorm, device=_device()).to(torch.float32).expand(cshape))
    stream = _lib.stream_handle()
    if periodic:
        A = A * float(N)
    else:
        A1 = _2c(meshes[0]).value.contiguous()
        A2 = A1 if fields[1] == fields[0] else _2c(meshes[1]).value.contiguous()
        prod = torch.empty_like(A1)
        _lib.call('pk_conj_multiply', stream, _lib.ptr(A2), _lib.ptr(A1), 1, A1.numel(), _lib.ptr(prod))
        # Q = c2r(W1 W2*) (irfftn's 1 / N), times the 1 / N of the c2r of A, taken unscaled
        Q = _c2r(prod, meshsize, scale=False, destroy_input=True)
        del prod, A1, A2
        _lib.call('pk_scale_real', stream, _lib.ptr(Q), Q.numel(), float(np.float64(np.float32(1.) / N) ** 2))
        real = _c2r(A, meshsize, scale=False, destroy_input=True)
        _lib.call('pk_window_multiply', stream, _lib.ptr(real), 1, _lib.ptr(Q), Q.numel())
        A = _r2c(real, meshsize)
        del real, Q
    A = A.contiguous()
    even = [ill for ill, ell in enumerate(ells) if ell % 2 == 0]
    num = np.zeros((len(ells), bin.nbins))
    if even:
        nbytes = _lib.c_size_t()
        _lib.call('pk_bin_batch_workspace_size', _lib.i32(meshsize), len(bin._edges1d), len(even), 1,
                  _lib.ctypes.byref(nbytes))
        ws = _workspace(nbytes.value)
        raw = torch.empty((len(even), bin.nbins), dtype=torch.float64, device=_device())
        _lib.call('pk_bin_window_batch', stream, _lib.ptr(A), 1, _lib.i32(meshsize), _lib.f32(mattrs.kfun),
                  _lib.f32(vlos), _lib.ptr(bin.d_edges), len(bin._edges1d), bin._step, mattrs.backend_code, len(even),
                  _lib.i32([ells[ill] for ill in even]), 0, _lib.ptr(raw), _lib.ptr(ws), ws.numel())
        raw = raw.cpu().numpy()
        with np.errstate(invalid='ignore', divide='ignore'):
            for q, ill in enumerate(even):
                num[ill] = (2 * ells[ill] + 1) * raw[q] / bin.nmodes
    volume = float(np.prod(mattrs.kfun.astype('f8'))) * bin.nmodes
    return Mesh2SpectrumPoles([Mesh2SpectrumPole(k=bin.xavg, k_edges=bin.edges, nmodes=bin.nmodes, num_raw=num[ill],
                                                 norm=np.ones(bin.nbins) * norm, volume=volume, ell=ell,
                                                 attrs=dict(los=np.asarray(vlos).tolist()))
                               for ill, ell in enumerate(ells)])


def _window_coeffs(ell, ellin):
    """``get_window_coeffs`` (``mesh2.py:759-765``): (q, (2 ell + 1) (ell ellin q; 0 0 0)^2) with the
    Wigner 3j squares read off the Legendre expansion ``L_ell L_ellin = sum_q (2 q + 1) (3j)^2 L_q``."""
    from numpy.polynomial import legendre as npleg
    c = npleg.legmul([0.] * ell + [1.], [0.] * ellin + [1.])
    out = []
    for q in range(abs(ell - ellin), ell + ellin + 1):
        coeff = (2 * ell + 1) * (c[q] / (2 * q + 1) if q < len(c) else 0.)
        if abs(coeff) >= 1e-7:
            out.append((q, coeff))
    return out


def compute_smooth2_spectrum_window(window, edgesin, ellsin=None, bin=None, flags=('rect',), batch_size=None):
    """'Smooth' (no binning effect) window matrix from configuration-space window multipoles
    (``mesh2.py:803-918``), 'rect' integration.

    ``window``: a ``Mesh2CorrelationPoles`` (e.g. from ``compute_mesh2_correlation`` of the
    selection function).  For each input ell_in and output ell, ``Qs = sum_q c_q W_q(s)``
    (``_window_coeffs``), then per input bin (mid-point k_in) and output k
    ``(-1)^(ell/2) sum_s j_ell(k s) n_s (-1)^(ell_in/2) / (2 pi)^3 j_ell_in(k_in s) V_in Qs(s)``,
    ``n_s`` the window's ``volume`` (ones if absent), ``V_in = 4 pi / 3 (k_hi^3 - k_lo^3)``.  These
    are 1D host sums over the window's separations (no mesh work).  Wide-angle inputs
    (ell_in, n) take the window multipoles labelled with order n (``window.wa_orders``) and an
    extra s^n (``mesh2.py:845-851, 869``); an order n > 0 needs a window carrying wide-angle
    labels (``ValueError`` otherwise, as the reference).  The 'fftlog' integration (any flag
    set without 'rect') raises ``NotImplementedError``.
    """
    from scipy.special import spherical_jn
    if 'rect' not in flags:
        raise NotImplementedError("only the 'rect' integration of the smooth window is supported")
    ells = bin.ells
    if hasattr(edgesin, 'ells') and hasattr(edgesin, 'poles'):
        ellsin = edgesin.ells
        edgesin = next(iter(edgesin)).k_edges
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    ellsin = [e if isinstance(e, tuple) else (int(e), 0) for e in ((ellsin,) if isinstance(ellsin, (int, np.integer)) else ellsin)]
    labelled = any(getattr(window, 'wa_orders', ()))
    if any(wa != 0 for _, wa in ellsin) and not labelled:
        raise ValueError('wa_orders must be provided in input window')
    kout = np.asarray(bin.xavg, dtype='f8')
    first = next(iter(window))
    s = np.asarray(first.coords('s'), dtype='f8')
    snmodes = np.ones_like(s) if first.volume is None else np.asarray(first.volume, dtype='f8')
    savg = np.where(snmodes == 0, 0., s)
    kin = np.mean(edgesin, axis=-1)
    vin = 4. / 3. * np.pi * (edgesin[:, 1] ** 3 - edgesin[:, 0] ** 3)

    def get_w(q, wa):
        keys = list(zip(window.ells, window.wa_orders)) if labelled else [(e, 0) for e in window.ells]
        if (q, wa) in keys:
            return np.real(np.asarray(window.get(q, wa_orders=wa if labelled else None).value(), dtype='c16'))
        return 0.

    blocks = []
    for ellin, wa in ellsin:
        col = []
        for ell in ells:
            Qs = sum(coeff * get_w(q, wa) for q, coeff in _window_coeffs(ell, ellin))
            Qs = np.where(snmodes == 0, 0., Qs)
            tophat = ((-1) ** (ellin // 2) / (2. * np.pi) ** 3 * spherical_jn(ellin, savg[None, :] * kin[:, None])
                      * vin[:, None] * Qs * savg[None, :] ** wa)  # (nin, ns)
            jk = (-1) ** (ell // 2) * spherical_jn(ell, kout[:, None] * savg[None, :])  # (nbins, ns)
            col.append(jk.dot((snmodes * tophat).T))  # (nbins, nin)
        blocks.append(np.concatenate(col, axis=0))
    wmat = np.concatenate(blocks, axis=1)
    observable = Mesh2SpectrumPoles([Mesh2SpectrumPole(k=bin.xavg, k_edges=bin.edges, nmodes=bin.nmodes,
                                                       num_raw=np.zeros(len(kout)), num_shotnoise=np.zeros(len(kout)),
                                                       norm=np.ones(len(kout)), ell=ell) for ell in ells])
    theory = Mesh2SpectrumPoles([Mesh2SpectrumPole(k=kin, k_edges=edgesin, nmodes=np.ones(len(kin)),
                                                   num_raw=np.zeros(len(kin)), ell=ellin,
                                                   attrs=dict(wa_order=wa) if wa else None) for ellin, wa in ellsin])
    from .types import WindowMatrix
    return WindowMatrix(observable=observable, theory=theory, value=wmat)
