"""k-binning and the power-spectrum estimators (oracle; test only).

Restates:

- ``mesh2.py:25-62``   ``_make_edges2``: edges = ``np.arange(0, kfun.min() * min(N) / 2, step)``
  (float64), compared in float32 by ``jnp.digitize(right=False)``;
- ``mesh.py:2833-2863`` ``_get_bin_attrs``: ibin, nmodes (Hermitian weights), xavg;
- ``mesh.py:2876-2910`` ``_bincount``: per-bin sums over bins ``[1:-1]``;
- ``mesh2.py:100-119``  ``BinMesh2SpectrumPoles.__call__`` (remove_zero, / nmodes);
- ``mesh2.py:253-374``  ``compute_mesh2_spectrum``: global line of sight
  (Legendre of mu = k.los/|k| with |k|(0) = 1) and first-point line of sight
  (``4 pi * bin(conj(sum_m r2c(rho Y_lm(xhat)) Y_lm(khat)) A0)``), endpoint swap,
  real part for even ell;
- ``mesh2.py:508-621`` / ``mesh.py:3042-3129``  FKP normalisation and shot noise;
- ``mesh.py:2226-2381`` ``get_mesh_attrs`` / ``next_fft_size``.

``accum='f32'`` accumulates bins serially in float32 in flat mode order (the
reference's CPU bincount order); ``accum='f64'`` accumulates the same float32
per-mode products in float64 (the accuracy the CUDA kernels are held to).
"""
import math
from itertools import product

import numpy as np

from .coords import Geometry, kcoords, rcoords, hermitian_weights, r2c, c2r
from .paint import paint as paint_field
from .ylm import get_ylm, legendre


class Bins:
    """``BinMesh2SpectrumPoles(mattrs, edges={'step': step}, ells)`` restated."""

    def __init__(self, geom, step=None, edges=None, ells=(0, 2, 4), kmin=0., kmax=None, mode_oversampling=0):
        dt = geom.dtype
        self.geom = geom
        self.ells = tuple(sorted((ells,) if np.ndim(ells) == 0 else ells))
        if edges is None:
            vec0 = geom.kfun.min()
            vecmax = dt.type(vec0 * dt.type(np.min(geom.meshsize))) / dt.type(2.)
            stop = float(vecmax) if kmax is None else kmax
            edges = np.arange(kmin, stop, step)
        self.edges = np.asarray(edges, dtype='f8')
        self.edges_dtype = self.edges.astype(dt)
        self.wmodes = hermitian_weights(geom)
        nb = len(self.edges) + 1
        w = self.wmodes.ravel()
        # mode oversampling (mesh2.py:48-61): one bin index per integer shift in [-s, s]^3 of the
        # k coordinates, nmodes averaged over the shifts, xavg = summed sum(|k + shift| w) / nmodes
        r = range(-int(mode_oversampling), int(mode_oversampling) + 1)
        shifts = list(product(r, r, r)) if mode_oversampling else [(0, 0, 0)]
        self.ibins, nmodes, ksum = [], 0., 0.
        for shift in shifts:
            knorm = self.knorm(shift if mode_oversampling else None)
            ibin = np.searchsorted(self.edges_dtype, knorm.ravel(), side='right').reshape(knorm.shape)
            self.ibins.append(ibin)
            nmodes = nmodes + np.bincount(ibin.ravel(), weights=w, minlength=nb)[1:-1]
            ksum = ksum + np.bincount(ibin.ravel(), weights=(knorm.ravel().astype('f8') * w), minlength=nb)[1:-1]
        self.ibin = self.ibins[0]
        self.nmodes = nmodes / len(shifts) if mode_oversampling else nmodes
        with np.errstate(invalid='ignore', divide='ignore'):
            self.xavg = ksum / self.nmodes

    @property
    def nbins(self):
        return len(self.edges) - 1

    def knorm(self, shift=None):
        dt = self.geom.dtype
        kx, ky, kz = kcoords(self.geom)
        if shift is not None:  # xx + ss in the mesh dtype (mesh2.py:50)
            kx, ky, kz = [(kk + dt.type(ss)).astype(dt) for kk, ss in zip((kx, ky, kz), shift)]
        k2 = (((dt.type(0.) + kx * kx).astype(dt) + ky * ky).astype(dt) + kz * kz).astype(dt)
        return np.sqrt(k2).astype(dt)

    def __call__(self, value, remove_zero=False, accum='f64'):
        """Per-bin mean of ``value`` with Hermitian weights (``mesh2.py:100-119``)."""
        value = np.array(value, copy=True)
        if remove_zero:
            value[0, 0, 0] = 0.
        nb = len(self.edges) + 1
        ib = self.ibin.ravel()
        if accum == 'f64':
            wv = value.ravel() * self.wmodes.ravel().astype(value.real.dtype)
            s = 0.
            for ibin in self.ibins:  # the mean over the oversampling shifts (mesh.py:2894-2895)
                ib = ibin.ravel()
                if np.iscomplexobj(wv):
                    s = s + np.bincount(ib, weights=wv.real, minlength=nb) + 1j * np.bincount(ib, weights=wv.imag,
                                                                                              minlength=nb)
                else:
                    s = s + np.bincount(ib, weights=wv, minlength=nb)
            return s[1:-1] / len(self.ibins) / self.nmodes
        if len(self.ibins) > 1:
            raise NotImplementedError('float32 serial accumulation without mode oversampling only')
        dt = value.real.dtype
        wv = (value.ravel() * self.wmodes.ravel().astype(dt))
        if np.iscomplexobj(wv):
            re = np.zeros(nb, dtype=dt)
            im = np.zeros(nb, dtype=dt)
            np.add.at(re, ib, wv.real.astype(dt))
            np.add.at(im, ib, wv.imag.astype(dt))
            s = re + 1j * im
        else:
            s = np.zeros(nb, dtype=dt)
            np.add.at(s, ib, wv.astype(dt))
        return s[1:-1] / self.nmodes.astype(dt)


def _to_complex(geom, mesh):
    return mesh if np.iscomplexobj(mesh) else r2c(geom, mesh)


def _to_real(geom, mesh):
    return mesh if not np.iscomplexobj(mesh) else c2r(geom, mesh)


def compute_mesh2_spectrum(mesh, bins, los='z', accum='f64', mesh2=None):
    """``compute_mesh2_spectrum(mesh, bin=bins, los=los)`` (``mesh2.py:253-374``).

    Returns dict(ells, k, nmodes, num_raw (nells, nbins), norm).
    """
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    norm = t(np.prod(geom.meshsize.astype(dt))) / t(np.prod(geom.cellsize))
    swap = False
    if isinstance(los, str) and los in ('firstpoint', 'local', 'endpoint'):
        swap = los == 'endpoint'
        vlos = None
    else:
        vlos = np.zeros(3)
        if isinstance(los, str):
            vlos['xyz'.index(los)] = 1.
        else:
            vlos = np.asarray(los, dtype='f8')
    num = []
    if vlos is None:
        rmesh = _to_real(geom, mesh)
        A0 = _to_complex(geom, mesh if mesh2 is None else mesh2)
        cross = mesh2 is not None
        if swap and cross:
            rmesh, A0 = _to_real(geom, mesh2), _to_complex(geom, mesh)
        if 0 in ells:
            if not cross:
                A = (A0.real * A0.real + A0.imag * A0.imag).astype(dt)
            else:
                A = (np.conj(_to_complex(geom, rmesh)) * A0)
            num.append(bins(A, accum=accum))
        xvec = rcoords(geom)
        kvec = kcoords(geom)
        for ell in ells:
            if ell == 0:
                continue
            carry = np.zeros(geom.cshape, dtype=A0.dtype)
            for m in range(-ell, ell + 1):
                Y = get_ylm(ell, m)
                F = r2c(geom, (rmesh * Y(*xvec)).astype(dt))
                carry = (carry + F * Y(*kvec)).astype(A0.dtype)
            A = (np.conj(carry) * A0).astype(A0.dtype)
            num.append(t(4. * np.pi) * bins(A, remove_zero=True, accum=accum))
        if swap:
            num = [np.conj(n) for n in num]
    else:
        A0 = _to_complex(geom, mesh)
        if mesh2 is None:
            A = (A0.real * A0.real + A0.imag * A0.imag).astype(dt)
        else:
            A = np.conj(A0) * _to_complex(geom, mesh2)
        if 0 in ells:
            num.append(bins(A, accum=accum))
        kvec = kcoords(geom)
        kl = [(kk * t(ll)).astype(dt) for kk, ll in zip(kvec, vlos)]
        mu_num = (((t(0.) + kl[0]).astype(dt) + kl[1]).astype(dt) + kl[2]).astype(dt)
        knorm = bins.knorm().copy()
        knorm[0, 0, 0] = 1.
        mu = (mu_num / knorm).astype(dt)
        for ell in ells:
            if ell == 0:
                continue
            num.append(t(2 * ell + 1) * bins((A * legendre(ell, mu)), remove_zero=True, accum=accum))
    num = [np.real(n) if ell % 2 == 0 else np.imag(n) for ell, n in zip(ells, num)]
    return dict(ells=ells, k=bins.xavg, edges=bins.edges, nmodes=bins.nmodes,
                num_raw=np.array(num), norm=norm,
                volume=np.prod(geom.kfun.astype('f8')) * bins.nmodes)



def compute_mesh2_spectrum_window(bins, edgesin, ellsin, los='z', meshes=None, norm=None):
    """``compute_mesh2_spectrum_window(*meshes or mattrs, edgesin=, ellsin=, bin=bins, los=)``,
    global line of sight, input power on the mesh (``mesh2.py:921-1133``, ``1462-1482``).

    ``meshes``: None (periodic box: ``MeshAttrs`` given) or one / two real selection meshes.
    Returns the window matrix, (len(ells) nbins, len(ellsin) len(edgesin)), float64.
    """
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    N = t(np.prod(geom.meshsize.astype(dt)))
    _norm = t(N / t(np.prod(geom.cellsize.astype(dt))))
    norm = np.asarray(_norm if norm is None else norm, dtype=dt)
    if norm.ndim <= 1:
        norm = norm * np.ones(len(ells), dtype=dt)
    rnorm = (_norm / norm / N).astype(dt)
    vlos = np.zeros(3)
    if isinstance(los, str):
        vlos['xyz'.index(los)] = 1.
    else:
        vlos = np.asarray(los, dtype='f8')
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    edgesin_dt = edgesin.astype(dt)
    Q, common = None, False
    if meshes is not None:
        W = [_to_complex(geom, m) for m in meshes]
        W2 = W[0] if len(W) == 1 else W[1]
        Q = (c2r(geom, (W[0] * np.conj(W2)).astype(W[0].dtype)) / N).astype(dt)
    else:
        bedges = np.column_stack([bins.edges[:-1], bins.edges[1:]])
        mask_in = np.all(edgesin >= bedges[0], axis=-1) & np.all(edgesin <= bedges[-1], axis=-1)
        mask_edges = np.all(bedges >= edgesin[0], axis=-1) & np.all(bedges <= edgesin[-1], axis=-1)
        common = mask_edges.sum() == mask_in.sum() and np.allclose(edgesin[mask_in], bedges[mask_edges])
    kvec = kcoords(geom)
    knorm = bins.knorm()
    kl = [(kk * t(ll)).astype(dt) for kk, ll in zip(kvec, vlos)]
    num = (((t(0.) + kl[0]).astype(dt) + kl[1]).astype(dt) + kl[2]).astype(dt)
    mu = (num / np.where(knorm == 0., t(1.), knorm)).astype(dt)

    def _bin(A):
        spectrum = []
        for ill, ell in enumerate(ells):
            leg = legendre(ell, mu)
            odd = ell % 2
            if odd:
                leg = (leg + legendre(ell, (-mu).astype(dt))).astype(dt)
            spectrum.append((2 * ell + 1) / (1 + odd) * bins((A * leg).astype(A.dtype), remove_zero=True) * rnorm[ill])
        return np.concatenate(spectrum)

    wmat = []
    for ellin in ellsin:
        legin = legendre(ellin, mu)
        if common:
            spectrum = _bin((legin * N).astype(np.complex64))
            nb = bins.nbins
            w = np.zeros((len(edgesin), len(ells), nb), dtype=spectrum.dtype)
            for ill in range(len(ells)):
                w[np.flatnonzero(mask_in), ill, np.flatnonzero(mask_edges)] = spectrum[ill * nb:(ill + 1) * nb][mask_edges]
            wmat.append(w.reshape(len(edgesin), -1))
            continue
        rows = []
        for lo, hi in edgesin_dt:
            A = (((knorm >= lo) & (knorm < hi)) * legin * N).astype(np.complex64)
            if Q is not None:
                A = r2c(geom, (Q * c2r(geom, A)).astype(dt))
            rows.append(_bin(A))
        wmat.append(np.array(rows))
    return np.real(np.concatenate(wmat, axis=0).T)


def compute_mesh2_spectrum_mean(bins, theory, los='z', meshes=None):
    """``compute_mesh2_spectrum_mean(*meshes or mattrs, theory=, bin=bins, los=)``, global line of
    sight (``mesh2.py:1485-1605``).  ``theory``: a callable of the k vector or a dict
    {ell: callable of |k|}.  ``meshes``: None (periodic box, float64 normalisation as the
    reference's ``rdtype = float``) or one / two real selection meshes.

    Returns num_raw (nells, nbins) and norm.
    """
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    if meshes is None:
        N = float(np.prod(geom.meshsize.astype('f8')))
        norm = N / float(np.prod(geom.cellsize.astype('f8')))
    else:
        N = t(np.prod(geom.meshsize.astype(dt)))
        norm = t(N / t(np.prod(geom.cellsize.astype(dt))))
    rnorm = norm / N
    vlos = np.zeros(3)
    if isinstance(los, str):
        vlos['xyz'.index(los)] = 1.
    else:
        vlos = np.asarray(los, dtype='f8')
    kvec = kcoords(geom)
    knorm = bins.knorm()
    kl = [(kk * t(ll)).astype(dt) for kk, ll in zip(kvec, vlos)]
    num = (((t(0.) + kl[0]).astype(dt) + kl[1]).astype(dt) + kl[2]).astype(dt)
    mu = (num / np.where(knorm == 0., t(1.), knorm)).astype(dt)
    if callable(theory):
        pk = theory(kvec)
    else:
        pk = sum(np.asarray(pole(knorm)) * legendre(ell, mu) for ell, pole in theory.items())
    A = np.broadcast_to(np.asarray(pk * rnorm, dtype=dt), geom.cshape).astype(np.complex64)
    if meshes is not None:
        W = [_to_complex(geom, m) for m in meshes]
        W2 = W[0] if len(W) == 1 else W[1]
        Q = c2r(geom, (W[0] * np.conj(W2)).astype(W[0].dtype))
        A = r2c(geom, (Q * c2r(geom, A)).astype(dt))
    else:
        A = (A * N).astype(np.complex64)
    out = []
    for ell in ells:
        leg = legendre(ell, mu)
        odd = ell % 2
        if odd:
            leg = (leg + legendre(ell, (-mu).astype(dt))).astype(dt)
        value = (2 * ell + 1) / (1 + odd) * bins((A * leg).astype(A.dtype))
        out.append(np.real(value) if ell % 2 == 0 else np.imag(value))
    return dict(num_raw=np.array(out), norm=norm)


def compute_mesh2_spectrum_mean_firstpoint(bins, theory, meshes=None, swap=False, theory_los='firstpoint'):
    """``compute_mesh2_spectrum_mean(..., theory=dict, los='firstpoint' / 'endpoint')``
    (``mesh2.py:1607-1669``, wide-angle order 0): for each output (ell, m),
    ``Q = sum_{ell1 m1} 4 pi / (2 ell1 + 1) xi_{ell1 m1} c2r(conj(r2c(W1 Y_lm(xhat) Y_l1m1(xhat))) A0)``,
    ``xi = c2r(P_ell1(|k|) rnorm Y_l1m1(khat))``, ``A_ell += r2c(Q) Y_lm(khat)``; then
    ``4 pi bin(A_ell)``.  ``theory``: {ell: callable of |k|}; ``meshes``: None (periodic) or
    one / two real selection meshes.  Returns num_raw (nells, nbins)."""
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    if meshes is None:
        N = float(np.prod(geom.meshsize.astype('f8')))
        norm = N / float(np.prod(geom.cellsize.astype('f8')))
        meshes = [np.ones(geom.rshape, dtype=dt)]
    else:
        N = t(np.prod(geom.meshsize.astype(dt)))
        norm = t(N / t(np.prod(geom.cellsize.astype(dt))))
        meshes = list(meshes)
    rnorm = norm / N
    if swap:
        meshes = meshes[::-1]
    rmesh1 = _to_real(geom, meshes[0])
    A0 = _to_complex(geom, meshes[0] if len(meshes) == 1 else meshes[1])
    xvec = rcoords(geom)
    kvec = kcoords(geom)
    knorm = bins.knorm()
    if theory_los == 'local':  # mesh2.py:1646-1661
        rmesh2 = rmesh1 if len(meshes) == 1 else _to_real(geom, meshes[1])
        coeff2 = {(0, 0): [(0, 1.), (4, -7. / 18.)], (0, 2): [(2, 1. / 2.), (4, -5. / 18.)], (2, 2): [(4, 35. / 18.)]}
        coeff2[2, 0] = coeff2[0, 2]
        xil, Bl = {}, {}
        for ell1 in (0, 2):
            for ell2 in (0, 2):
                kernel = (sum(c * np.asarray(theory[ell](knorm)) for ell, c in coeff2[ell1, ell2]) * rnorm).astype(dt)
                for m1 in range(-ell1, ell1 + 1):
                    for m2 in range(-ell2, ell2 + 1):
                        y = (kernel * get_ylm(ell1, m1)(*kvec)).astype(dt) * get_ylm(ell2, m2)(*[-kk for kk in kvec])
                        xil[ell1, m1, ell2, m2] = c2r(geom, y.astype(np.complex64))
        for ell2 in (0, 2):
            for m2 in range(-ell2, ell2 + 1):
                Bl[ell2, m2] = r2c(geom, (rmesh2 * get_ylm(ell2, m2)(*xvec)).astype(dt))
        out = []
        for ell in bins.ells:
            Aell = np.zeros(geom.cshape, dtype=np.complex64)
            for m in range(-ell, ell + 1):
                Ylm = get_ylm(ell, m)
                Q = np.zeros(geom.rshape, dtype=dt)
                for (ell1, m1, ell2, m2), x in xil.items():
                    F = r2c(geom, ((rmesh1 * Ylm(*xvec)).astype(dt) * get_ylm(ell1, m1)(*xvec)).astype(dt))
                    G = c2r(geom, (np.conj(F) * Bl[ell2, m2]).astype(np.complex64))
                    Q = (Q + t((4. * np.pi) ** 2 / ((2 * ell1 + 1) * (2 * ell2 + 1))) * x * G).astype(dt)
                Aell = (Aell + r2c(geom, Q) * Ylm(*kvec)).astype(np.complex64)
            value = 4. * np.pi * bins(Aell)
            if swap:
                value = np.conj(value)
            out.append(np.real(value) if ell % 2 == 0 else np.imag(value))
        return np.array(out)
    # theory keys: ell or (ell, wide-angle order wa): xi * |s|^wa, W1 * |x|^-wa (mesh2.py:1641-1645)
    theory = {(k if isinstance(k, tuple) else (k, 0)): v for k, v in theory.items()}
    sv = separation_coords(geom)
    snorm = np.sqrt(((sv[0] * sv[0] + sv[1] * sv[1]) + sv[2] * sv[2]).astype(dt)).astype(dt)
    xnorm = np.sqrt(((xvec[0] * xvec[0] + xvec[1] * xvec[1]) + xvec[2] * xvec[2]).astype(dt)).astype(dt)
    xi = {}
    for (ell1, wa), pole in theory.items():
        kernel = (np.asarray(pole(knorm)) * rnorm).astype(dt)
        for m1 in range(-ell1, ell1 + 1):
            xi[ell1, wa, m1] = (c2r(geom, (kernel * get_ylm(ell1, m1)(*kvec)).astype(np.complex64)) * snorm ** wa).astype(dt)
    out = []
    for ell in bins.ells:
        Aell = np.zeros(geom.cshape, dtype=np.complex64)
        for m in range(-ell, ell + 1):
            Ylm = get_ylm(ell, m)
            Q = np.zeros(geom.rshape, dtype=dt)
            for ell1, wa in theory:
                for m1 in range(-ell1, ell1 + 1):
                    Y1 = get_ylm(ell1, m1)
                    F = r2c(geom, (((rmesh1 * xnorm ** (-wa)).astype(dt) * Ylm(*xvec)).astype(dt) * Y1(*xvec)).astype(dt))
                    G = c2r(geom, (np.conj(F) * A0).astype(np.complex64))
                    Q = (Q + t(4. * np.pi / (2 * ell1 + 1)) * xi[ell1, wa, m1] * G).astype(dt)
            Aell = (Aell + r2c(geom, Q) * Ylm(*kvec)).astype(np.complex64)
        value = 4. * np.pi * bins(Aell)
        if swap:
            value = np.conj(value)
        out.append(np.real(value) if ell % 2 == 0 else np.imag(value))
    return np.array(out)


def _wide_angle_factors(geom, wa):
    """``xnorm**(-wain)`` and ``snorm**wain`` of the first-point window (``mesh2.py:1212-1214``):
    |x| of the cell-corner positions and |s| of the separation grid, in the geometry's dtype
    (negative powers as 1 / |x|^-wa)."""
    dt = geom.dtype
    t = dt.type
    x = rcoords(geom)
    s = separation_coords(geom)
    xn = np.sqrt((((t(0.) + x[0] * x[0]).astype(dt) + x[1] * x[1]).astype(dt) + x[2] * x[2]).astype(dt)).astype(dt)
    sn = np.sqrt((((t(0.) + s[0] * s[0]).astype(dt) + s[1] * s[1]).astype(dt) + s[2] * s[2]).astype(dt)).astype(dt)
    with np.errstate(divide='ignore'):
        return (t(1.) / xn ** wa).astype(dt), (sn ** wa).astype(dt)


def _wa_terms(ellsin):
    return [e if isinstance(e, tuple) else (int(e), 0) for e in ellsin]


def compute_mesh2_spectrum_window_firstpoint(bins, edgesin, ellsin, meshes=None, swap=False, norm=None,
                                             theory_los='firstpoint'):
    """``compute_mesh2_spectrum_window(..., los='firstpoint' / 'endpoint')``, input power on the
    mesh (``mesh2.py:1135-1304``, ``1462-1470``); inputs ell_in or (ell_in, wide-angle order).  ``meshes``: None
    (periodic box) or one / two real selection meshes.  Returns the window matrix
    (len(ells) nbins, len(ellsin) len(edgesin))."""
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    N = t(np.prod(geom.meshsize.astype(dt)))
    _norm = t(N / t(np.prod(geom.cellsize.astype(dt))))
    norm = np.asarray(_norm if norm is None else norm, dtype=dt)
    if norm.ndim <= 1:
        norm = norm * np.ones(len(ells), dtype=dt)
    rnorm = (_norm / norm / N).astype(dt)
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    meshes = [np.ones(geom.rshape, dtype=dt)] if meshes is None else list(meshes)
    if swap:
        meshes = meshes[::-1]
    rmesh1 = _to_real(geom, meshes[0])
    A0 = _to_complex(geom, meshes[0] if len(meshes) == 1 else meshes[1])
    xvec = rcoords(geom)
    kvec = kcoords(geom)
    knorm = bins.knorm()
    if theory_los == 'local':  # mesh2.py:1398-1455
        rmesh2 = rmesh1 if len(meshes) == 1 else _to_real(geom, meshes[1])
        coeff2 = {(0, 0): [(0, 1.), (4, -7. / 18.)], (0, 2): [(2, 1. / 2.), (4, -5. / 18.)], (2, 2): [(4, 35. / 18.)]}
        coeff2[2, 0] = coeff2[0, 2]
        wmat = np.zeros((len(ellsin), len(edgesin), len(ells) * bins.nbins), dtype='c16')
        for ell1 in (2, 0):
            for ell2 in (2, 0):
                pairs = [(m1, m2) for m1 in range(-ell1, ell1 + 1) for m2 in range(-ell2, ell2 + 1)]
                w = t((4. * np.pi) ** 2 / ((2 * ell1 + 1) * (2 * ell2 + 1)))
                Qs = {}
                for ell in ells:
                    for m in range(-ell, ell + 1):
                        for m1, m2 in pairs:
                            F = r2c(geom, ((rmesh1 * get_ylm(ell, m)(*xvec)).astype(dt) * get_ylm(ell1, m1)(*xvec)).astype(dt))
                            B = r2c(geom, (rmesh2 * get_ylm(ell2, m2)(*xvec)).astype(dt))
                            Qs[ell, m, m1, m2] = (w * c2r(geom, (np.conj(F) * B).astype(np.complex64))).astype(dt)
                block = []
                for lo, hi in edgesin.astype(dt):
                    shell = ((knorm >= lo) & (knorm <= hi))
                    xi = {(m1, m2): c2r(geom, ((shell * get_ylm(ell1, m1)(*kvec)).astype(dt)
                                               * get_ylm(ell2, m2)(*[-kk for kk in kvec])).astype(np.complex64))
                          for m1, m2 in pairs}
                    spectrum = []
                    for ill, ell in enumerate(ells):
                        Aell = np.zeros(geom.cshape, dtype=np.complex64)
                        for m in range(-ell, ell + 1):
                            tmp = sum(xi[pr] * Qs[(ell, m) + pr] for pr in pairs).astype(dt)
                            Aell = (Aell + r2c(geom, tmp) * get_ylm(ell, m)(*kvec)).astype(np.complex64)
                        spectrum.append(4. * np.pi * bins(Aell, remove_zero=ell == 0) * rnorm[ill])
                    block.append(np.concatenate(spectrum))
                for illin, ellin in enumerate(ellsin):
                    wmat[illin] += sum(c * (ell == ellin) for ell, c in coeff2[ell1, ell2]) * np.array(block)
        wmat = wmat.reshape(-1, wmat.shape[-1]).T
        nb = bins.nbins
        first = wmat[:nb].imag if ells[0] % 2 else wmat[:nb].real
        wmat = wmat.real.copy()
        wmat[:nb] = first
        return wmat
    blocks = []
    for ellin, wa in _wa_terms(ellsin):  # wide-angle order wa: W1 |x|^-wa, Q |s|^wa (mesh2.py:1273)
        xf, sf = _wide_angle_factors(geom, wa)
        rho = (rmesh1 * xf).astype(dt) if wa else rmesh1
        Qs = {}
        for ell in ells:
            for m in range(-ell, ell + 1):
                for m1 in range(-ellin, ellin + 1):
                    F = r2c(geom, ((rho * get_ylm(ell, m)(*xvec)).astype(dt) * get_ylm(ellin, m1)(*xvec)).astype(dt))
                    Qs[ell, m, m1] = (t(4. * np.pi / (2 * ellin + 1)) * c2r(geom, (np.conj(F) * A0).astype(np.complex64))).astype(dt)
                    if wa:
                        Qs[ell, m, m1] = (Qs[ell, m, m1] * sf).astype(dt)
        rows = []
        for lo, hi in edgesin.astype(dt):
            xi = {m1: c2r(geom, (((knorm >= lo) & (knorm <= hi)) * get_ylm(ellin, m1)(*kvec)).astype(np.complex64))
                  for m1 in range(-ellin, ellin + 1)}
            spectrum = []
            for ill, ell in enumerate(ells):
                Aell = np.zeros(geom.cshape, dtype=np.complex64)
                for m in range(-ell, ell + 1):
                    tmp = sum(xi[m1] * Qs[ell, m, m1] for m1 in xi).astype(dt)
                    Aell = (Aell + r2c(geom, tmp) * get_ylm(ell, m)(*kvec)).astype(np.complex64)
                spectrum.append(4. * np.pi * bins(Aell, remove_zero=ell == 0) * rnorm[ill])
            rows.append(np.concatenate(spectrum))
        blocks.append(np.array(rows))
    wmat = np.concatenate(blocks, axis=0).T
    nb = bins.nbins
    first = wmat[:nb].imag if ells[0] % 2 else wmat[:nb].real
    wmat = wmat.real.copy()
    wmat[:nb] = first
    return wmat


def compute_mesh2_spectrum_window_smooth(bins, sedges, edgesin, ellsin, los='z', meshes=None, norm=None):
    """``compute_mesh2_spectrum_window(..., flags=('smooth',))``, global line of sight
    (``mesh2.py:1061-1093``): ``Qs = sbin(Q L_ell(mu_s) L_ell_in(mu_s))`` on the separation grid
    (bins ``sedges``; first bin 0 for ell > 0), then per input bin
    ``(2 ell + 1) rnorm (-1)^(ell/2) sum_s n_s j_ell(k s) W(s) V Qs`` with
    ``W = (-1)^(ell_in/2) / (2 pi)^3 4 pi int_lo^hi k^2 j_ell_in(k s) dk`` (``utils.py:470-504``,
    integrated here by adaptive quadrature)."""
    from scipy.integrate import quad
    from scipy.special import spherical_jn
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    N = t(np.prod(geom.meshsize.astype(dt)))
    _norm = t(N / t(np.prod(geom.cellsize.astype(dt))))
    norm = np.asarray(_norm if norm is None else norm, dtype=dt)
    if norm.ndim <= 1:
        norm = norm * np.ones(len(ells), dtype=dt)
    rnorm = (_norm / norm / N).astype(dt)
    vlos = np.zeros(3)
    if isinstance(los, str):
        vlos['xyz'.index(los)] = 1.
    else:
        vlos = np.asarray(los, dtype='f8')
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    if meshes is None:
        Q = np.ones(geom.rshape, dtype=dt)
    else:
        W = [_to_complex(geom, m) for m in meshes]
        W2 = W[0] if len(W) == 1 else W[1]
        Q = (c2r(geom, (W[0] * np.conj(W2)).astype(W[0].dtype)) / N).astype(dt)
    sbin = CorrelationBins(geom, edges=sedges)
    svec = separation_coords(geom)
    snorm = sbin.snorm.astype('f8')
    smu = sum(xx.astype('f8') * ll for xx, ll in zip(svec, vlos)) / np.where(snorm == 0., 1., snorm)
    snmodes = sbin.nmodes
    with np.errstate(invalid='ignore', divide='ignore'):
        savg = np.where(snmodes == 0, 0., sbin.xavg)
    kout = np.where(bins.nmodes == 0, 0., bins.xavg)
    volume = float(np.prod(geom.boxsize.astype('f8')))

    def shell(ell, lo, hi, s):
        if s == 0.:
            return 4. * np.pi * (hi ** 3 - lo ** 3) / 3. if ell == 0 else 0.
        return 4. * np.pi * quad(lambda k: k * k * spherical_jn(ell, k * s), lo, hi, limit=500, epsabs=0.,
                                 epsrel=1e-9)[0]

    wmat = []
    for ellin in ellsin:
        blocks = []
        for ill, ell in enumerate(ells):
            Qs = sbin(Q.astype('f8') * legendre(ell, smu) * legendre(ellin, smu))
            if ell != 0:
                Qs[0] = 0.
            Qs = np.where(snmodes == 0, 0., Qs)
            cols = []
            for lo, hi in edgesin:
                w = np.array([shell(ellin, lo, hi, s) for s in savg]) * (-1) ** (ellin // 2) / (2. * np.pi) ** 3
                tq = w * volume * Qs
                cols.append((2 * ell + 1) * rnorm[ill] * (-1) ** (ell // 2)
                            * np.sum(snmodes[None, :] * spherical_jn(ell, kout[:, None] * savg[None, :]) * tq[None, :], axis=-1))
            blocks.append(np.array(cols))
        wmat.append(np.concatenate(blocks, axis=-1))
    return np.concatenate(wmat, axis=0).T


def compute_mesh2_spectrum_window_infinite(bins, edgesin, ellsin, los='z', meshes=None, norm=None):
    """``compute_mesh2_spectrum_window(..., flags=('infinite',))``, global line of sight
    (``mesh2.py:1095-1107``): column (ell_in, edge) is the estimator applied to
    ``r2c(Q V W(|s|) L_ell_in(mu_s))``, ``W = (-1)^(ell_in/2) / (2 pi)^3 4 pi int k^2 j_ell_in(k s) dk``
    (adaptive quadrature here)."""
    from scipy.integrate import quad
    from scipy.special import spherical_jn
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    N = t(np.prod(geom.meshsize.astype(dt)))
    _norm = t(N / t(np.prod(geom.cellsize.astype(dt))))
    norm = np.asarray(_norm if norm is None else norm, dtype=dt)
    if norm.ndim <= 1:
        norm = norm * np.ones(len(ells), dtype=dt)
    rnorm = (_norm / norm / N).astype(dt)
    vlos = np.zeros(3)
    if isinstance(los, str):
        vlos['xyz'.index(los)] = 1.
    else:
        vlos = np.asarray(los, dtype='f8')
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    Q = None
    if meshes is not None:
        W = [_to_complex(geom, m) for m in meshes]
        W2 = W[0] if len(W) == 1 else W[1]
        Q = (c2r(geom, (W[0] * np.conj(W2)).astype(W[0].dtype)) / N).astype(dt)
    svec = separation_coords(geom)
    s2 = (((t(0.) + svec[0] * svec[0]).astype(dt) + svec[1] * svec[1]).astype(dt) + svec[2] * svec[2]).astype(dt)
    snorm = np.sqrt(s2).astype('f8')
    smu = sum(xx.astype('f8') * ll for xx, ll in zip(svec, vlos)) / np.where(snorm == 0., 1., snorm)
    uniq, inverse = np.unique(snorm.ravel(), return_inverse=True)
    kvec = kcoords(geom)
    kl = [(kk * t(ll)).astype(dt) for kk, ll in zip(kvec, vlos)]
    num = (((t(0.) + kl[0]).astype(dt) + kl[1]).astype(dt) + kl[2]).astype(dt)
    knorm = bins.knorm()
    mu = (num / np.where(knorm == 0., t(1.), knorm)).astype(dt)
    volume = float(np.prod(geom.boxsize.astype('f8')))

    def shell(ell, lo, hi, s):
        if s == 0.:
            return 4. * np.pi * (hi ** 3 - lo ** 3) / 3. if ell == 0 else 0.
        return 4. * np.pi * quad(lambda k: k * k * spherical_jn(ell, k * s), lo, hi, limit=500, epsabs=0.,
                                 epsrel=1e-9)[0]

    wmat = []
    for ellin in ellsin:
        rows = []
        for lo, hi in edgesin.astype(dt):
            prof = np.array([shell(ellin, float(lo), float(hi), s) for s in uniq]) * (-1) ** (ellin // 2) / (2. * np.pi) ** 3
            A = (prof[inverse].reshape(snorm.shape) * legendre(ellin, smu) * volume)
            if Q is not None:
                A = A * Q
            A = r2c(geom, A.astype(dt))
            spectrum = []
            for ill, ell in enumerate(ells):
                odd = ell % 2
                leg = legendre(ell, mu)
                if odd:
                    leg = (leg + legendre(ell, (-mu).astype(dt))).astype(dt)
                spectrum.append((2 * ell + 1) / (1 + odd) * bins((A * leg).astype(A.dtype), remove_zero=True) * rnorm[ill])
            rows.append(np.concatenate(spectrum))
        wmat.append(np.array(rows))
    return np.real(np.concatenate(wmat, axis=0).T)


def compute_mesh2_spectrum_window_firstpoint_smooth(bins, sedges, edgesin, ellsin, meshes=None, swap=False):
    """``compute_mesh2_spectrum_window(..., los='firstpoint', flags=('smooth',))``, inputs ell_in
    or (ell_in, wide-angle order) (``mesh2.py:1196-1238``): ``Qs = 4 pi V_cell sum_{m, m1} sbin(Q Y_lm(shat) Y_l1m1(shat))``,
    ``Q = 4 pi / (2 ell_in + 1) c2r(conj(r2c(W1 Y_lm(xhat) Y_l1m1(xhat))) A0)``, then
    ``rnorm (-1)^(ell/2) sum_s n_s j_ell(k s) W(s) Qs`` (adaptive quadrature for W)."""
    from scipy.integrate import quad
    from scipy.special import spherical_jn
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    N = t(np.prod(geom.meshsize.astype(dt)))
    rnorm = np.full(len(ells), t(1.) / N, dtype=dt)
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    meshes = [np.ones(geom.rshape, dtype=dt)] if meshes is None else list(meshes)
    if swap:
        meshes = meshes[::-1]
    rmesh1 = _to_real(geom, meshes[0])
    A0 = _to_complex(geom, meshes[0] if len(meshes) == 1 else meshes[1])
    xvec = rcoords(geom)
    svec = separation_coords(geom)
    sbin = CorrelationBins(geom, edges=sedges)
    snmodes = sbin.nmodes
    with np.errstate(invalid='ignore', divide='ignore'):
        savg = np.where(snmodes == 0, 0., sbin.xavg)
    kout = np.where(bins.nmodes == 0, 0., bins.xavg)
    cellvol = float(np.prod(geom.cellsize.astype('f8')))

    def shell(ell, lo, hi, s):
        if s == 0.:
            return 4. * np.pi * (hi ** 3 - lo ** 3) / 3. if ell == 0 else 0.
        return 4. * np.pi * quad(lambda k: k * k * spherical_jn(ell, k * s), lo, hi, limit=500, epsabs=0.,
                                 epsrel=1e-9)[0]

    blocks = []
    for ellin, wa in _wa_terms(ellsin):  # wide-angle order wa: W1 |x|^-wa, Q |s|^wa (mesh2.py:1214)
        xf, sf = _wide_angle_factors(geom, wa)
        rho = (rmesh1 * xf).astype(dt) if wa else rmesh1
        block = np.zeros((len(edgesin), len(ells) * bins.nbins))
        for ill, ell in enumerate(ells):
            Qs = 0.
            for m1 in range(-ellin, ellin + 1):
                Y1 = get_ylm(ellin, m1)
                for m in range(-ell, ell + 1):
                    Y = get_ylm(ell, m)
                    F = r2c(geom, ((rho * Y(*xvec)).astype(dt) * Y1(*xvec)).astype(dt))
                    Q = (t(4. * np.pi / (2 * ellin + 1)) * c2r(geom, (np.conj(F) * A0).astype(np.complex64))).astype(dt)
                    if wa:
                        Q = (Q * sf).astype(dt)
                    Qs = Qs + 4. * np.pi * sbin(Q.astype('f8') * Y(*svec) * Y1(*svec)) * cellvol
            if ell != 0:
                Qs[0] = 0.
            Qs = np.where(snmodes == 0, 0., Qs)
            for e, (lo, hi) in enumerate(edgesin.astype(dt)):
                w = np.array([shell(ellin, float(lo), float(hi), s) for s in savg]) * (-1) ** (ellin // 2) / (2. * np.pi) ** 3
                block[e, ill * bins.nbins:(ill + 1) * bins.nbins] = (-1) ** (ell // 2) * np.sum(
                    snmodes[None, :] * spherical_jn(ell, kout[:, None] * savg[None, :]) * (w * Qs)[None, :], axis=-1) * rnorm[ill]
        blocks.append(block)
    wmat = np.concatenate(blocks, axis=0).T
    if ells[0] % 2:
        wmat[:bins.nbins] = 0.
    return wmat


def compute_smooth2_spectrum_window(s, windows, snmodes, edgesin, ellsin, ells, kout):
    """``compute_smooth2_spectrum_window(window, edgesin, ellsin, bin, flags=('rect',))``
    (``mesh2.py:803-918``) as plain loops: ``windows`` {q: W_q(s)} or, with wide-angle inputs
    (ell_in, n), {(q, n): W_q,n(s)} with the extra s^n of ``mesh2.py:869``; coefficients
    ``(2 ell + 1) (ell ellin q; 0 0 0)^2`` from sympy's Wigner 3j symbols."""
    from scipy.special import spherical_jn
    from sympy.physics.wigner import wigner_3j
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    savg = np.where(snmodes == 0, 0., s)
    wmat = np.zeros((len(ells) * len(kout), len(ellsin) * len(edgesin)))
    for iin, ellin in enumerate(ellsin):
        ellin, wa = ellin if isinstance(ellin, tuple) else (ellin, None)
        for ill, ell in enumerate(ells):
            Qs = np.zeros_like(s)
            for q in range(abs(ell - ellin), ell + ellin + 1):
                c = (2 * ell + 1) * float(wigner_3j(ell, ellin, q, 0, 0, 0)) ** 2
                key = q if wa is None else (q, wa)
                if abs(c) >= 1e-7 and key in windows:
                    Qs = Qs + c * windows[key]
            Qs = np.where(snmodes == 0, 0., Qs) * savg ** (wa or 0)
            for e, (lo, hi) in enumerate(edgesin):
                kin = (lo + hi) / 2.
                tophat = (-1) ** (ellin // 2) / (2. * np.pi) ** 3 * spherical_jn(ellin, savg * kin) * 4. / 3. * np.pi * (hi ** 3 - lo ** 3) * Qs
                for b, k in enumerate(kout):
                    wmat[ill * len(kout) + b, iin * len(edgesin) + e] = (-1) ** (ell // 2) * np.sum(
                        spherical_jn(ell, k * savg) * snmodes * tophat)
    return wmat


def compute_mesh2_spectrum_window_firstpoint_infinite(bins, edgesin, ellsin, meshes=None, swap=False):
    """``compute_mesh2_spectrum_window(..., los='firstpoint', flags=('infinite',))``, inputs
    ell_in or (ell_in, wide-angle order) (``mesh2.py:1240-1262``): ``Qs = V_cell sum_m1 Y_l1m1(shat) Q``, then per input bin
    ``4 pi rnorm sum_m bin(Y_lm(khat) r2c(W(|s|) Qs))`` (adaptive quadrature for W)."""
    from scipy.integrate import quad
    from scipy.special import spherical_jn
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    N = t(np.prod(geom.meshsize.astype(dt)))
    rnorm = t(1.) / N
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    meshes = [np.ones(geom.rshape, dtype=dt)] if meshes is None else list(meshes)
    if swap:
        meshes = meshes[::-1]
    rmesh1 = _to_real(geom, meshes[0])
    A0 = _to_complex(geom, meshes[0] if len(meshes) == 1 else meshes[1])
    xvec, kvec, svec = rcoords(geom), kcoords(geom), separation_coords(geom)
    s2 = (((t(0.) + svec[0] * svec[0]).astype(dt) + svec[1] * svec[1]).astype(dt) + svec[2] * svec[2]).astype(dt)
    snorm = np.sqrt(s2).astype('f8')
    uniq, inverse = np.unique(snorm.ravel(), return_inverse=True)
    cellvol = float(np.prod(geom.cellsize.astype('f8')))

    def shell(ell, lo, hi, s):
        if s == 0.:
            return 4. * np.pi * (hi ** 3 - lo ** 3) / 3. if ell == 0 else 0.
        return 4. * np.pi * quad(lambda k: k * k * spherical_jn(ell, k * s), lo, hi, limit=500, epsabs=0.,
                                 epsrel=1e-9)[0]

    blocks = []
    for ellin, wa in _wa_terms(ellsin):  # wide-angle order wa: W1 |x|^-wa, Q |s|^wa (mesh2.py:1249)
        xf, sf = _wide_angle_factors(geom, wa)
        rho = (rmesh1 * xf).astype(dt) if wa else rmesh1
        profiles = []
        for lo, hi in edgesin.astype(dt):
            prof = np.array([shell(ellin, float(lo), float(hi), x) for x in uniq]) * (-1) ** (ellin // 2) / (2. * np.pi) ** 3
            profiles.append(prof[inverse].reshape(snorm.shape))
        block = np.zeros((len(edgesin), len(ells) * bins.nbins), dtype='c16')
        for ill, ell in enumerate(ells):
            for m in range(-ell, ell + 1):
                Y = get_ylm(ell, m)
                Qs = 0.
                for m1 in range(-ellin, ellin + 1):
                    Y1 = get_ylm(ellin, m1)
                    F = r2c(geom, ((rho * Y(*xvec)).astype(dt) * Y1(*xvec)).astype(dt))
                    Q = (t(4. * np.pi / (2 * ellin + 1)) * c2r(geom, (np.conj(F) * A0).astype(np.complex64))).astype(dt)
                    if wa:
                        Q = (Q * sf).astype(dt)
                    Qs = Qs + Y1(*svec).astype('f8') * Q * cellvol
                for e, prof in enumerate(profiles):
                    A = (Y(*kvec) * r2c(geom, (prof * Qs).astype(dt))).astype(np.complex64)
                    block[e, ill * bins.nbins:(ill + 1) * bins.nbins] += 4. * np.pi * bins(A, remove_zero=ell == 0) * rnorm
        blocks.append(block)
    wmat = np.concatenate(blocks, axis=0).T
    nb = bins.nbins
    first = wmat[:nb].imag if ells[0] % 2 else wmat[:nb].real
    wmat = wmat.real.copy()
    wmat[:nb] = first
    return wmat


def real_gaunt(lm1, lm2, lm3):
    """Integral over the sphere of three real Y_lm (``utils.py:540-622``), by quadrature of the
    oracle's own Y_lm (``get_ylm``) on a Gauss-Legendre x uniform-phi grid."""
    x, wx = np.polynomial.legendre.leggauss(16)
    phi = 2. * np.pi * np.arange(48) / 48.
    st = np.sqrt(1. - x ** 2)[:, None]
    X, Y, Z = st * np.cos(phi)[None, :], st * np.sin(phi)[None, :], np.broadcast_to(x[:, None], (16, 48))
    prod = 1.
    for ell, m in (lm1, lm2, lm3):
        prod = prod * get_ylm(ell, m)(X, Y, Z)
    return float(np.sum(wx[:, None] * (2. * np.pi / 48.) * prod))


def compute_mesh2_spectrum_window_local_smooth(bins, sedges, edgesin, ellsin, meshes=None, swap=False):
    """``compute_mesh2_spectrum_window(..., ellsin=(ellsin, 'local'), los='firstpoint',
    flags=('smooth',))`` (``mesh2.py:1319-1361``, ``1447-1455``), as direct sums over every
    (m, m1, m2, mp) term."""
    from scipy.integrate import quad
    from scipy.special import spherical_jn
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    N = t(np.prod(geom.meshsize.astype(dt)))
    rnorm = t(1.) / N
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    meshes = [np.ones(geom.rshape, dtype=dt)] if meshes is None else list(meshes)
    if swap:
        meshes = meshes[::-1]
    rmesh1 = _to_real(geom, meshes[0])
    rmesh2 = rmesh1 if len(meshes) == 1 else _to_real(geom, meshes[1])
    xvec, svec = rcoords(geom), separation_coords(geom)
    sbin = CorrelationBins(geom, edges=sedges)
    snmodes = sbin.nmodes
    with np.errstate(invalid='ignore', divide='ignore'):
        savg = np.where(snmodes == 0, 0., sbin.xavg)
    kout = np.where(bins.nmodes == 0, 0., bins.xavg)
    cellvol = float(np.prod(geom.cellsize.astype('f8')))

    def shell(ell, lo, hi, s):
        if s == 0.:
            return 4. * np.pi * (hi ** 3 - lo ** 3) / 3. if ell == 0 else 0.
        return 4. * np.pi * quad(lambda k: k * k * spherical_jn(ell, k * s), lo, hi, limit=500, epsabs=0.,
                                 epsrel=1e-9)[0]

    coeff2 = {(0, 0): [(0, 1.), (4, -7. / 18.)], (0, 2): [(2, 1. / 2.), (4, -5. / 18.)], (2, 2): [(4, 35. / 18.)]}
    coeff2[2, 0] = coeff2[0, 2]
    wmat = np.zeros((len(ellsin), len(edgesin), len(ells) * bins.nbins))
    for ell1 in (2, 0):
        for ell2 in (2, 0):
            ps = [p for p in (0, 2, 4) if abs(real_gaunt((p, 0), (ell1, 0), (ell2, 0))) > 1e-10]
            block = np.zeros((len(edgesin), len(ells) * bins.nbins))
            for ill, ell in enumerate(ells):
                Qs = {p: 0. for p in ps}
                for m1 in range(-ell1, ell1 + 1):
                    for m2 in range(-ell2, ell2 + 1):
                        for m in range(-ell, ell + 1):
                            Yl = get_ylm(ell, m)
                            F = r2c(geom, ((rmesh1 * Yl(*xvec)).astype(dt) * get_ylm(ell1, m1)(*xvec)).astype(dt))
                            B = r2c(geom, (rmesh2 * get_ylm(ell2, m2)(*xvec)).astype(dt))
                            Q = t((4. * np.pi) ** 2 / ((2 * ell1 + 1) * (2 * ell2 + 1))) * c2r(geom, (np.conj(F) * B).astype(np.complex64))
                            for p in ps:
                                tmp = 0.
                                for mp in range(-p, p + 1):
                                    rg = real_gaunt((p, mp), (ell1, m1), (ell2, m2))
                                    if abs(rg) > 1e-12:
                                        tmp = tmp + rg * Yl(*svec) * get_ylm(p, mp)(*svec) * Q.astype('f8')
                                if not np.isscalar(tmp):
                                    Qs[p] = Qs[p] + 4. * np.pi * sbin(tmp) * cellvol
                for p in ps:
                    Qp = np.broadcast_to(np.asarray(Qs[p], dtype='f8'), savg.shape).copy()
                    if ell != 0:
                        Qp[0] = 0.
                    Qp = np.where(snmodes == 0, 0., Qp)
                    for e, (lo, hi) in enumerate(edgesin.astype(dt)):
                        w = np.array([shell(p, float(lo), float(hi), s) for s in savg]) * (-1) ** (p // 2) / (2. * np.pi) ** 3
                        block[e, ill * bins.nbins:(ill + 1) * bins.nbins] += (-1) ** (ell // 2) * np.sum(
                            snmodes[None, :] * spherical_jn(ell, kout[:, None] * savg[None, :]) * (w * Qp)[None, :], axis=-1) * rnorm
            for illin, ellin in enumerate(ellsin):
                wmat[illin] += sum(c * (ell == ellin) for ell, c in coeff2[ell1, ell2]) * block
    wmat = wmat.reshape(-1, wmat.shape[-1]).T
    if ells[0] % 2:
        wmat[:bins.nbins] = 0.
    return wmat


def compute_mesh2_spectrum_window_local_infinite(bins, edgesin, ellsin, meshes=None, swap=False):
    """``compute_mesh2_spectrum_window(..., ellsin=(ellsin, 'local'), los='firstpoint',
    flags=('infinite',))`` (``mesh2.py:1363-1396``, ``1447-1455``), as direct sums."""
    from scipy.integrate import quad
    from scipy.special import spherical_jn
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    ells = bins.ells
    N = t(np.prod(geom.meshsize.astype(dt)))
    rnorm = t(1.) / N
    edgesin = np.asarray(edgesin, dtype='f8')
    if edgesin.ndim != 2:
        edgesin = np.column_stack([edgesin[:-1], edgesin[1:]])
    meshes = [np.ones(geom.rshape, dtype=dt)] if meshes is None else list(meshes)
    if swap:
        meshes = meshes[::-1]
    rmesh1 = _to_real(geom, meshes[0])
    rmesh2 = rmesh1 if len(meshes) == 1 else _to_real(geom, meshes[1])
    xvec, kvec, svec = rcoords(geom), kcoords(geom), separation_coords(geom)
    s2 = (((t(0.) + svec[0] * svec[0]).astype(dt) + svec[1] * svec[1]).astype(dt) + svec[2] * svec[2]).astype(dt)
    snorm = np.sqrt(s2).astype('f8')
    uniq, inverse = np.unique(snorm.ravel(), return_inverse=True)
    cellvol = float(np.prod(geom.cellsize.astype('f8')))

    def shell(ell, lo, hi, s):
        if s == 0.:
            return 4. * np.pi * (hi ** 3 - lo ** 3) / 3. if ell == 0 else 0.
        return 4. * np.pi * quad(lambda k: k * k * spherical_jn(ell, k * s), lo, hi, limit=500, epsabs=0.,
                                 epsrel=1e-9)[0]

    prof = {p: [(np.array([shell(p, float(lo), float(hi), x) for x in uniq]) * (-1) ** (p // 2)
                 / (2. * np.pi) ** 3)[inverse].reshape(snorm.shape) for lo, hi in edgesin.astype(dt)] for p in (0, 2, 4)}
    coeff2 = {(0, 0): [(0, 1.), (4, -7. / 18.)], (0, 2): [(2, 1. / 2.), (4, -5. / 18.)], (2, 2): [(4, 35. / 18.)]}
    coeff2[2, 0] = coeff2[0, 2]
    wmat = np.zeros((len(ellsin), len(edgesin), len(ells) * bins.nbins), dtype='c16')
    for ell1 in (2, 0):
        for ell2 in (2, 0):
            ps = [p for p in (0, 2, 4) if abs(real_gaunt((p, 0), (ell1, 0), (ell2, 0))) > 1e-10]
            block = np.zeros((len(edgesin), len(ells) * bins.nbins), dtype='c16')
            for ill, ell in enumerate(ells):
                for m in range(-ell, ell + 1):
                    Yl = get_ylm(ell, m)
                    Qs = {p: 0. for p in ps}
                    for m1 in range(-ell1, ell1 + 1):
                        for m2 in range(-ell2, ell2 + 1):
                            F = r2c(geom, ((rmesh1 * Yl(*xvec)).astype(dt) * get_ylm(ell1, m1)(*xvec)).astype(dt))
                            B = r2c(geom, (rmesh2 * get_ylm(ell2, m2)(*xvec)).astype(dt))
                            Q = t((4. * np.pi) ** 2 / ((2 * ell1 + 1) * (2 * ell2 + 1))) * c2r(geom, (np.conj(F) * B).astype(np.complex64))
                            for p in ps:
                                for mp in range(-p, p + 1):
                                    rg = real_gaunt((p, mp), (ell1, m1), (ell2, m2))
                                    if abs(rg) > 1e-12:
                                        Qs[p] = Qs[p] + rg * get_ylm(p, mp)(*svec) * Q.astype('f8')
                    for e in range(len(edgesin)):
                        xi = sum(prof[p][e] * Qs[p] * cellvol for p in ps)
                        A = (Yl(*kvec) * r2c(geom, np.asarray(xi, dtype=dt))).astype(np.complex64)
                        block[e, ill * bins.nbins:(ill + 1) * bins.nbins] += 4. * np.pi * bins(A, remove_zero=ell == 0) * rnorm
            for illin, ellin in enumerate(ellsin):
                wmat[illin] += sum(c * (ell == ellin) for ell, c in coeff2[ell1, ell2]) * block
    wmat = wmat.reshape(-1, wmat.shape[-1]).T
    nb = bins.nbins
    first = wmat[:nb].imag if ells[0] % 2 else wmat[:nb].real
    wmat = wmat.real.copy()
    wmat[:nb] = first
    return wmat

# --------------------------------------------------------------------------- FKP

def next_fft_size(n, primes=(2, 3, 5, 7), divisors=()):
    """``next_fft_size`` (``mesh.py:2304-2340``)."""
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


def get_mesh_attrs(*positions, meshsize=None, boxsize=None, boxcenter=None, cellsize=None,
                   boxpad=2., primes=None, dtype=np.float32):
    """``get_mesh_attrs`` (``mesh.py:2271-2381``) without sharding; returns a Geometry."""
    dt = np.dtype(dtype)
    if cellsize is not None and meshsize is not None:
        meshsize = np.broadcast_to(np.asarray(meshsize, 'i4'), (3,))
        boxsize = meshsize * np.broadcast_to(np.asarray(cellsize, dt), (3,))
    if boxsize is None or boxcenter is None:
        pmin = np.min([np.min(p, axis=0) for p in positions if p.size], axis=0)
        pmax = np.max([np.max(p, axis=0) for p in positions if p.size], axis=0)
        delta = np.abs(pmax - pmin)
        if boxcenter is None:
            boxcenter = (dt.type(0.5) * (pmin + pmax)).astype(dt)
        if boxsize is None:
            boxsize = (delta.max() * dt.type(boxpad)).astype(dt)
    boxsize = np.broadcast_to(np.asarray(boxsize, dt), (3,)).copy()
    if meshsize is None:
        cs = np.broadcast_to(np.asarray(cellsize, dt), (3,))
        meshsize = np.ceil((boxsize / cs).astype(dt)).astype('i4')
        meshsize = np.array([next_fft_size(n, primes=primes or ()) for n in meshsize])
        boxsize = (meshsize * cs).astype(dt)
    return Geometry(meshsize, boxsize=boxsize, boxcenter=boxcenter, dtype=dt)


def fkp_particles(data_pos, data_w, rand_pos, rand_w, dtype=np.float32):
    """``FKPField.particles`` (``mesh.py:2965-2971``): data - alpha * randoms."""
    dt = np.dtype(dtype)
    data_w = np.ones(len(data_pos), dt) if data_w is None else np.asarray(data_w, dt)
    rand_w = np.ones(len(rand_pos), dt) if rand_w is None else np.asarray(rand_w, dt)
    alpha = (np.sum(data_w, dtype=dt) / np.sum(rand_w, dtype=dt)).astype(dt)
    pos = np.concatenate([np.asarray(data_pos, dt), np.asarray(rand_pos, dt)])
    w = np.concatenate([data_w, (-alpha * rand_w).astype(dt)])
    return pos, w, alpha


def fkp2_shotnoise(weights):
    """``compute_fkp2_shotnoise`` auto case (``mesh2.py:601-611``): sum of w^2."""
    w = np.asarray(weights, dtype='f8')
    return float(np.sum(w * w))


def fkp2_normalization(geom, data_pos, data_w, rand_pos, rand_w, cellsize=10., split=None):
    """``compute_fkp2_normalization`` auto case (``mesh2.py:516-574``, ``mesh.py:3002-3118``).

    alpha * sum(rho_d * rho_r) / V_cell with CIC meshes at the given cellsize (None: the
    geometry's own mesh).  ``split=(seed, ids)``: the randoms split in two disjoint halves by
    one uniform per id (``split_particles``, ``mesh.py:3160-3204``), alpha^2 rescaled by
    each half's weight share (``mesh2.py:543-553``), sum(rho_r0 * rho_r1) / V_cell.
    """
    dt = geom.dtype
    data_w = np.ones(len(data_pos), dt) if data_w is None else np.asarray(data_w, dt)
    rand_w = np.ones(len(rand_pos), dt) if rand_w is None else np.asarray(rand_w, dt)
    alpha = np.sum(data_w.astype('f8')) / np.sum(rand_w.astype('f8'))
    g2 = geom if cellsize is None else norm_geometry(geom, cellsize)

    def cic(pos, w):
        return paint_field(g2, pos, w, resampler='cic', interlacing=0, compensate=False).astype('f8')

    if split is not None:
        m0, m1 = split_masks(split, len(rand_pos), nsplits=2)
        w0, w1 = (rand_w * m0).astype(dt), (rand_w * m1).astype(dt)
        total = np.sum(rand_w.astype('f8'))
        alpha = alpha**2 * (total / np.sum(w0.astype('f8'))) * (total / np.sum(w1.astype('f8')))
        return float(alpha * np.sum(cic(rand_pos, w0) * cic(rand_pos, w1)) / np.prod(g2.cellsize.astype('f8')))
    return float(alpha * np.sum(cic(data_pos, data_w) * cic(rand_pos, rand_w)) / np.prod(g2.cellsize.astype('f8')))


def split_masks(seed, size, nsplits=2):
    """Masks of ``split_particles`` (``mesh.py:3160-3204``) for one field split ``nsplits`` ways:
    x = jax.random.uniform per particle (``create_sharded_random``, ``mesh.py:237-329``, x64),
    subsample i keeps i / n <= x < (i + 1) / n."""
    from .threefry import seed_key, fold_in_index, uniform_per_key, uniform
    key, ids = seed if isinstance(seed, tuple) else (seed, None)
    if isinstance(ids, str) and ids == 'index':
        ids = np.arange(size)
    if ids is None:
        x = uniform(seed_key(key), (size,), np.float64, partitionable=True)
    else:
        x = uniform_per_key(fold_in_index(seed_key(key), np.asarray(ids, dtype='i8')), 1, np.float64)[:, 0]
    return [(x >= i * 1. / nsplits) & (x < (i + 1) * 1. / nsplits) for i in range(nsplits)]


def norm_geometry(geom, cellsize=10.):
    """``get_halo_for_new_mattrs(mattrs, cellsize=...)`` (``mesh.py:3002-3039``), no sharding."""
    dt = geom.dtype
    cs = np.broadcast_to(np.asarray(cellsize, dt), (3,))
    meshsize = np.ceil((geom.boxsize / cs).astype(dt)).astype('i4')
    boxsize = (meshsize * cs.astype('f8')).astype(dt)
    odd = (meshsize - geom.meshsize) % 2 != 0
    if np.any(odd):
        # keep an even difference with the painted mesh: one more cell on every axis
        cell = (boxsize / meshsize.astype(dt)).astype(dt)
        meshsize = meshsize + 1
        boxsize = (cell * meshsize.astype(dt)).astype(dt)
    return Geometry(meshsize, boxsize=boxsize, boxcenter=geom.boxcenter, dtype=dt, backend=geom.backend)


def separation_coords(geom):
    """``MeshAttrs.rcoords(kind='separation')`` (``mesh.py:392-394``): fftfreq(n) * cellsize * n."""
    dt = geom.dtype
    out = []
    for axis in range(3):
        n = int(geom.meshsize[axis])
        sf = np.where(np.arange(n) < (n + 1) // 2, np.arange(n), np.arange(n) - n).astype(dt)
        x = ((sf / dt.type(n)).astype(dt) * geom.cellsize[axis]).astype(dt) * dt.type(n)
        shape = [1, 1, 1]
        shape[axis] = n
        out.append(x.astype(dt).reshape(shape))
    return out


class CorrelationBins:
    """``BinMesh2CorrelationPoles(mattrs, edges={'step': step}, ells)`` restated
    (``mesh2.py:124-192``, ``_make_edges2('real')`` ``mesh2.py:25-62``): |s| of the separation
    grid binned by ``digitize``; unit weights."""

    def __init__(self, geom, step=None, edges=None, ells=(0, 2, 4), mode_oversampling=0):
        dt = geom.dtype
        self.geom = geom
        self.ells = tuple(sorted((ells,) if np.ndim(ells) == 0 else ells))
        if edges is None:
            vec0 = geom.cellsize.min()
            vecmax = dt.type(vec0 * dt.type(np.min(geom.meshsize))) / dt.type(2.)
            edges = np.arange(0., float(vecmax), step)
        self.edges = np.asarray(edges, dtype='f8')
        sx, sy, sz = separation_coords(geom)
        s2 = (((dt.type(0.) + sx * sx).astype(dt) + sy * sy).astype(dt) + sz * sz).astype(dt)
        self.snorm = np.sqrt(s2).astype(dt)
        nb = len(self.edges) + 1
        # mode oversampling (mesh2.py:48-61): one binning per integer shift of the separations,
        # |s + shift| in the geometry's dtype; nmodes their mean, xavg the summed |s + shift| over it
        r = range(-int(mode_oversampling), int(mode_oversampling) + 1)
        shifts = list(product(r, r, r)) if mode_oversampling else [(0, 0, 0)]
        self.ibins, nmodes, ssum = [], 0., 0.
        for sh in shifts:
            if mode_oversampling:
                a, b, c = [(x + dt.type(v)).astype(dt) for x, v in zip((sx, sy, sz), sh)]
                norm = np.sqrt((((dt.type(0.) + a * a).astype(dt) + b * b).astype(dt) + c * c).astype(dt)).astype(dt)
                norm = np.broadcast_to(norm, self.snorm.shape)
            else:
                norm = self.snorm
            ib = np.searchsorted(self.edges.astype(dt), norm.ravel(), side='right')
            self.ibins.append(ib)
            nmodes = nmodes + np.bincount(ib, minlength=nb)[1:-1].astype('f8')
            ssum = ssum + np.bincount(ib, weights=norm.ravel().astype('f8'), minlength=nb)[1:-1]
        self.ibin = self.ibins[0].reshape(self.snorm.shape)
        self.nmodes = nmodes / len(shifts)
        with np.errstate(invalid='ignore', divide='ignore'):
            self.xavg = ssum / self.nmodes

    @property
    def nbins(self):
        return len(self.edges) - 1

    def __call__(self, value, remove_zero=False):
        value = np.array(value, dtype='f8', copy=True)
        if remove_zero:
            value[0, 0, 0] = 0.
        nb = len(self.edges) + 1
        total = sum(np.bincount(ib, weights=value.ravel(), minlength=nb)[1:-1] for ib in self.ibins)
        return total / len(self.ibins) / self.nmodes


def compute_mesh2_correlation(mesh, bins, los='z', mesh2=None):
    """Fixed line-of-sight branch of ``compute_mesh2_correlation`` (``mesh2.py:465-499``):
    A = c2r(|delta|^2) (or c2r(conj(d1) d2)), xi_0 = bin(A), xi_ell = (2 ell + 1) bin(A L_ell(mu))
    (s = 0 dropped), mu = s.los / |s| with |s|(0) = 1; num_raw = xi / V_cell."""
    geom = bins.geom
    dt = geom.dtype
    d1 = _to_complex(geom, mesh)
    if mesh2 is None:
        prod = (d1.real**2 + d1.imag**2).astype(d1.dtype)
    else:
        prod = np.conj(d1) * _to_complex(geom, mesh2)
    A = c2r(geom, prod)
    vlos = {'x': (1., 0., 0.), 'y': (0., 1., 0.), 'z': (0., 0., 1.)}[los] if isinstance(los, str) else los
    sx, sy, sz = separation_coords(geom)
    s = bins.snorm.copy()
    s[0, 0, 0] = 1.
    mu = ((sx * dt.type(vlos[0]) + sy * dt.type(vlos[1])) + sz * dt.type(vlos[2])) / s
    cellvol = float(np.prod(geom.cellsize.astype('f8')))
    out = {}
    for ell in bins.ells:
        if ell == 0:
            num = bins(A)
        else:
            num = (2 * ell + 1) * bins(A * legendre(ell, mu.astype(dt)), remove_zero=True)
        out[ell] = num / cellvol
    return {'num_raw': np.array([out[ell] for ell in bins.ells]), 'nmodes': bins.nmodes, 'xavg': bins.xavg}


def compute_mesh2_correlation_firstpoint(mesh, bins, mesh2=None, swap=False):
    """First-point branch of ``compute_mesh2_correlation`` (``mesh2.py:414-463``):
    xi_0 = bin(c2r(|A0|^2)), xi_ell = 4 pi bin(sum_m c2r(conj(r2c(rho Y_lm(xhat))) A0) Y_lm(shat))
    with the s = 0 cell dropped; num_raw = xi / V_cell."""
    geom = bins.geom
    dt = geom.dtype
    m1, m2 = (mesh2, mesh) if (swap and mesh2 is not None) else (mesh, mesh2)
    A0 = _to_complex(geom, m1 if m2 is None else m2)
    rho = _to_real(geom, m1)
    xvec = rcoords(geom)
    svec = separation_coords(geom)
    cellvol = float(np.prod(geom.cellsize.astype('f8')))
    out = []
    for ell in bins.ells:
        if ell == 0:
            prod = (A0.real**2 + A0.imag**2).astype(A0.dtype) if m2 is None else np.conj(_to_complex(geom, m1)) * A0
            out.append(bins(c2r(geom, prod)) / cellvol)
            continue
        carry = np.zeros(geom.rshape, dtype=dt)
        for m in range(-ell, ell + 1):
            Y = get_ylm(ell, m)
            F = r2c(geom, (rho * Y(*xvec)).astype(dt))
            carry = (carry + c2r(geom, np.conj(F) * A0) * Y(*svec)).astype(dt)
        out.append(4. * np.pi * bins(carry, remove_zero=True) / cellvol)
    return {'num_raw': np.array(out), 'nmodes': bins.nmodes, 'xavg': bins.xavg}


def spherical_jn(ell, x):
    """``get_spherical_jn(ell)`` (``utils.py:443-450``) in float64: the closed form for x > 0.1
    (``utils.py:419-440``; evaluated by scipy's spherical Bessel function, the same function)
    and, for x <= 0.1, its Taylor series x^l / (2l+1)!! sum_k (-x^2/2)^k / (k! (2l+3)...(2l+2k+1))
    through x^(l+10), the terms the reference keeps."""
    from scipy import special
    x = np.asarray(x, dtype='f8')
    out = np.empty_like(x)
    hi = x > 0.1
    out[hi] = special.spherical_jn(ell, x[hi])
    xl = x[~hi]
    lead = xl**ell / np.prod(np.arange(1, 2 * ell + 2, 2, dtype='f8'))
    term, total = lead.copy(), lead.copy()
    for k in range(5):
        term = term * (-0.5 * xl * xl) / ((k + 1) * (2 * ell + 2 * k + 3))
        total = total + term
    out[~hi] = total
    return out


def compute_mesh2_correlation_bessel(mesh, bins, los='z', mesh2=None, klimit=None):
    """``compute_mesh2_correlation`` with ``BinMesh2CorrelationPoles(basis='bessel')``
    (``mesh2.py:169-177`` and the 'bessel' branches of ``mesh2.py:414-500``).

    The estimator's Fourier-space mode values A_ell (fixed los: |d1|^2 or conj(d1) d2 times
    L_ell(mu); first point: |A0|^2 and conj(sum_m r2c(rho Y_lm(xhat)) Y_lm(khat)) A0), k = 0
    dropped for ell > 0, projected as (-1)^(ell//2) sum_k Re(A_ell) j_ell(|k| s_b) / N over
    the stored half-complex modes (no Hermitian weight), s_b = xavg; |k| and |k| s_b in the
    geometry's dtype, j_ell in float64; times 1, 2 ell + 1 or 4 pi; num_raw = / V_cell.
    """
    geom = bins.geom
    dt = geom.dtype
    t = dt.type
    kx, ky, kz = kcoords(geom)
    k2 = (((t(0.) + kx * kx).astype(dt) + ky * ky).astype(dt) + kz * kz).astype(dt)
    knorm = np.sqrt(k2).astype(dt)
    sep = np.asarray(bins.xavg).astype(dt)
    mask = 1.
    if klimit is not None:
        mask = ((knorm >= t(klimit[0])) & (knorm < t(klimit[1]))).astype('f8')
    nmesh = float(np.prod(geom.meshsize.astype('f8')))
    cellvol = float(np.prod(geom.cellsize.astype('f8')))

    def project(value, ell):
        value = np.real(value).astype('f8') * mask
        out = np.empty(len(sep))
        for b, s in enumerate(sep):
            x = (knorm * s).astype(dt)
            out[b] = np.sum(value * spherical_jn(ell, x))
        return (-1.)**(ell // 2) * out / nmesh

    out = []
    if isinstance(los, str) and los in ('firstpoint', 'local', 'endpoint'):
        swap = los == 'endpoint'
        m1, m2 = (mesh2, mesh) if (swap and mesh2 is not None) else (mesh, mesh2)
        A0 = _to_complex(geom, m1 if m2 is None else m2)
        rho = _to_real(geom, m1)
        xvec = rcoords(geom)
        kvec = (kx, ky, kz)
        for ell in bins.ells:
            if ell == 0:
                A = (A0.real**2 + A0.imag**2).astype(dt) if m2 is None else np.conj(_to_complex(geom, m1)) * A0
                out.append(project(A, 0))
                continue
            carry = np.zeros(geom.cshape, dtype=A0.dtype)
            for m in range(-ell, ell + 1):
                Y = get_ylm(ell, m)
                F = r2c(geom, (rho * Y(*xvec)).astype(dt))
                carry = (carry + F * Y(*kvec)).astype(A0.dtype)
            A = np.conj(carry) * A0
            A[0, 0, 0] = 0.
            out.append(4. * np.pi * project(A, ell))
    else:
        vlos = {'x': (1., 0., 0.), 'y': (0., 1., 0.), 'z': (0., 0., 1.)}[los] if isinstance(los, str) else los
        d1 = _to_complex(geom, mesh)
        A = (d1.real**2 + d1.imag**2).astype(dt) if mesh2 is None else np.conj(d1) * _to_complex(geom, mesh2)
        kl = [(kk * t(ll)).astype(dt) for kk, ll in zip((kx, ky, kz), vlos)]
        mu_num = (((t(0.) + kl[0]).astype(dt) + kl[1]).astype(dt) + kl[2]).astype(dt)
        kn = knorm.copy()
        kn[0, 0, 0] = 1.
        mu = (mu_num / kn).astype(dt)
        for ell in bins.ells:
            if ell == 0:
                out.append(project(A, 0))
                continue
            value = A * legendre(ell, mu)
            value[0, 0, 0] = 0.
            out.append((2 * ell + 1) * project(value, ell))
    return {'num_raw': np.array(out) / cellvol, 'nmodes': bins.nmodes, 'xavg': bins.xavg}
