"""Particle painting, reading and the ``_paint`` pipeline (oracle; test only).

Restates:

- ``resamplers.py:57-63``  NGP / CIC / TSC / PCS kernels (same float op order);
- ``resamplers.py:66-97``  paint: base index floor (even order) or
  round-half-even (odd order), stencil offsets ``arange(order) - (order-1)//2``
  in ``itertools.product`` order, periodic wrap, serial scatter-add;
- ``resamplers.py:100-125`` read (the gather transpose);
- ``resamplers.py:16-26``  compensation ``prod_d sinc(k_d / 2pi)^-order``;
- ``mesh.py:2673-2754``    ``_paint``: position normalisation, interlacing
  phases with circular k, compensation, optional c2r.

float32 mode reproduces the reference's operation order: the scatter is an
``np.add.at`` in particle order per stencil offset (the order of XLA's serial
CPU scatter), so the mesh matches the reference's to float32 rounding of the
(order-dependent) sums.
"""
from itertools import product

import numpy as np

from . import _native
from .coords import Geometry, kcoords, r2c, c2r


def kernel(order, s, dtype):
    """``_resampler_kernels[order](s)`` (``resamplers.py:57-63``) in ``dtype``."""
    t = np.dtype(dtype).type
    s = s.astype(dtype, copy=False)
    if order == 1:
        return np.ones_like(s)
    if order == 2:
        return (t(1.) - s).astype(dtype)
    if order == 3:
        a = (s <= t(0.5)).astype(dtype) * (t(0.75) - s * s)
        b = ((t(0.5) < s).astype(dtype) / t(2.)) * ((t(1.5) - s) * (t(1.5) - s))
        return (a + b).astype(dtype)
    if order == 4:
        s2 = s * s
        s3 = s2 * s
        a = ((s <= t(1.)).astype(dtype) / t(6.)) * ((t(4.) - t(6.) * s2) + t(3.) * s3)
        u = t(2.) - s
        b = ((t(1.) < s).astype(dtype) / t(6.)) * ((u * u) * u)
        return (a + b).astype(dtype)
    raise ValueError(order)


def kernel_derivative(order, s, dtype):
    """dW/ds of the kernels above (what JAX autodiff of ``resamplers.py:57-63`` gives)."""
    t = np.dtype(dtype).type
    s = s.astype(dtype, copy=False)
    if order == 1:
        return np.zeros_like(s)
    if order == 2:
        return -np.ones_like(s)
    if order == 3:
        return np.where(s <= 0.5, -2. * s, -(1.5 - s)).astype(dtype)
    if order == 4:
        return np.where(s <= 1., (-12. * s + 9. * s * s) / 6., -3. * (2. - s)**2 / 6.).astype(dtype)
    raise ValueError(order)


def stencil(order):
    """Stencil offsets in ``itertools.product`` order (``resamplers.py:84-85``)."""
    ishifts = np.arange(order) - (order - 1) // 2
    return np.array(list(product(ishifts, ishifts, ishifts)), dtype='i8')


def base_index(u, order):
    """``(jnp.round if order % 2 else jnp.floor)(positions).astype(int16)``."""
    return (np.round(u) if order % 2 else np.floor(u)).astype('i8')


def cell_index(u, order, shape):
    """Wrapped base cell of each particle (int64 (N, 3)); the bit-exact index the GPU must match."""
    return base_index(u, order) % np.asarray(shape, dtype='i8')


_NATIVE = None


def _native_ok():
    """True when the C restatement (``paint_c.c``) builds; the NumPy loops are the fallback."""
    global _NATIVE
    if _NATIVE is None:
        try:
            _native.load()
            _NATIVE = True
        except Exception:
            _NATIVE = False
    return _NATIVE


def paint_mesh(shape, u, weights, order, dtype=np.float32, accum=None, native=True):
    """``resamplers.paint`` (``resamplers.py:66-97``) onto a zero mesh of ``shape``.

    ``u``: (N, 3) positions in cell units (already normalised), ``weights``: (N,).
    float32: serial ``np.add.at`` in particle order for each offset (reference order).
    float64: same kernels in float64, accumulated with ``np.bincount``.
    ``accum='f64'`` with float32: the reference's float32 contributions ``w * ker``
    summed in float64 and rounded once to float32 (an order-independent sum).
    """
    if native and np.dtype(dtype) == np.float64 and _native_ok():
        return _native.paint(shape, u, weights, order, 'double')
    if native and np.dtype(dtype) == np.float32 and _native_ok():
        # the C restatement of the loops below (paint_c.c): same float32 arithmetic
        if accum == 'f64':
            return _native.paint(shape, u, weights, order, 'f64').astype(np.float32)
        return _native.paint(shape, u, weights, order, 'serial')
    if accum == 'f64' and np.dtype(dtype) == np.float32:
        shape = tuple(int(s) for s in shape)
        u = np.asarray(u, dtype=np.float32)
        w = np.asarray(weights, dtype=np.float32)
        nshape = np.asarray(shape, dtype='i8')
        id0 = base_index(u, order)
        acc = np.zeros(int(np.prod(shape)), dtype='f8')
        strides = np.array([shape[1] * shape[2], shape[2], 1], dtype='i8')
        for ishift in stencil(order):
            idx = id0 + ishift
            k = kernel(order, np.abs(idx.astype(np.float32) - u), np.float32)
            val = (w * ((k[:, 0] * k[:, 1]) * k[:, 2])).astype(np.float32)
            acc += np.bincount((idx % nshape) @ strides, weights=val.astype('f8'), minlength=acc.size)
        return acc.astype(np.float32).reshape(shape)
    dtype = np.dtype(dtype)
    shape = tuple(int(s) for s in shape)
    u = np.asarray(u, dtype=dtype)
    w = np.asarray(weights, dtype=dtype)
    nshape = np.asarray(shape, dtype='i8')
    id0 = base_index(u, order)
    mesh = np.zeros(shape, dtype=dtype)
    flat = mesh.reshape(-1)
    strides = np.array([shape[1] * shape[2], shape[2], 1], dtype='i8')
    for ishift in stencil(order):
        idx = id0 + ishift
        s = np.abs(idx.astype(dtype) - u)
        k = kernel(order, s, dtype)
        ker = (k[:, 0] * k[:, 1]) * k[:, 2]
        val = (w * ker).astype(dtype)
        lin = (idx % nshape) @ strides
        if dtype == np.float32:
            np.add.at(flat, lin, val)
        else:
            flat += np.bincount(lin, weights=val, minlength=flat.size)
    return mesh


def read_mesh(mesh, u, order, dtype=None):
    """``resamplers.read`` (``resamplers.py:100-125``): gather with the same stencil."""
    dtype = np.dtype(dtype or mesh.dtype)
    shape = mesh.shape
    u = np.asarray(u, dtype=dtype)
    nshape = np.asarray(shape, dtype='i8')
    id0 = base_index(u, order)
    out = np.zeros(u.shape[0], dtype=dtype)
    flat = mesh.reshape(-1).astype(dtype)
    strides = np.array([shape[1] * shape[2], shape[2], 1], dtype='i8')
    for ishift in stencil(order):
        idx = id0 + ishift
        s = np.abs(idx.astype(dtype) - u)
        k = kernel(order, s, dtype)
        ker = (k[:, 0] * k[:, 1]) * k[:, 2]
        out = (out + flat[(idx % nshape) @ strides] * ker).astype(dtype)
    return out


def normalize_positions(geom, positions):
    """``(positions + boxsize / 2. - boxcenter) / cellsize`` (``mesh.py:2684``) in the mesh dtype."""
    dt = geom.dtype
    p = np.asarray(positions, dtype=dt)
    half = (geom.boxsize / dt.type(2.)).astype(dt)
    return (((p + half).astype(dt) - geom.boxcenter).astype(dt) / geom.cellsize).astype(dt)


def interlacing_shifts(interlacing, dtype):
    interlacing = max(int(interlacing), 1)
    dt = np.dtype(dtype)
    return [(dt.type(i) / dt.type(interlacing)) for i in range(interlacing)]


def rfftn(x):
    import scipy.fft
    return scipy.fft.rfftn(x, workers=-1)


def irfftn(x, shape):
    import scipy.fft
    return scipy.fft.irfftn(x, s=shape, workers=-1)


def compensation_kernel(geom, order):
    """``resampler.compensate`` window on the Hermitian grid (``resamplers.py:16-26``).

    Returns ``(prod_d sinc(k_d / 2 pi))**(-order)`` with circular k, as a broadcastable array.
    """
    dt = geom.dtype
    t = dt.type
    kc = kcoords(geom, kind='circular')
    ker = None
    for kk in kc:
        x = (kk / t(2. * np.pi)).astype(dt)
        pix = (t(np.pi) * x).astype(dt)
        with np.errstate(invalid='ignore', divide='ignore'):
            sinc = np.where(x == 0, t(1.), np.sin(pix) / pix).astype(dt)
        ker = sinc if ker is None else (ker * sinc).astype(dt)
    # lax.integer_pow(ker, -order): binary exponentiation then reciprocal
    acc, x, y = None, ker, order
    while y > 0:
        if y & 1:
            acc = x if acc is None else (acc * x).astype(dt)
        y >>= 1
        if y > 0:
            x = (x * x).astype(dt)
    return (t(1.) / acc).astype(dt)


def interlacing_phase(geom, shift, interlacing):
    """``exp(i shift (kx + ky + kz)) / interlacing`` with circular k (``mesh.py:2740-2744``)."""
    dt = geom.dtype
    cdt = np.result_type(dt, np.complex64)
    kc = kcoords(geom, kind='circular')
    ksum = ((kc[0] + kc[1]).astype(dt) + kc[2]).astype(dt)
    theta = (dt.type(shift) * ksum).astype(dt)
    return (np.cos(theta) + 1j * np.sin(theta)).astype(cdt)


def hermitian_planes(value, nlast=None):
    """Hermitian-symmetrise the k_z = 0 and (even N) k_z = N/2 planes.

    numpy / pocketfft / ducc ``irfftn`` discard the imaginary part of the last-axis
    DC and Nyquist samples after the inverse transforms along the first two axes;
    projecting those planes on their Hermitian part first gives the same real mesh
    with any C2R implementation.
    """
    out = value.copy()
    n0, n1, nz = value.shape
    if nlast is None:
        nlast = 2 * (nz - 1)
    planes = [0]
    if nlast % 2 == 0 and nz > 1:  # an even last axis ends on its self-conjugate Nyquist plane
        planes.append(nz - 1)
    return _sym(out, planes)


def _sym(out, planes):
    n0, n1, _ = out.shape
    i0 = (-np.arange(n0)) % n0
    i1 = (-np.arange(n1)) % n1
    for p in planes:
        plane = out[:, :, p]
        mirror = np.conj(plane[i0][:, i1])
        out[:, :, p] = 0.5 * (plane + mirror)
    return out


def paint(geom, positions, weights=None, resampler='cic', interlacing=0, compensate=False,
          out='real', shifts_only=False, accum=None):
    """``ParticleField.paint`` → ``_paint`` (``mesh.py:2604-2754``).

    Returns a real mesh (out='real') or the Hermitian complex mesh (out='complex').
    ``accum='f64'`` (float32 geometry): each shifted mesh is the float32 contributions
    summed in float64 and rounded once, instead of the serial float32 scatter.
    """
    order = {'ngp': 1, 'cic': 2, 'tsc': 3, 'pcs': 4}[resampler] if isinstance(resampler, str) else int(resampler)
    dt = geom.dtype
    cdt = np.result_type(dt, np.complex64)
    positions = np.asarray(positions, dtype=dt)
    if weights is None:
        weights = np.ones(positions.shape[0], dtype=dt)
    weights = np.asarray(weights, dtype=dt)
    u = normalize_positions(geom, positions)
    shape = geom.rshape
    interlacing = max(int(interlacing), 1)
    if interlacing == 1:
        mesh = paint_mesh(shape, u, weights, order, dtype=dt, accum=accum)
        if compensate:
            c = (r2c(geom, mesh) * compensation_kernel(geom, order)).astype(cdt)
            if out == 'real':
                return c2r(geom, c)
            return c
        if out != 'real':
            return r2c(geom, mesh)
        return mesh
    acc = np.zeros(geom.cshape, dtype=cdt)
    for shift in interlacing_shifts(interlacing, dt):
        us = (u + dt.type(shift)).astype(dt)
        mesh = paint_mesh(shape, us, weights, order, dtype=dt, accum=accum)
        c = r2c(geom, mesh)
        ph = interlacing_phase(geom, shift, interlacing)
        acc = (acc + ((c * ph).astype(cdt) / dt.type(interlacing)).astype(cdt)).astype(cdt)
    if compensate:
        acc = (acc * compensation_kernel(geom, order)).astype(cdt)
    if out == 'real':
        return c2r(geom, acc)
    return acc
