"""Mesh geometry and coordinate grids (oracle; test infrastructure only).

Restates ``mesh.py:360-403`` (``fftfreq``) and ``mesh.py:1559-1636``
(``MeshAttrs.cellsize/kfun/knyq/rcoords/kcoords``) of jax-power, with the
float32 rounding of ``jax.numpy.fft.fftfreq``: ``k / (d * n)`` evaluated in the
target dtype, then ``* spacing * n``.
"""
import numpy as np


class Geometry:
    """Mesh attributes in a fixed real dtype (float32 = JAX default, x64 off).

    Mirrors ``MeshAttrs`` (``mesh.py:1455-1491``): boxsize / boxcenter are
    stored in the real dtype, meshsize as int32.
    """

    def __init__(self, meshsize, boxsize=None, boxcenter=0., dtype=np.float32, backend='jax'):
        # backend 'jax': Hermitian (N, N, N//2 + 1) complex layout (rfftn);
        # backend 'jaxdecomp': full complex layout (fftn), as ``mesh.py:1679-1719`` with jaxdecomp
        self.backend = backend
        self.dtype = np.dtype(dtype)
        self.meshsize = np.broadcast_to(np.asarray(meshsize, dtype='i4'), (3,)).copy()
        if boxsize is None:
            boxsize = 1. * self.meshsize
        self.boxsize = np.broadcast_to(np.asarray(boxsize, dtype=self.dtype), (3,)).copy()
        self.boxcenter = np.broadcast_to(np.asarray(boxcenter, dtype=self.dtype), (3,)).copy()

    @property
    def cellsize(self):
        # mesh.py:1575  boxsize / meshsize (int32 promoted to the real dtype)
        return (self.boxsize / self.meshsize.astype(self.dtype)).astype(self.dtype)

    @property
    def kfun(self):
        # mesh.py:1580  2 pi / boxsize: python float (weak) / real array
        return (self.dtype.type(2. * np.pi) / self.boxsize).astype(self.dtype)

    @property
    def knyq(self):
        return (np.pi * self.meshsize / self.boxsize.astype('f8')).astype(self.dtype)

    @property
    def hermitian(self):
        return self.backend == 'jax'

    @property
    def cshape(self):
        n = self.meshsize
        if not self.hermitian:
            return self.rshape
        return (int(n[0]), int(n[1]), int(n[2]) // 2 + 1)

    @property
    def rshape(self):
        return tuple(int(n) for n in self.meshsize)


def fftfreq(n, dtype, hermitian=False):
    """``jnp.fft.fftfreq(n)`` / ``rfftfreq(n)`` in ``dtype``: signed index / n."""
    dtype = np.dtype(dtype)
    if hermitian:
        k = np.arange(0, n // 2 + 1, dtype=dtype)
    else:
        idx = np.arange(n)
        k = np.where(idx < (n + 1) // 2, idx, idx - n).astype(dtype)
    return (k / dtype.type(n)).astype(dtype)


def kcoords(geom, kind='wavenumber', sparse=True):
    """``MeshAttrs.kcoords`` (``mesh.py:1605-1636``) for the Hermitian layout.

    kind='wavenumber': fftfreq * kfun * n; kind='circular': fftfreq * (2 pi / n) * n,
    in [-pi, pi).  Returns three broadcastable arrays (sparse meshgrid).
    """
    dt = geom.dtype
    out = []
    for axis in range(3):
        n = int(geom.meshsize[axis])
        if kind == 'wavenumber':
            spacing = geom.kfun[axis]
        elif kind == 'circular':
            spacing = dt.type(2. * np.pi / n)  # float64 quotient rounded to dtype
        elif kind == 'index':
            spacing = dt.type(1.)
        else:
            raise ValueError(kind)
        f = fftfreq(n, dt, hermitian=(axis == 2 and geom.hermitian))
        k = ((f * spacing).astype(dt) * dt.type(n)).astype(dt)
        shape = [1, 1, 1]
        shape[axis] = k.size
        out.append(k.reshape(shape))
    return tuple(out)


def rcoords(geom, sparse=True):
    """``MeshAttrs.rcoords(kind='position')`` (``mesh.py:1594-1603``): cell corners.

    x_i = i * cellsize + (boxcenter - boxsize / 2), in the real dtype.
    """
    dt = geom.dtype
    offset = (geom.boxcenter - (geom.boxsize / dt.type(2.)).astype(dt)).astype(dt)
    out = []
    for axis in range(3):
        n = int(geom.meshsize[axis])
        x = (np.arange(n, dtype=dt) * geom.cellsize[axis]).astype(dt)
        x = (x + offset[axis]).astype(dt)
        shape = [1, 1, 1]
        shape[axis] = n
        out.append(x.reshape(shape))
    return tuple(out)


def hermitian_weights(geom):
    """``_get_hermitian_weights`` (``mesh.py:2814-2828``): 1 + (k_z > 0); 1 for a full complex grid."""
    w = np.ones(geom.cshape, dtype='i4')
    if geom.hermitian:
        w += (kcoords(geom)[2] > 0)
    return w


def r2c(geom, x):
    """``MeshAttrs.r2c`` (``mesh.py:1679-1697``): rfftn, or full fftn for the jaxdecomp layout."""
    import scipy.fft
    cdt = np.result_type(geom.dtype, np.complex64)
    if geom.hermitian:
        return scipy.fft.rfftn(x, workers=-1).astype(cdt)
    return scipy.fft.fftn(x, workers=-1).astype(cdt)


def c2r(geom, x):
    """``MeshAttrs.c2r`` (``mesh.py:1699-1719``): irfftn, or real part of ifftn (jaxdecomp)."""
    import scipy.fft
    if geom.hermitian:
        return scipy.fft.irfftn(x, s=geom.rshape, workers=-1).astype(geom.dtype)
    return scipy.fft.ifftn(x, workers=-1).real.astype(geom.dtype)
