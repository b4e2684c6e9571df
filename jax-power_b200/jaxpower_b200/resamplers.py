"""Resampler namespaces ``ngp``, ``cic``, ``tsc``, ``pcs`` (``resamplers.py:128-143``).

Each namespace has ``order``, ``compensate`` (the ``kind='circular'`` window of
``resamplers.py:16-26``, applied on the GPU by the fused compensation pass when
given to ``ComplexMeshField.apply``), ``aliasing_shotnoise`` (``resamplers.py:29-53``),
``paint`` and ``read``.  ``paint`` / ``read`` here take torch tensors in cell
units on a zero mesh / a mesh, like the reference's functional forms.
"""
import math

import torch

__all__ = ['ngp', 'cic', 'tsc', 'pcs', 'get_resampler']


def _compensate_tophat_convolution_kernel(order):

    def fn(value, kvec):
        kernel = 1.
        for kk in kvec:
            kernel = kernel * torch.sinc(kk / (2 * math.pi))
        return value * kernel**(-order)

    fn.kind = 'circular'
    fn.compensate_order = order
    return fn


def _aliasing_shotnoise_kernel(order):

    def k1(angle):
        return torch.ones_like(angle)

    def k2(angle):
        return 1. - 2. / 3. * torch.sin(angle / 2.)**2

    def k3(angle):
        s2 = torch.sin(angle / 2.)**2
        return 1. - s2 + 2. / 15. * s2**2

    def k4(angle):
        s2 = torch.sin(angle / 2.)**2
        return 1. - 4. / 3. * s2 + 2. / 5. * s2 * s2 - 4. / 315. * s2**3

    kernels = [None, k1, k2, k3, k4]

    def fn(value, kvec):
        kernel = 1.
        for kk in kvec:
            kernel = kernel * kernels[order](kk)
        return value * kernel

    fn.kind = 'circular'
    return fn


def _make(name, order):

    def paint(mesh, positions, weights=None):
        """Paint positions given in cell units (mesh origin at 0) onto ``mesh`` (a tensor or a shape)."""
        from .mesh import MeshAttrs, _paint_shifts, _as_positions, _as_weights
        shape = tuple(mesh) if isinstance(mesh, tuple) else tuple(mesh.shape)
        attrs = MeshAttrs(meshsize=shape, boxsize=shape, boxcenter=[s / 2. for s in shape])
        positions = _as_positions(positions)
        out = _paint_shifts(attrs, positions, _as_weights(weights, positions.shape[0]), order, 1)[0][0]
        if not isinstance(mesh, tuple):
            out = out + mesh
        return out

    def read(mesh, positions):
        from .mesh import MeshAttrs, RealMeshField
        shape = tuple(mesh.shape)
        attrs = MeshAttrs(meshsize=shape, boxsize=shape, boxcenter=[s / 2. for s in shape])
        return RealMeshField(mesh, attrs=attrs).read(positions, resampler=name)

    ns = type(name, (), dict(order=order, paint=staticmethod(paint), read=staticmethod(read),
                             compensate=staticmethod(_compensate_tophat_convolution_kernel(order)),
                             aliasing_shotnoise=staticmethod(_aliasing_shotnoise_kernel(order))))
    return ns


ngp = _make('ngp', 1)
cic = _make('cic', 2)
tsc = _make('tsc', 3)
pcs = _make('pcs', 4)


def get_resampler(resampler):
    if isinstance(resampler, str):
        try:
            return {'ngp': ngp, 'cic': cic, 'tsc': tsc, 'pcs': pcs}[resampler]
        except KeyError:
            raise ValueError('unknown resampler {}'.format(resampler))
    return resampler
