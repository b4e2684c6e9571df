"""Mesh attributes on the CPU (no particles, so no device): ``MeshAttrs`` (``mesh.py:1455-1719``),
``next_fft_size`` (``mesh.py:2227-2262``) and ``get_mesh_attrs`` (``mesh.py:2271-2381``), with
the cases of the reference's ``tests/test_mesh.py:24-35`` that take no positions."""
import itertools
import math

import numpy as np
import pytest


def _smooth(m, primes):
    for p in primes:
        while m % p == 0:
            m //= p
    return m == 1


def test_next_fft_size_brute_force():
    from jaxpower_b200 import next_fft_size
    for primes, divisors in itertools.product([(2, 3, 5, 7), (2, 3, 5), (2,), ()], [(), (2,), (2, 3), (4, 6)]):
        D = 1
        for d in divisors:
            D = D * d // math.gcd(D, d)
        if primes and not _smooth(D, primes):
            continue  # no such size exists (the search, as the reference's, would not end)
        for n in range(1, 200):
            m = next_fft_size(n, primes=primes, divisors=divisors)
            expected = next(x for x in range(n, 10 * n + 100)
                            if x % D == 0 and (not primes or _smooth(x, primes)))
            assert m == expected, (n, primes, divisors, m, expected)
    assert next_fft_size(97) == 98 and next_fft_size(101, primes=(2,)) == 128
    assert next_fft_size(17, primes=(2, 3, 5), divisors=(2, 3)) == 18
    # a prime or divisor of 1 (or less) is ignored
    assert next_fft_size(7, primes=(1, 2), divisors=(1,)) == 8


def test_get_mesh_attrs_without_positions():
    from jaxpower_b200 import get_mesh_attrs
    attrs = get_mesh_attrs(boxsize=1000., boxcenter=0., cellsize=10.)
    assert np.array_equal(attrs.meshsize, [100] * 3) and np.allclose(attrs.cellsize, 10.)
    attrs = get_mesh_attrs(boxsize=1000., boxcenter=0., meshsize=128)
    assert np.array_equal(attrs.meshsize, [128] * 3) and np.allclose(attrs.cellsize, 1000. / 128)
    attrs = get_mesh_attrs(boxcenter=(1., 2., 3.), meshsize=(64, 32, 16), cellsize=(2., 4., 8.))
    assert np.array_equal(attrs.boxsize, [128.] * 3) and np.array_equal(attrs.boxcenter, [1., 2., 3.])
    with pytest.raises(ValueError):
        get_mesh_attrs(boxsize=100., boxcenter=0., meshsize=10, cellsize=10.)
    with pytest.raises(ValueError):  # 1000 / 12 cells: the box would change
        get_mesh_attrs(boxsize=1000., boxcenter=0., cellsize=12.)
    attrs = get_mesh_attrs(boxsize=1000., boxcenter=0., cellsize=12., approximate=True)
    assert np.array_equal(attrs.meshsize, [84] * 3) and np.allclose(attrs.boxsize, 1008.)
    attrs = get_mesh_attrs(boxsize=1000., boxcenter=0., cellsize=12., approximate=True, primes=(2, 3, 5),
                           divisors=(2, 3))
    assert np.array_equal(attrs.meshsize, [90] * 3) and np.allclose(attrs.cellsize, 12.)
    with pytest.raises(ValueError):
        get_mesh_attrs(boxcenter=0., cellsize=10.)  # no boxsize and no positions
    with pytest.raises(ValueError):
        get_mesh_attrs(boxsize=100., boxcenter=0.)  # neither meshsize nor cellsize


def test_mesh_attrs_fields():
    from jaxpower_b200 import MeshAttrs
    attrs = MeshAttrs(meshsize=(64, 48, 32), boxsize=(100., 120., 90.), boxcenter=(3., -5., 10.))
    assert attrs.cellsize.dtype == np.float32 and attrs.kfun.dtype == np.float32
    assert np.array_equal(attrs.cellsize, (attrs.boxsize / attrs.meshsize.astype('f4')).astype('f4'))
    assert np.array_equal(attrs.kfun, (np.float32(2. * np.pi) / attrs.boxsize).astype('f4'))
    assert attrs.fft_backend == 'jax' and dict(**attrs)['meshsize'] is attrs.meshsize
    assert attrs.clone() == attrs and attrs.clone(boxcenter=0.) != attrs
    assert np.array_equal(MeshAttrs(meshsize=16).boxsize, [16.] * 3)
    assert MeshAttrs(meshsize=16, fft_backend='jaxdecomp').fft_backend == 'jaxdecomp'
    with pytest.raises(NotImplementedError):
        MeshAttrs(meshsize=16, dtype='f8')
    with pytest.raises(ValueError):
        MeshAttrs(meshsize=16, fft_backend='other')
