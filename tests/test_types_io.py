"""Observable I/O: write / read round trips of the multipole containers (CPU)."""
import numpy as np

from jaxpower_b200.types import (Mesh2SpectrumPole, Mesh2SpectrumPoles, Mesh2CorrelationPole,
                                 Mesh2CorrelationPoles, read, write)


def _poles(cls_pole, cls_poles, rng):
    edges = np.linspace(0., 0.2, 11)
    poles = []
    for ell in (0, 2, 4):
        num = rng.normal(size=10) + (1j * rng.normal(size=10) if ell == 2 else 0.)
        poles.append(cls_pole(0.5 * (edges[:-1] + edges[1:]), np.column_stack([edges[:-1], edges[1:]]),
                              rng.integers(1, 100, 10), num, num_shotnoise=(3. if ell == 0 else 0.),
                              norm=2.5, volume=1e9, ell=ell, attrs={'los': 'firstpoint', 'meshsize': [64, 64, 64]}))
    return cls_poles(poles)


def _same(a, b):
    assert type(a) is type(b)
    assert a.ells == b.ells
    for p, q in zip(a, b):
        for name in p._fields:
            x, y = getattr(p, name), getattr(q, name)
            if x is None:
                assert y is None
            else:
                assert np.array_equal(np.asarray(x), np.asarray(y)), name
        assert p.ell == q.ell and p.attrs == q.attrs
        assert np.array_equal(p.value(), q.value())


def test_write_read_spectrum_poles(tmp_path):
    poles = _poles(Mesh2SpectrumPole, Mesh2SpectrumPoles, np.random.default_rng(0))
    fn = str(tmp_path / 'poles.npz')
    poles.write(fn)
    _same(poles, read(fn))
    single = poles.get(2)
    write(str(tmp_path / 'pole.npz'), single)
    back = read(str(tmp_path / 'pole.npz'))
    assert isinstance(back, Mesh2SpectrumPole) and back.ell == 2
    assert np.array_equal(back.num_raw, single.num_raw)


def test_write_read_correlation_poles(tmp_path):
    poles = _poles(Mesh2CorrelationPole, Mesh2CorrelationPoles, np.random.default_rng(1))
    fn = str(tmp_path / 'xi.npz')
    write(fn, poles)
    back = read(fn)
    _same(poles, back)
    assert np.array_equal(back.get(0).s, poles.get(0).s)


def test_package_read_is_the_observable_reader():
    import jaxpower_b200 as jp
    from jaxpower_b200 import types
    assert jp.read is types.read and jp.write is types.write


def test_deferred_rows_read_once_and_match(tmp_path):
    """Per-bin sums left on the device are read back on first use, once for all poles, and
    give the values the eager construction gives."""
    import torch
    from jaxpower_b200.types import DeferredRows
    rng = np.random.default_rng(3)
    raw = rng.normal(size=(3, 10))
    nmodes = rng.integers(1, 50, 10).astype('f8')
    factors = [1., 5., 9.]
    edges = np.column_stack([np.arange(10.), np.arange(1., 11.)])
    rows = DeferredRows(torch.as_tensor(raw), nmodes, factors)
    lazy = Mesh2SpectrumPoles([Mesh2SpectrumPole(np.arange(10.), edges, nmodes, rows.row(i), num_shotnoise=np.zeros(10),
                                                 norm=np.full(10, 2.), ell=ell) for i, ell in enumerate((0, 2, 4))])
    eager = Mesh2SpectrumPoles([Mesh2SpectrumPole(np.arange(10.), edges, nmodes, raw[i] / nmodes * factors[i],
                                                  num_shotnoise=np.zeros(10), norm=np.full(10, 2.), ell=ell)
                                for i, ell in enumerate((0, 2, 4))])
    assert rows._host is None  # nothing read yet
    assert np.array_equal(lazy.get(2).num_raw, eager.get(2).num_raw)
    assert rows._sums is None and rows._host is not None  # one read-back, tensor released
    assert np.array_equal(lazy.value(), eager.value())
    fn = str(tmp_path / 'lazy.npz')
    lazy.write(fn)
    _same(eager, read(fn))


def test_wide_angle_labels_round_trip(tmp_path):
    """Theory multipoles labelled with wide-angle orders (attrs['wa_order']): wa_orders, get by
    (ell, order), and the labels survive write / read."""
    edges = np.linspace(0., 0.1, 6)
    k = 0.5 * (edges[:-1] + edges[1:])
    pairs = [(0, 0), (2, 0), (0, 1), (2, 1)]
    poles = Mesh2SpectrumPoles([Mesh2SpectrumPole(k, np.column_stack([edges[:-1], edges[1:]]), np.ones(5),
                                                  np.full(5, 10. * ell + wa), ell=ell,
                                                  attrs=dict(wa_order=wa) if wa else None) for ell, wa in pairs])
    assert poles.ells == (0, 2, 0, 2) and poles.wa_orders == (0, 0, 1, 1)
    assert poles.get(0).num_raw[0] == 0. and poles.get(0, wa_orders=1).num_raw[0] == 1.
    sub = poles.get([2, 2], wa_orders=[1, 0])
    assert [p.num_raw[0] for p in sub] == [21., 20.]
    fn = str(tmp_path / 'wa.npz')
    poles.write(fn)
    back = read(fn)
    assert back.wa_orders == (0, 0, 1, 1)
    _same(poles, back)


def test_window_input_multipoles_parsing():
    """Input multipoles of a window matrix: ints stay ints, (ell, order) pairs become pairs, and a
    fixed line of sight rejects orders > 0."""
    import pytest
    from jaxpower_b200.mesh2 import _window_edges, _plain_ells, _no_wide_angle
    e, ells = _window_edges(np.array([0., 0.1, 0.2]), (0, 2))
    assert e.shape == (2, 2) and ells == [0, 2]
    _, ells = _window_edges(np.array([0., 0.1]), [(0, 0), 2, (4, 1)])
    assert ells == [(0, 0), (2, 0), (4, 1)]
    assert _plain_ells([(0, 0), 2]) == [0, 2]
    with pytest.raises(ValueError):
        _plain_ells([(0, 1)])
    with pytest.raises(NotImplementedError):
        _no_wide_angle([(2, 2)])
