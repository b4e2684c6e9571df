"""Host-side pieces of the window functions, on the CPU: the tophat Bessel integrals, the real
Gaunt and Legendre-product coefficients, and the parsing of theory and input-edge arguments."""
import numpy as np
import pytest


def test_bessel_primitive_and_shell():
    from scipy.integrate import quad
    from scipy.special import sici, spherical_jn
    from jaxpower_b200.mesh2 import _bessel_primitive, _bessel_shell
    x = np.array([0., 1e-3, 0.7, 3.1, 42.2, 350.5])
    assert np.allclose(_bessel_primitive(0, x), np.sin(x) - x * np.cos(x), rtol=1e-11, atol=1e-13)
    assert np.allclose(_bessel_primitive(2, x), x * np.cos(x) - 4. * np.sin(x) + 3. * sici(x)[0], rtol=1e-11,
                       atol=1e-13)
    ref4 = [quad(lambda t: t * t * spherical_jn(4, t), 0., xi, limit=1000)[0] for xi in x]
    assert np.allclose(_bessel_primitive(4, x), ref4, rtol=1e-9, atol=1e-12)
    s = np.array([0., 5., 80.])
    lo, hi = 0.02, 0.05
    got = _bessel_shell(0, lo, hi, s)
    assert np.isclose(got[0], 4. * np.pi * (hi ** 3 - lo ** 3) / 3.)
    ref = [4. * np.pi * quad(lambda k: k * k * spherical_jn(0, k * si), lo, hi)[0] for si in s[1:]]
    assert np.allclose(got[1:], ref, rtol=1e-10)
    assert _bessel_shell(2, lo, hi, np.zeros(1))[0] == 0.


def test_real_gaunt_matches_oracle_quadrature():
    from jaxpower_b200.mesh2 import _real_gaunt
    from oracle.spectrum import real_gaunt
    for p in (0, 2, 4):
        for mp in range(-p, p + 1):
            for m1 in range(-2, 3):
                for m2 in range(-2, 3):
                    a, b = _real_gaunt((p, mp), (2, m1), (2, m2)), real_gaunt((p, mp), (2, m1), (2, m2))
                    assert abs(a - b) < 1e-10, ((p, mp), m1, m2, a, b)
    assert abs(_real_gaunt((2, 0), (2, 0), (2, 0)) - 0.18022375157286857) < 1e-12


def test_window_coeffs_match_wigner_3j():
    from sympy.physics.wigner import wigner_3j
    from jaxpower_b200.mesh2 import _window_coeffs
    for ell in (0, 1, 2, 4):
        for ellin in (0, 2, 3, 4):
            got = dict(_window_coeffs(ell, ellin))
            for q in range(abs(ell - ellin), ell + ellin + 1):
                ref = (2 * ell + 1) * float(wigner_3j(ell, ellin, q, 0, 0, 0)) ** 2
                assert abs(got.get(q, 0.) - ref) < 1e-12, (ell, ellin, q)


def test_theory_and_edges_parsing():
    import jaxpower_b200 as jp
    from jaxpower_b200.mesh2 import _theory_poles, _window_edges
    f = lambda k: k
    assert _theory_poles({0: f}) == (None, {0: f}, 'firstpoint')
    kin, poles, los = _theory_poles(({0: f}, 'local'))
    assert los == 'local' and poles == {0: f}
    kin, poles, los = _theory_poles((np.arange(3.), [np.ones(2), np.zeros(2)], 'firstpoint'))
    assert np.array_equal(kin, np.arange(3.)) and set(poles) == {0, 2}
    with pytest.raises(NotImplementedError):
        _theory_poles(({0: f}, 'other'))
    edges, ells = _window_edges(np.arange(0., 0.1, 0.02), 2)
    assert edges.shape == (4, 2) and ells == [2]
    k_edges = np.column_stack([np.arange(0., 0.08, 0.02), np.arange(0.02, 0.1, 0.02)])
    poles = jp.Mesh2SpectrumPoles([jp.Mesh2SpectrumPole(k=k_edges.mean(-1), k_edges=k_edges, nmodes=np.ones(4),
                                                        num_raw=np.zeros(4), ell=ell) for ell in (0, 2)])
    edges, ells = _window_edges(poles, None)
    assert np.array_equal(edges, k_edges) and ells == [0, 2]


def test_wide_angle_edges_parsing():
    """Input multipoles given as (ell, wide-angle order) pairs (``mesh2.py:826-836``): pairs
    anywhere turn every input into a pair, a container's ``wa_order`` labels are read back, and
    the fixed-line-of-sight and 'local' paths refuse orders > 0."""
    import jaxpower_b200 as jp
    from jaxpower_b200.mesh2 import _no_wide_angle, _plain_ells, _wide_angle_terms, _window_edges
    edges = np.arange(0., 0.1, 0.02)
    _, ells = _window_edges(edges, [(0, 0), 2, (2, 1)])
    assert ells == [(0, 0), (2, 0), (2, 1)]
    _, ells = _window_edges(edges, (0, 2))
    assert ells == [0, 2]
    assert _wide_angle_terms([0, (2, 1)]) == [(0, 0), (2, 1)]
    assert _plain_ells([(0, 0), 2]) == [0, 2]
    with pytest.raises(ValueError):
        _plain_ells([(0, 0), (2, 1)])
    _no_wide_angle([(0, 0), 2])
    with pytest.raises(NotImplementedError):
        _no_wide_angle([(1, 1)])
    k_edges = np.column_stack([edges[:-1], edges[1:]])
    poles = jp.Mesh2SpectrumPoles([jp.Mesh2SpectrumPole(k=k_edges.mean(-1), k_edges=k_edges, nmodes=np.ones(4),
                                                        num_raw=np.zeros(4), ell=ell, attrs={'wa_order': wa})
                                   for ell, wa in ((0, 0), (2, 0), (1, 1))])
    assert poles.wa_orders == (0, 0, 1)
    got, ells = _window_edges(poles, None)
    assert np.array_equal(got, k_edges) and ells == [(0, 0), (2, 0), (1, 1)]
    assert poles.get(ells=1, wa_orders=1).ell == 1
