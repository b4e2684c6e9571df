"""The oracle's spherical Bessel functions against the reference's closed forms.

``get_spherical_jn`` (utils.py:443-450) switches from a closed form (x > 0.1,
utils.py:419-428) to a truncated Taylor series (x <= 0.1).  The closed forms for ell <= 4
are the textbook Rayleigh expressions, written out here; the oracle evaluates them with
scipy and the series itself.
"""
import numpy as np

from oracle.spectrum import spherical_jn


def _closed(ell, x):
    s, c = np.sin(x), np.cos(x)
    if ell == 0:
        return s / x
    if ell == 1:
        return -c / x + s / x**2
    if ell == 2:
        return (-1. / x + 3. / x**3) * s - 3. * c / x**2
    if ell == 3:
        return (-6. / x**2 + 15. / x**4) * s + (1. / x - 15. / x**3) * c
    return (10. / x**2 - 105. / x**4) * c + (1. / x - 45. / x**3 + 105. / x**5) * s


def test_spherical_jn_closed_forms_and_series():
    x = np.concatenate([np.linspace(0.1001, 3., 200), np.linspace(3., 1500., 500)])
    for ell in range(5):
        ref = _closed(ell, x)
        got = spherical_jn(ell, x)
        # the closed forms cancel for x < ell in float64: compare on their own precision
        tol = 1e-12 * (1. + (2. * ell / x)**ell) * np.max(np.abs(ref))
        assert np.all(np.abs(got - ref) <= tol + 1e-13), ell
        # the series branch (x <= 0.1) agrees with the function there
        from scipy import special
        xs = np.array([1e-3, 0.03, 0.1])
        assert np.allclose(spherical_jn(ell, xs), special.spherical_jn(ell, xs), rtol=1e-12, atol=0.), ell
    assert spherical_jn(0, np.array([0.]))[0] == 1.
    assert all(spherical_jn(ell, np.array([0.]))[0] == 0. for ell in range(1, 5))
