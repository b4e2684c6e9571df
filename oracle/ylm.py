"""Real spherical harmonics and Legendre polynomials (oracle; test only).

Restates ``utils.py:190-334`` (``get_Ylm(ell, m, real=True)``): the sympy
derivation — associated Legendre ``P_l^|m|(cos theta)`` (Condon-Shortley phase
included by sympy) times ``cos(m phi)`` (m > 0) or ``sin(|m| phi)`` (m < 0),
rewritten in Cartesian unit vectors, expanded, and scaled by

    amp = sqrt((2l+1)/(4 pi)) * sqrt((l-|m|)!/(l+|m|)!) * sqrt(2) * (-1)^m   (m != 0)

— and ``utils.py:341-360`` (Legendre polynomials up to l = 10).  Evaluation
divides by |x| with 0 where |x| = 0 (``utils.py:252-261``).
"""
from functools import lru_cache

import numpy as np


@lru_cache(maxsize=64)
def ylm_expr(ell, m):
    """sympy expression of the real Y_lm in (xhat, yhat, zhat), as the reference derives it."""
    import sympy as sp
    amp = np.sqrt((2 * ell + 1) / (4 * np.pi))
    if m != 0:
        fac = 1
        for n in range(ell - abs(m) + 1, ell + abs(m) + 1):
            fac *= n
        amp *= np.sqrt(1. / fac)
        amp *= np.sqrt(2.) * (-1)**m
    x, y, z, r = sp.symbols('x y z r', real=True, positive=True)
    xhat, yhat, zhat = sp.symbols('xhat yhat zhat', real=True, positive=True)
    phi, theta = sp.symbols('phi theta', real=True)
    defs = [(sp.sin(phi), y / sp.sqrt(x**2 + y**2)),
            (sp.cos(phi), x / sp.sqrt(x**2 + y**2)),
            (sp.cos(theta), z / sp.sqrt(x**2 + y**2 + z**2))]
    expr = sp.assoc_legendre(ell, abs(m), sp.cos(theta))
    if m < 0:
        eimphi = sp.sin(abs(m) * phi)
    elif m > 0:
        eimphi = sp.cos(m * phi)
    else:
        eimphi = 1
    expr *= sp.expand_trig(eimphi)
    expr = sp.together(expr.subs(defs)).subs(x**2 + y**2 + z**2, r**2)
    expr = amp * expr.expand().subs([(x / r, xhat), (y / r, yhat), (z / r, zhat)])
    return expr, (xhat, yhat, zhat)


def ylm_monomials(ell, m):
    """The expression as a list of (coefficient, (px, py, pz)) monomials in (xhat, yhat, zhat)."""
    import sympy as sp
    expr, syms = ylm_expr(ell, m)
    poly = sp.Poly(sp.expand(expr), *syms)
    return [(float(c), tuple(int(p) for p in mon)) for mon, c in zip(poly.monoms(), poly.coeffs())]


@lru_cache(maxsize=64)
def get_ylm(ell, m):
    """Callable Y(x, y, z) on unnormalised vectors (numpy), as ``get_Ylm(ell, m, real=True)``."""
    import sympy as sp
    expr, syms = ylm_expr(ell, m)
    func = sp.lambdify(syms, expr, modules=['numpy'])

    def ylm(x, y, z):
        dt = np.result_type(x, y, z)
        xnorm = np.sqrt((x * x + y * y) + z * z).astype(dt)
        with np.errstate(divide='ignore', invalid='ignore'):
            xh = np.where(xnorm == 0, dt.type(0.), x / xnorm).astype(dt)
            yh = np.where(xnorm == 0, dt.type(0.), y / xnorm).astype(dt)
            zh = np.where(xnorm == 0, dt.type(0.), z / xnorm).astype(dt)
        out = np.asarray(func(xh, yh, zh))
        return np.broadcast_to(out, np.broadcast_shapes(xh.shape, yh.shape, zh.shape)).astype(dt)

    return ylm


def ylm_scipy(ell, m, x, y, z):
    """Independent evaluation through ``scipy.special.sph_harm_y`` (the reference's scipy fallback)."""
    from scipy import special
    r = np.sqrt(x * x + y * y + z * z)
    theta = np.arccos(np.clip(z / r, -1, 1))
    phi = np.arctan2(y, x)
    if m == 0:
        return special.sph_harm_y(ell, 0, theta, phi).real
    c = special.sph_harm_y(ell, abs(m), theta, phi)
    # real form: sqrt(2) (-1)^m Re/Im Y_l^|m| (scipy includes Condon-Shortley)
    if m > 0:
        return np.sqrt(2.) * (-1)**m * c.real
    return np.sqrt(2.) * (-1)**m * c.imag


_LEGENDRE = {
    0: lambda x: np.ones_like(x),
    1: lambda x: x,
    2: lambda x: 3 * x**2 / 2 - 1 / 2,
    3: lambda x: 5 * x**3 / 2 - 3 * x / 2,
    4: lambda x: 35 * x**4 / 8 - 15 * x**2 / 4 + 3 / 8,
    5: lambda x: 63 * x**5 / 8 - 35 * x**3 / 4 + 15 * x / 8,
    6: lambda x: 231 * x**6 / 16 - 315 * x**4 / 16 + 105 * x**2 / 16 - 5 / 16,
    7: lambda x: 429 * x**7 / 16 - 693 * x**5 / 16 + 315 * x**3 / 16 - 35 * x / 16,
    8: lambda x: 6435 * x**8 / 128 - 3003 * x**6 / 32 + 3465 * x**4 / 64 - 315 * x**2 / 32 + 35 / 128,
}


def legendre(ell, x):
    """``get_legendre(ell)`` (``utils.py:341-360``)."""
    return _LEGENDRE[ell](x).astype(np.asarray(x).dtype)
