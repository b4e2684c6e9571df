"""Generate ``ylm_table.cuh``: the real spherical harmonics as Cartesian polynomials.

Build-time step (sympy), run by hand when the table changes::

    python jax-power_b200/csrc/gen_ylm.py

The polynomials follow the derivation of jax-power's ``get_Ylm(ell, m, real=True)``
(``jaxpower/utils.py:300-332``): sympy's associated Legendre function (with the
Condon-Shortley phase) of cos(theta) times cos(m phi) / sin(|m| phi), rewritten in
(xhat, yhat, zhat), expanded, with amplitude
sqrt((2l+1)/4pi) sqrt((l-|m|)!/(l+|m|)!) sqrt(2) (-1)^m for m != 0.  The expanded
form matters where xhat = 0 (the observer cell, k = 0): only true constant terms
survive, e.g. Y_20(0) = 0 but Y_40(0) = 3/8 * sqrt(9/4pi).
"""
import os

import numpy as np
import sympy as sp

LMAX = 8


def ylm_monomials(ell, m):
    amp = np.sqrt((2 * ell + 1) / (4 * np.pi))
    if m != 0:
        fac = 1
        for n in range(ell - abs(m) + 1, ell + abs(m) + 1):
            fac *= n
        amp *= np.sqrt(1. / fac) * np.sqrt(2.) * (-1)**m
    x, y, z, r = sp.symbols('x y z r', real=True, positive=True)
    xh, yh, zh = sp.symbols('xhat yhat zhat', real=True, positive=True)
    phi, theta = sp.symbols('phi theta', real=True)
    defs = [(sp.sin(phi), y / sp.sqrt(x**2 + y**2)),
            (sp.cos(phi), x / sp.sqrt(x**2 + y**2)),
            (sp.cos(theta), z / sp.sqrt(x**2 + y**2 + z**2))]
    expr = sp.assoc_legendre(ell, abs(m), sp.cos(theta))
    eimphi = sp.sin(abs(m) * phi) if m < 0 else (sp.cos(m * phi) if m > 0 else 1)
    expr *= sp.expand_trig(eimphi)
    expr = sp.together(expr.subs(defs)).subs(x**2 + y**2 + z**2, r**2)
    expr = amp * expr.expand().subs([(x / r, xh), (y / r, yh), (z / r, zh)])
    poly = sp.Poly(sp.expand(expr), xh, yh, zh)
    return [(float(c), tuple(int(p) for p in mon)) for mon, c in zip(poly.monoms(), poly.coeffs())]


def power(var, p):
    if p == 0:
        return None
    return f'{var}{p}'


def main():
    lines = ['// Generated by gen_ylm.py: real Y_lm(xhat, yhat, zhat) for ell <= %d.' % LMAX,
             '// Expanded monomial form of jaxpower/utils.py:300-332 (sympy derivation).',
             '#pragma once', '', 'namespace pk {', '',
             'constexpr int YLM_LMAX = %d;' % LMAX, '',
             '__device__ __forceinline__ float ylm_eval(int ell, int m, float x, float y, float z) {',
             '  float x2 = x * x, y2 = y * y, z2 = z * z;',
             '  float x1 = x, y1 = y, z1 = z;',
             '  float x3 = x2 * x, y3 = y2 * y, z3 = z2 * z;',
             '  float x4 = x2 * x2, y4 = y2 * y2, z4 = z2 * z2;',
             '  float x5 = x4 * x, y5 = y4 * y, z5 = z4 * z;',
             '  float x6 = x4 * x2, y6 = y4 * y2, z6 = z4 * z2;',
             '  float x7 = x6 * x, y7 = y6 * y, z7 = z6 * z;',
             '  float x8 = x4 * x4, y8 = y4 * y4, z8 = z4 * z4;',
             '  (void)x1; (void)y1; (void)z1; (void)x3; (void)y3; (void)z3; (void)x5; (void)y5; (void)z5;',
             '  (void)x6; (void)y6; (void)z6; (void)x7; (void)y7; (void)z7; (void)x8; (void)y8; (void)z8;',
             '  (void)x4; (void)y4; (void)z4; (void)x2; (void)y2; (void)z2;',
             '  switch (ell * 32 + (m + 16)) {']
    for ell in range(LMAX + 1):
        for m in range(-ell, ell + 1):
            terms = []
            for c, (px, py, pz) in ylm_monomials(ell, m):
                factors = [f for f in (power('x', px), power('y', py), power('z', pz)) if f]
                coef = repr(float(c)) + 'f'
                terms.append(' * '.join([coef] + factors))
            body = ' + '.join(terms) if terms else '0.f'
            lines.append(f'    case {ell * 32 + m + 16}: return {body};')
    lines += ['    default: return 0.f;', '  }', '}', '', '}  // namespace pk', '']
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'ylm_table.cuh')
    with open(path, 'w') as f:
        f.write('\n'.join(lines))
    print('wrote', path)


if __name__ == '__main__':
    main()
