#!/usr/bin/env python3
"""Generate fj_special_coeffs.h: the polynomial coefficients of the FP32 and
FP64 special functions used by the F-J kernels.

Every coefficient set is a least-squares fit on Chebyshev nodes (a near-minimax
fit) to values computed with mpmath at 40 significant digits from the
defining functions:

  J0, J1, Y0, Y1                Bessel functions (A&S 9.1)
  BJ(x) = int_0^x J0(t) dt      = x J0 + (pi x/2)(J1 H0 - J0 H1)   (A&S 11.1.7)
  BY(x) = int_0^x Y0(t) dt      = x Y0 + (pi x/2)(Y1 H0 - Y0 H1)   (A&S 11.1.8)
  H0, H1                        Struve functions (A&S 12.1)

Ranges (the same split for both precisions):
  S0  0 <= x < 2   w = (x/2)^2;   J0 = A(w), J1 = x B(w), BJ = x C(w),
                   Y0 = L J0 + D(w), Y1 = L J1 - 2/(pi x) + x E(w),
                   BY = L BJ + x F(w),  L = (2/pi) ln(x/2)
                   (A..F are entire in w: A&S 9.1.10-9.1.13 and the
                   integral of those series)
  S1  2 <= x < 5   u = (x - 3.5)/1.5, each function a polynomial in u
  S2  5 <= x < 8   u = (x - 6.5)/1.5
  L   x >= 8       Hankel form with chi = x - pi/4, M = sqrt(2/(pi x)):
                   J0 = M (P0 cos chi - Q0 sin chi),  Y0 = M (P0 sin chi + Q0 cos chi)
                   J1 = M (P1 sin chi + Q1 cos chi),  Y1 = M (Q1 sin chi - P1 cos chi)
                   BJ = 1 + J1 rho0 - J0 rho1,        BY = Y1 rho0 - Y0 rho1
                   rho0 = (pi x/2)(H0 - Y0), rho1 = x((pi/2)(H1 - Y1) - 1)
                   (the Wronskian J1 Y0 - J0 Y1 = 2/(pi x), A&S 9.1.16, removes
                   the growing x Z0 term); P0, P1, rho0 are polynomials in
                   z = (8/x)^2 and Q0, Q1, rho1 are s = 8/x times polynomials in z
                   (A&S 9.2.5-9.2.10 and 12.1.30-12.1.31 give their asymptotic
                   forms).
  sin/cos of (pi/2) v for |v| <= 0.5 (a quarter-turn reduced phase).

Run:  python gen_fj_special.py  (needs mpmath and numpy; about a minute)
"""
import os
import sys

import mpmath as mp
import numpy as np

mp.mp.dps = 40
HERE = os.path.dirname(os.path.abspath(__file__))


def all_funcs(x):
    x = mp.mpf(x)
    j0, j1 = mp.besselj(0, x), mp.besselj(1, x)
    y0, y1 = mp.bessely(0, x), mp.bessely(1, x)
    h0, h1 = mp.struveh(0, x), mp.struveh(1, x)
    bj = x * j0 + mp.pi * x / 2 * (j1 * h0 - j0 * h1)
    by = x * y0 + mp.pi * x / 2 * (y1 * h0 - y0 * h1)
    return dict(j0=j0, j1=j1, bj=bj, y0=y0, y1=y1, by=by, h0=h0, h1=h1)


def cheb_nodes(n):
    k = np.arange(n)
    return np.cos(np.pi * (k + 0.5) / n)  # in (-1, 1)


def fit_monomial(t, vals, deg):
    """Least-squares fit in the Chebyshev basis on t in [-1,1], returned as
    monomial coefficients in t (lowest first)."""
    cf = np.polynomial.chebyshev.chebfit(t, vals, deg)
    return np.polynomial.chebyshev.cheb2poly(cf)


def to_var(coef_t, a, b):
    """Re-express a polynomial in t = a + b*v as a polynomial in v."""
    p = np.polynomial.Polynomial(coef_t)
    return p(np.polynomial.Polynomial([a, b])).coef


def horner_err(coef, v, ref, dtype):
    v = v.astype(dtype)
    c = [dtype(x) for x in coef]
    acc = np.full_like(v, c[-1])
    for ci in c[-2::-1]:
        acc = (acc.astype(np.longdouble) * v.astype(np.longdouble) + np.longdouble(ci)).astype(dtype)
    return float(np.max(np.abs(acc.astype(np.float64) - ref)))


# ---------------------------------------------------------------- sampling
NS = 160


def sample_S0():
    t = cheb_nodes(NS)
    w = (t + 1) / 2
    rows = []
    for wi in w:
        x = 2 * mp.sqrt(mp.mpf(wi))
        F = all_funcs(x)
        L = 2 / mp.pi * mp.log(x / 2)
        rows.append([F['j0'], F['j1'] / x, F['bj'] / x, F['y0'] - L * F['j0'],
                     (F['y1'] - L * F['j1'] + 2 / (mp.pi * x)) / x,
                     (F['by'] - L * F['bj']) / x])
    return t, w, np.array([[float(v) for v in r] for r in rows])


def sample_mid(xc, H):
    t = cheb_nodes(NS)
    rows = []
    for ti in t:
        F = all_funcs(mp.mpf(xc) + mp.mpf(H) * mp.mpf(ti))
        rows.append([F[k] for k in ('j0', 'j1', 'bj', 'y0', 'y1', 'by')])
    return t, np.array([[float(v) for v in r] for r in rows])


def sample_L():
    t = cheb_nodes(NS)
    z = (t + 1) / 2
    rows = []
    for zi in z:
        s = mp.sqrt(mp.mpf(zi))
        x = 8 / s
        F = all_funcs(x)
        chi = x - mp.pi / 4
        sq = mp.sqrt(mp.pi * x / 2)
        c, sn = mp.cos(chi), mp.sin(chi)
        P0 = sq * (F['j0'] * c + F['y0'] * sn)
        Q0 = sq * (F['y0'] * c - F['j0'] * sn)
        P1 = sq * (F['j1'] * sn - F['y1'] * c)
        Q1 = sq * (F['j1'] * c + F['y1'] * sn)
        rho0 = mp.pi * x / 2 * (F['h0'] - F['y0'])
        rho1 = x * (mp.pi / 2 * (F['h1'] - F['y1']) - 1)
        rows.append([P0, Q0 / s, P1, Q1 / s, rho0, rho1 / s])
    return t, z, np.array([[float(v) for v in r] for r in rows])


def sample_sincos():
    t = cheb_nodes(NS)
    v = t * 0.5
    sn = np.array([float(mp.sin(mp.pi / 2 * mp.mpf(vi)) / mp.mpf(vi)) for vi in v])
    cs = np.array([float(mp.cos(mp.pi / 2 * mp.mpf(vi))) for vi in v])
    return t, v, sn, cs


# ---------------------------------------------------------------- fitting
DEG = {
    'f32': dict(S0=6, MID=10, PQ=2, RHO=5, SIN=4, COS=4),
    'f64': dict(S0=13, MID=22, PQ=11, RHO=20, SIN=7, COS=8),
}


def main():
    out = {}
    report = []
    print('sampling ...', file=sys.stderr)
    t0, w0, V0 = sample_S0()
    t1, V1 = sample_mid(3.5, 1.5)
    t2, V2 = sample_mid(6.5, 1.5)
    tL, zL, VL = sample_L()
    tS, vS, SN, CS = sample_sincos()
    names6 = ['j0', 'j1', 'bj', 'y0', 'y1', 'by']
    namesL = ['p0', 'q0', 'p1', 'q1', 'rho0', 'rho1']
    for prec, dt in (('f32', np.float32), ('f64', np.float64)):
        D = DEG[prec]
        # S0 in w = (t+1)/2
        for i, nm in enumerate(['a', 'b', 'c', 'd', 'e', 'f']):
            cw = to_var(fit_monomial(t0, V0[:, i], D['S0']), -1.0, 2.0)
            out[(prec, 's0_' + nm)] = cw
            report.append((prec, 's0_' + nm, horner_err(cw, w0, V0[:, i], dt)))
        for tag, tt, VV in (('s1', t1, V1), ('s2', t2, V2)):
            for i, nm in enumerate(names6):
                cu = fit_monomial(tt, VV[:, i], D['MID'])
                out[(prec, tag + '_' + nm)] = cu
                report.append((prec, tag + '_' + nm, horner_err(cu, tt, VV[:, i], dt)))
        for i, nm in enumerate(namesL):
            deg = D['RHO'] if nm.startswith('rho') else D['PQ']
            cz = to_var(fit_monomial(tL, VL[:, i], deg), -1.0, 2.0)
            err = horner_err(cz, zL, VL[:, i], dt)
            if prec == 'f64' and err > 1e-14:
                # monomial in z is ill-conditioned at high degree: use t = 2z-1
                cz = fit_monomial(tL, VL[:, i], deg)
                out[(prec, 'L_' + nm + '_t')] = cz
                report.append((prec, 'L_' + nm + '_t', horner_err(cz, tL, VL[:, i], dt)))
            else:
                out[(prec, 'L_' + nm)] = cz
                report.append((prec, 'L_' + nm, err))
        # sin(pi v/2)/v odd part as polynomial in v^2, cos as polynomial in v^2
        v2 = vS * vS
        ts = 8 * v2 - 1  # p = 4 v^2 in [0, 1] -> t = 2p - 1 in [-1, 1]
        scale = 4.0 ** np.arange(D['SIN'] + 1)
        cs_ = to_var(fit_monomial(ts, SN, D['SIN']), -1.0, 2.0) * scale
        scale = 4.0 ** np.arange(D['COS'] + 1)
        cc_ = to_var(fit_monomial(ts, CS, D['COS']), -1.0, 2.0) * scale
        out[(prec, 'sin')] = cs_
        out[(prec, 'cos')] = cc_
        report.append((prec, 'sin', horner_err(cs_, v2, SN, dt)))
        report.append((prec, 'cos', horner_err(cc_, v2, CS, dt)))

    lines = [
        '// Generated by gen_fj_special.py: do not edit by hand.',
        '// Polynomial coefficients (lowest degree first) of the F-J special',
        '// functions; each comment gives the max abs error of Horner evaluation',
        '// in that precision on the fit nodes.',
        '#pragma once',
        '',
    ]
    for (prec, nm), cf in out.items():
        err = [e for p, n, e in report if p == prec and n == nm][0]
        ty = 'float' if prec == 'f32' else 'double'
        suf = 'f' if prec == 'f32' else ''
        body = ', '.join(repr(float(dt(c))) + suf if prec == 'f32' else repr(float(c)) for c in cf
                         for dt in [np.float32 if prec == 'f32' else np.float64])
        lines.append('// max err %.2e' % err)
        lines.append('#define FJC_%s_%s_N %d' % (prec.upper(), nm.upper(), len(cf)))
        lines.append('#define FJC_%s_%s { %s }' % (prec.upper(), nm.upper(), body))
    with open(os.path.join(HERE, 'fj_special_coeffs.h'), 'w') as fh:
        fh.write('\n'.join(lines) + '\n')
    for p, n, e in report:
        print('%s %-10s %.2e' % (p, n, e))


if __name__ == '__main__':
    main()
