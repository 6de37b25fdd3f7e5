"""FP64 CPU restatement of CC-FJpy's F-J path -- TEST INFRASTRUCTURE ONLY.

This module is the checker for the CUDA implementation: only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import it. The
product (cc-fjpy_b200/ccfj) never imports it and has no CPU fallback.

What it restates (reference file:line):

* fj_integral / fj_trap -- the four pair-sum loops of src/FJcpu.cpp
  (integral_J :230-273, integral_Y :276-319, trap_J :323-362,
  trap_Y :364-399) with their dispatchers FJ/FH (:401-419): for every
  (f, c), k = 2 pi f / c, sum over the intervals of the distance-sorted
  pairs of the integral of the linearly interpolated spectrum times
  r Z0(k r), Z = J (FJ) or Y (FH), with b = (g2 - g1) / max(r2 - r1, 0.1),
  a = g1 - r1 b. The trapezoid sums (g1 Z0(k r1) r1 + g2 Z0(k r2) r2) dr0 / 2.
* fj_noise / fj_earthquake / MWFJ / win -- the Python layer of
  src/ccfj-gpu.pyx:168-313: np.argsort(r), float32 casts, fstride slicing,
  np.fft.rfft, scipy.fftpack.hilbert (scipy is the reference's own
  dependency; pinned here to the installed scipy 1.18.1), magnitude and the
  per-frequency max-abs normalisation with Python's builtin max.

Arithmetic: everything in float64 on the float32-cast inputs, with exact pi
(the reference rounds k to float32 and redefines pi as 3.14159265358). The
integral of one interval is computed
  - with the reference's closed form (A&S 11.1.7/11.1.8 for the integral of
    Z0; scipy's j0, j1, y0, y1, jv and struve_h01 below) when k dr >= 1,
    where it is well conditioned, and
  - by 6-point Gauss-Legendre quadrature of the same integrand when
    k dr < 1 (exact for polynomials of degree 11; error < 1e-15 relative
    there), because the closed form cancels catastrophically for short
    intervals (about log10(2/(k dr)^2) digits).
fj_integral_closed() is the literal closed form everywhere, used to pin the
restatement against the reference's own outputs.
"""
import numpy as np
import scipy.special as sp
from scipy import fftpack

__all__ = ["struve_h01", "z_values", "fj_integral", "fj_integral_closed", "fj_trap", "fj_transform",
           "fj_noise", "fj_earthquake", "fj_earthquake_columns", "MWFJ", "mwfj_window_columns",
           "win", "hilbert_rows", "rel_error"]

_GL_X, _GL_W = np.polynomial.legendre.leggauss(6)
DR_FLOOR = float(np.float32(0.1))  # fmaxf(r2 - r1, 0.1) in float32, src/FJcpu.cpp:259


_ASYM_FROM = 40.0     # the asymptotic series reaches < 1e-19 relative there


def struve_h01(x):
    """Struve H0(x), H1(x) in float64 for x >= 0.

    x < 40: the Bessel-function series (A&S 12.1.19-20)
        H0 = (4/pi) sum_{k>=0} J_{2k+1}(x) / (2k+1)
        H1 = (2/pi)(1 - J0(x)) + (4/pi) sum_{k>=1} J_{2k}(x) / (4k^2 - 1)
    whose terms are bounded (no cancellation) and vanish once 2k > x + 35.
    x >= 40: H_nu - Y_nu from the asymptotic series (A&S 12.1.30) with
        Gamma(k+1/2)/Gamma(nu+1/2-k) = (-1)^k Gamma(k+1/2)^2 / (pi (1/2-k)^nu)
    truncated at 40 terms (its smallest term is below 1e-19 relative).
    scipy.special.struve is not used: it returns NaN at some arguments
    (for example x = 25.765)."""
    x = np.asarray(x, dtype=np.float64)
    h0 = np.empty_like(x)
    h1 = np.empty_like(x)
    for x_lo, x_hi in ((0.0, 10.0), (10.0, 20.0), (20.0, _ASYM_FROM)):
        lo = (x >= x_lo) & (x < x_hi)
        if not lo.any():
            continue
        xl = x[lo]
        nt = int(np.ceil((x_hi + 36) / 2))  # J_n(x) < 1e-30 once n > x + 35
        n = np.arange(nt)
        jodd = sp.jv((2 * n + 1)[:, None], xl[None, :])
        h0[lo] = 4 / np.pi * np.sum(jodd / (2 * n + 1)[:, None], axis=0)
        k = np.arange(1, nt)
        jeven = sp.jv((2 * k)[:, None], xl[None, :])
        h1[lo] = 2 / np.pi * (1 - sp.j0(xl)) + 4 / np.pi * np.sum(
            jeven / (4.0 * k * k - 1)[:, None], axis=0)
    hi = x >= _ASYM_FROM
    if hi.any():
        xh = x[hi]
        kk = np.arange(40)
        g2 = np.exp(2 * sp.gammaln(kk + 0.5)) * (-1.0) ** kk / np.pi  # (-1)^k Gamma(k+1/2)^2 / pi
        t = 2.0 / xh[None, :]
        r0 = np.sum(g2[:, None] * t ** (2 * kk + 1)[:, None], axis=0) / np.pi
        r1 = np.sum((g2 / (0.5 - kk))[:, None] * t ** (2 * kk)[:, None], axis=0) / np.pi
        h0[hi] = sp.y0(xh) + r0
        h1[hi] = sp.y1(xh) + r1
    return h0, h1


def z_values(x, basis):
    """Z0(x), Z1(x) and B(x) = int_0^x Z0 for basis 'J' or 'Y' (float64).
    B = x Z0 + (pi x / 2)(Z1 H0 - Z0 H1), as src/FJcpu.cpp:265-266."""
    x = np.asarray(x, dtype=np.float64)
    if basis == "J":
        z0, z1 = sp.j0(x), sp.j1(x)
    else:
        z0, z1 = sp.y0(x), sp.y1(x)
    h0, h1 = struve_h01(x)
    b = x * z0 + np.pi * x / 2 * (z1 * h0 - z0 * h1)
    return z0, z1, b


def _z0(x, basis):
    return sp.j0(x) if basis == "J" else sp.y0(x)


def _interval_sums(g, r, k, basis, closed_only):
    """Sum over intervals of int_{r1}^{r2} (a + b r) r Z0(k r) dr for every
    k in the vector `k` (one frequency column g of length nr)."""
    nr = len(r)
    if nr < 2:
        return np.zeros_like(k)
    r1, r2 = r[:-1], r[1:]
    g1, g2 = g[:-1], g[1:]
    dr0 = np.maximum(r2 - r1, DR_FLOOR)
    b = (g2 - g1) / dr0
    a = g1 - r1 * b
    K = k[:, None] * np.ones((1, nr - 1))
    x1, x2 = K * r1[None, :], K * r2[None, :]
    if closed_only:
        use_closed = np.ones(K.shape, dtype=bool)
    else:
        use_closed = np.abs(x2 - x1) >= 1.0
        if basis == "Y":
            use_closed |= np.abs(x2 - x1) > np.abs(x1)
    terms = np.zeros(K.shape)
    with np.errstate(all="ignore"):
        if use_closed.any():
            ci, ii = np.nonzero(use_closed)
            kk = k[ci]
            A1 = z_values(x1[ci, ii], basis)
            A2 = z_values(x2[ci, ii], basis)
            R1, R2, aa, bb = r1[ii], r2[ii], a[ii], b[ii]
            terms[ci, ii] = (aa * (R2 * A2[1] - R1 * A1[1]) / kk
                             + bb * (R2 * R2 * A2[1] - R1 * R1 * A1[1]) / kk
                             + bb * (R2 * A2[0] - R1 * A1[0]) / kk / kk
                             - bb * (A2[2] - A1[2]) / kk / kk / kk)
        short = ~use_closed
        if short.any():
            ci, ii = np.nonzero(short)
            rr1, rr2 = r1[ii], r2[ii]
            mid, half = 0.5 * (rr1 + rr2), 0.5 * (rr2 - rr1)
            rs = mid[:, None] + half[:, None] * _GL_X[None, :]
            kk = k[ci][:, None]
            # a + b r written as g1 + b (r - r1): no cancellation for short intervals
            fv = (g1[ii][:, None] + b[ii][:, None] * (rs - rr1[:, None])) * rs * _z0(kk * rs, basis)
            terms[ci, ii] = half * (fv @ _GL_W)
    return terms.sum(axis=1)


def fj_integral(U, r, f, c, basis="J", closed_only=False):
    """FJ/FH type 1 (src/FJcpu.cpp:230-319): U float[nr, nf] rows in the order
    of r, f[nf], c[nc] -> float64 [nc, nf]."""
    U = np.asarray(U, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    f = np.asarray(f, dtype=np.float64)
    c = np.asarray(c, dtype=np.float64)
    out = np.empty((len(c), len(f)))
    for i, fl in enumerate(f):
        k = 2 * np.pi * fl / c
        with np.errstate(all="ignore"):
            out[:, i] = _interval_sums(U[:, i], r, k, basis, closed_only)
            if len(r) > 1:
                # the reference divides by k: k = 0 (f = 0) gives NaN
                out[k == 0, i] = np.nan
    return out


def fj_integral_closed(U, r, f, c, basis="J"):
    """The reference's closed form for every interval (no quadrature)."""
    return fj_integral(U, r, f, c, basis, closed_only=True)


def fj_trap(U, r, f, c, basis="J"):
    """FJ/FH type 0 (src/FJcpu.cpp:323-399) in float64."""
    U = np.asarray(U, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    f = np.asarray(f, dtype=np.float64)
    c = np.asarray(c, dtype=np.float64)
    out = np.empty((len(c), len(f)))
    if len(r) < 2:
        out[:] = 0
        return out
    r1, r2 = r[:-1], r[1:]
    dr0 = np.maximum(r2 - r1, DR_FLOOR)
    for i, fl in enumerate(f):
        K = (2 * np.pi * fl / c)[:, None]
        g1, g2 = U[:-1, i], U[1:, i]
        with np.errstate(all="ignore"):
            t = (g1 * _z0(K * r1, basis) * r1 + g2 * _z0(K * r2, basis) * r2) * dr0 * 0.5
        out[:, i] = t.sum(axis=1)
    return out


def fj_transform(U, r, f, c, itype=1, basis="J"):
    """FJ (basis J) / FH (basis Y) dispatch of src/FJcpu.cpp:401-419; an
    itype other than 0 or 1 leaves the (zero) output untouched."""
    if itype == 1:
        return fj_integral(U, r, f, c, basis)
    if itype == 0:
        return fj_trap(U, r, f, c, basis)
    return np.zeros((len(c), len(f)))


def _prep(uf, r, c, f, fstride):
    """The `fj` shim's view of its arguments (src/ccfj-gpu.pyx:181-200):
    stride, flatten to [nr*nf], cast everything to float32."""
    nr, nf = len(r), len(f)
    u = np.asarray(uf)[:, ::fstride]
    u = u.reshape(nr * nf)
    if np.iscomplexobj(u):
        u = u.real
    return (u.astype(np.float32).reshape(nr, nf), np.asarray(r, dtype=np.float32),
            np.asarray(f, dtype=np.float32), np.asarray(c, dtype=np.float32))


def _normalize(out):
    """out[:, i] /= max(abs(out[:, i])) with Python's builtin max
    (src/ccfj-gpu.pyx:266-267)."""
    out = np.array(out)
    with np.errstate(all="ignore"):
        for i in range(out.shape[1]):
            out[:, i] = out[:, i] / max(np.abs(out[:, i]))
    return out


def hilbert_rows(uf):
    """scipy.fftpack.hilbert of every row (the real part of complex rows),
    as src/ccfj-gpu.pyx:258-260 stores it into a float32 array."""
    uf = np.asarray(uf)
    out = np.zeros(uf.shape, dtype=np.float32)
    for i in range(uf.shape[0]):
        out[i, :] = fftpack.hilbert(np.real(uf[i, :]))
    return out


def fj_noise(uf, r, c, f, fstride=1, itype=1, func=0, normalize=True):
    """src/ccfj-gpu.pyx:241-268 in float64 (returns float64 [nc, nf])."""
    indx = np.argsort(r)
    r = np.asarray(r)[indx]
    uf = np.asarray(uf)[indx]
    U, r32, f32, c32 = _prep(uf, r, c, f, fstride)
    if func == 0:
        out = fj_transform(U, r32, f32, c32, itype, "J")
    else:
        ufi = hilbert_rows(uf)
        Ui = _prep(ufi, r, c, f, fstride)[0]
        out = fj_transform(U, r32, f32, c32, itype, "J") - fj_transform(Ui, r32, f32, c32, itype, "Y")
    return _normalize(out) if normalize else out


def _eq_spectra(u, r, f, fstride):
    indx = np.argsort(r)
    r = np.asarray(r)[indx]
    u1 = np.asarray(u)[indx]
    uf = np.fft.rfft(u1)[:, 0:len(f) * fstride:fstride]
    return r, np.real(uf), np.imag(uf)


def fj_earthquake(u, r, c, f, fstride=1, itype=1, func=0, normalize=True):
    """src/ccfj-gpu.pyx:270-295 in float64 (returns float64 [nc, nf])."""
    r, ufr, ufi = _eq_spectra(u, r, f, fstride)
    R, r32, f32, c32 = _prep(ufr, r, c, f, fstride)
    I = _prep(ufi, r, c, f, fstride)[0]
    T = lambda X, basis: fj_transform(X, r32, f32, c32, itype, basis)  # noqa: E731
    if func == 0:
        outr, outi = T(R, "J"), T(I, "J")
    else:
        outr = T(R, "J") - T(I, "Y")
        outi = T(I, "J") + T(R, "Y")
    out = np.sqrt(outr ** 2 + outi ** 2)
    return _normalize(out) if normalize else out


def fj_earthquake_columns(u, r, c, f, cols, itype=1, func=0):
    """fj_earthquake (src/ccfj-gpu.pyx:270-295) restricted to the frequency
    bins `cols` of f (fstride 1): the same rfft, the same float32 casts, the
    transform of those columns only and their normalisation (every column
    is independent of the others, so this equals the full call's columns).
    Returns float64 [nc, len(cols)]."""
    r, ufr, ufi = _eq_spectra(u, r, f, 1)
    cols = np.asarray(cols)
    fc = np.asarray(f)[cols]
    R, r32, f32, c32 = _prep(ufr[:, cols], r, c, fc, 1)
    I = _prep(ufi[:, cols], r, c, fc, 1)[0]
    T = lambda X, basis: fj_transform(X, r32, f32, c32, itype, basis)  # noqa: E731
    if func == 0:
        outr, outi = T(R, "J"), T(I, "J")
    else:
        outr = T(R, "J") - T(I, "Y")
        outi = T(I, "J") + T(R, "Y")
    return _normalize(np.sqrt(outr ** 2 + outi ** 2))


def mwfj_window_columns(u, r, c, f, Fs, winl_w, winr_w, cols, taper=0.9, itype=1, func=0):
    """One window of MWFJ (src/ccfj-gpu.pyx:297-313): every trace j times
    win(npts, Fs, winl_w[j], winr_w[j], taper), then fj_earthquake on the
    bins `cols` (float64 [nc, len(cols)])."""
    u = np.asarray(u)
    nr, npts = len(r), u.shape[1]
    u0 = np.zeros([nr, npts])
    for j in range(nr):
        u0[j, :] = u[j, :] * win(npts, Fs, winl_w[j], winr_w[j], taper)
    return fj_earthquake_columns(u0, r, c, f, cols, itype, func)


def win(npts, Fs, T1, T2, taper=0.8):
    """src/ccfj-gpu.pyx:168-178 (same float64 arithmetic)."""
    n1 = max(0, np.floor(T1 * Fs))
    n2 = min(npts, np.floor(T2 * Fs))
    out = np.ones(npts)
    delta = np.floor((n2 - n1) * (1 - taper) / 2)
    out[0:int(n1)] = 0
    out[int(n2):int(npts)] = 0
    for i in range(int(delta)):
        out[int(n1 + i)] = np.sin(np.pi / 2 * i / delta)
        out[int(n2 - i - 1)] = np.sin(np.pi / 2 * i / delta)
    return out


def MWFJ(u, r, c, f, Fs, nwin, winl, winr, taper=0.9, fstride=1, itype=1, func=0,
         normalize=True):
    """src/ccfj-gpu.pyx:297-313 in float64 (returns float64 [nwin, nc, nf])."""
    nr = len(r)
    npts = len(u[0])
    out = np.zeros([nwin, len(c), len(f)])
    for i in range(nwin):
        u0 = np.zeros([nr, npts])
        for j in range(nr):
            u0[j, :] = u[j, :] * win(npts, Fs, winl[i, j], winr[i, j], taper)
        out[i] = fj_earthquake(u0, r, c, f, fstride, itype, func, normalize)
    return out


def rel_error(y, y64):
    """max over (c, f) of |y - y64| / max_c |y64[:, f]| (the absolute error
    after per-frequency normalisation), ignoring columns that are not finite
    in y64."""
    y = np.asarray(y, dtype=np.float64)
    y64 = np.asarray(y64, dtype=np.float64)
    scale = np.max(np.abs(y64), axis=-2, keepdims=True)
    ok = np.isfinite(scale) & (scale > 0)
    ok = np.broadcast_to(ok, y64.shape)
    d = np.abs(y - y64) / np.where(ok, scale, 1.0)
    return float(np.max(np.where(ok, d, 0.0)))
