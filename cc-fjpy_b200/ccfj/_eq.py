"""fj_earthquake and MWFJ (time-domain traces) over ccfj_fj_earthquake_v1."""
import ctypes
import os

import numpy as np

from . import _lib

_FUNC_MSG = "set func as 0 for Bessel function 1 for Hankel function"


class EqArgs(ctypes.Structure):
    """Mirror of struct ccfj_eq_args (include/ccfj_b200.h)."""

    _fields_ = [
        ("struct_size", ctypes.c_int),
        ("ntr", ctypes.c_int),
        ("npts", ctypes.c_int),
        ("nf", ctypes.c_int),
        ("nc", ctypes.c_int),
        ("itype", ctypes.c_int),
        ("func", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("normalize", ctypes.c_int),
        ("device_ptrs", ctypes.c_int),
        ("fstride", ctypes.c_int),
        ("nwin", ctypes.c_int),
        ("u", ctypes.c_void_p),
        ("u_ld", ctypes.c_longlong),
        ("u_rows", ctypes.c_longlong),
        ("perm", ctypes.c_void_p),
        ("r", ctypes.c_void_p),
        ("f", ctypes.c_void_p),
        ("c", ctypes.c_void_p),
        ("win_n1", ctypes.c_void_p),
        ("win_n2", ctypes.c_void_p),
        ("win_delta", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("tau", ctypes.c_float),
        ("out_f64", ctypes.c_int),
    ]


_lib.SIGNATURES["ccfj_fj_earthquake_v1"] = (ctypes.c_int, [ctypes.POINTER(EqArgs),
                                                            ctypes.c_void_p])
_lib.SIGNATURES["ccfj_set_mwfj_path"] = (ctypes.c_int, [ctypes.c_int])
_lib.SIGNATURES["ccfj_device_status"] = (ctypes.c_int, [ctypes.c_void_p])
_lib.SIGNATURES["ccfj_self_test_wait_timeout"] = (ctypes.c_int, [ctypes.c_void_p])


def _check_bins(nr, npts, nf, fstride):
    """The reference slices rfft bins 0:nf*fstride:fstride and then `fj`
    strides the result again (src/ccfj-gpu.pyx:278 and :185); numpy's
    reshape then fails unless the element counts agree. Reproduce that."""
    nb = npts // 2 + 1
    cols1 = len(range(0, min(nf * fstride, nb), fstride))
    cols2 = len(range(0, cols1, fstride))
    if nr * cols2 != nr * nf:
        raise ValueError("cannot reshape array of size %d into shape (%d,)" % (nr * cols2, nr * nf))


def _win_params(npts, Fs, T1, T2, taper):
    """Integer n1, n2, delta of the reference's `win` (src/ccfj-gpu.pyx:
    168-178), vectorised over arrays of T1, T2 in float64 as `win` does.

    `win` zeroes out[0:n1] and out[n2:npts] (a negative n2 counts from the
    end), then for i < delta writes sin(pi/2 i/delta) to out[n1 + i] and
    out[n2 - 1 - i] (a negative index again counts from the end). The device
    taper reproduces that from (n1, n2, delta); where the loop would index
    past the array, `win` raises IndexError, and so does this."""
    n1 = np.maximum(0, np.floor(np.asarray(T1, dtype=np.float64) * Fs))
    n2 = np.minimum(npts, np.floor(np.asarray(T2, dtype=np.float64) * Fs))
    delta = np.floor((n2 - n1) * (1 - taper) / 2)
    n1i = n1.astype(np.int64)
    n2i = n2.astype(np.int64)
    di = np.maximum(delta, 0).astype(np.int64)  # range(int(delta)) is empty if < 0
    # first loop index that leaves the array: out[n1 + i] past the end, or
    # out[n2 - 1 - i] before -npts (the n1 write comes first within an i)
    ia = np.maximum(npts - n1i, 0)
    ib = np.maximum(n2i + npts, 0)
    bad = np.minimum(ia, ib) < di
    if np.any(bad):
        k = np.flatnonzero(bad.ravel())[0]
        a_, b_ = ia.ravel()[k], ib.ravel()[k]
        idx = n1i.ravel()[k] + a_ if a_ <= b_ else n2i.ravel()[k] - 1 - b_
        raise IndexError("index %d is out of bounds for axis 0 with size %d" % (idx, npts))
    # beyond [-npts, npts] the slices clamp, which the device rule also does
    return (np.clip(n1i, 0, npts).astype(np.int32), np.clip(n2i, -npts, npts).astype(np.int32),
            di.astype(np.int32))


def _run(u, r, c, f, fstride, itype, func, nwin=0, wins=None, precision=_lib.PREC_FP32,
         dtype=np.float32):
    lib = _lib.load()
    u = np.asarray(u)
    nr, nc, nf = len(r), len(c), len(f)
    r = np.asarray(r)
    indx = np.argsort(r)
    rs = np.ascontiguousarray(r[indx], dtype=np.float32)
    if u.dtype == np.float32 and u.strides[1] == 4 and u.strides[0] % 4 == 0 and u.strides[0] > 0:
        u32, ld = u, u.strides[0] // 4
    else:
        u32 = np.ascontiguousarray(u, dtype=np.float32)
        ld = u32.shape[1]
    npts = u32.shape[1]
    if u32.shape[0] < nr:
        raise IndexError("index %d is out of bounds for axis 0 with size %d" % (nr - 1, u32.shape[0]))
    _check_bins(nr, npts, nf, fstride)
    f32 = np.ascontiguousarray(f, dtype=np.float32)
    c32 = np.ascontiguousarray(c, dtype=np.float32)
    perm = np.ascontiguousarray(indx, dtype=np.int64)
    nw = max(nwin, 1)
    # float64 (MWFJ's result) is converted by the library while it copies out
    out = np.empty((nw, nc, nf) if nwin > 0 else (nc, nf), dtype=np.dtype(dtype))
    if out.dtype not in (np.float32, np.float64):
        raise ValueError("dtype must be float32 or float64")
    a = EqArgs()
    a.struct_size = ctypes.sizeof(EqArgs)
    a.ntr, a.npts, a.nf, a.nc = nr, npts, nf, nc
    a.itype, a.func, a.precision = int(itype), int(func), int(precision)
    a.normalize, a.device_ptrs, a.fstride, a.nwin = 1, 0, int(fstride), int(nwin)
    a.u, a.u_ld, a.u_rows = u32.ctypes.data, ld, u32.shape[0]
    a.perm, a.r, a.f, a.c = perm.ctypes.data, rs.ctypes.data, f32.ctypes.data, c32.ctypes.data
    if nwin > 0:
        n1, n2, dl = wins
        a.win_n1, a.win_n2, a.win_delta = n1.ctypes.data, n2.ctypes.data, dl.ctypes.data
    a.out = out.ctypes.data
    a.out_f64 = int(out.dtype == np.float64)
    _lib.check(lib.ccfj_fj_earthquake_v1(ctypes.byref(a), None))
    return out


def fj_earthquake(u, r, c, f, fstride=1, itype=1, func=0, num=-1):
    """F-J spectrum of earthquake records (reference `fj_earthquake`,
    src/ccfj-gpu.pyx:270-295): argsort r, real FFT of every trace (on the
    GPU), bins 0..len(f)-1 (times fstride), F-J of the real and imaginary
    parts combined as a magnitude, per-frequency normalisation. u: [ntr, npts]
    traces; f must be the matching bin frequencies (Fs * k / npts).
    Returns float32 [nc, nf]."""
    if num != -1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(int(num))
    if func not in (0, 1):
        print(_FUNC_MSG)
        return 0
    if itype not in (0, 1):
        raise ValueError("itype must be 0 (trapezoid) or 1 (linear integral), got %r" % (itype,))
    return _run(u, r, c, f, fstride, itype, func)


def MWFJ(u, r, c, f, Fs, nwin, winl, winr, taper=0.9, fstride=1, itype=1, func=0, num=-1):
    """Multi-window F-J (reference `MWFJ`, src/ccfj-gpu.pyx:297-313): for
    window i every trace j is multiplied by win(npts, Fs, winl[i, j],
    winr[i, j], taper) and transformed as in fj_earthquake. All windows run
    in one batched device pass sharing the station geometry.
    Returns float64 [nwin, nc, nf]."""
    if num != -1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(int(num))
    if func not in (0, 1):
        # the reference prints once per window and stores 0 in out[i]
        out = np.zeros([nwin, len(c), len(f)])
        for _ in range(nwin):
            print(_FUNC_MSG)
        return out
    if itype not in (0, 1):
        raise ValueError("itype must be 0 (trapezoid) or 1 (linear integral), got %r" % (itype,))
    u = np.asarray(u)
    nr = len(r)
    npts = len(u[0])
    if nwin <= 0:
        return np.zeros([max(nwin, 0), len(c), len(f)])
    winl = np.asarray(winl, dtype=np.float64)[:nwin, :nr]
    winr = np.asarray(winr, dtype=np.float64)[:nwin, :nr]
    n1, n2, dl = _win_params(npts, Fs, winl, winr, taper)
    wins = tuple(np.ascontiguousarray(x, dtype=np.int32) for x in (n1, n2, dl))
    return _run(u[:nr], r, c, f, fstride, itype, func, nwin=nwin, wins=wins, dtype=np.float64)
