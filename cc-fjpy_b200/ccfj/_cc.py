"""Ambient-noise cross-correlation (the reference's `CC`, src/ccfj.pyx:125-147
and src/ccfj-gpu.pyx:146-167, over CrossCorrelation in src/CrossCorr.cpp)
on the device through ccfj_cc_v1.

Kept from the reference wrapper: steplen = int(fftlen * (1 - overlaprate)),
npairs = int(len(Pairs) / 2), a float32 cast of `data` that copies only when
the dtype differs (so one-bit rewrites a contiguous float32 caller array in
place, as the reference does), 1-D int32 Pairs / startend and 1-D float32
data (the reference's typed memoryviews raise ValueError otherwise), and a
complex64 [npairs, nf] result. nThreads (the reference's OpenMP thread
count) is ignored. A strided 1-D array, which the reference reads through a
bare pointer as if it were contiguous, is read at its own elements from a
contiguous copy.
"""
import ctypes

import numpy as np

from . import _lib


class CcArgs(ctypes.Structure):
    """Mirror of struct ccfj_cc_args (include/ccfj_b200.h)."""

    _fields_ = [
        ("struct_size", ctypes.c_int),
        ("nsta", ctypes.c_int),
        ("npts", ctypes.c_int),
        ("nf", ctypes.c_int),
        ("npairs", ctypes.c_int),
        ("fstride", ctypes.c_int),
        ("fftlen", ctypes.c_int),
        ("steplen", ctypes.c_int),
        ("onebit", ctypes.c_int),
        ("whiten", ctypes.c_int),
        ("device_ptrs", ctypes.c_int),
        ("accumulate", ctypes.c_int),
        ("out_layout", ctypes.c_int),
        ("pairs", ctypes.c_void_p),
        ("startend", ctypes.c_void_p),
        ("data", ctypes.c_void_p),
        ("out_re", ctypes.c_void_p),
        ("out_im", ctypes.c_void_p),
    ]


class CcData(ctypes.Structure):
    """Mirror of struct ccfj_cc_data, the reference's CC_data
    (include/CrossCorr.h:13-29)."""

    _fields_ = [
        ("nsta", ctypes.c_int),
        ("npts", ctypes.c_int),
        ("nf", ctypes.c_int),
        ("npairs", ctypes.c_int),
        ("fstride", ctypes.c_int),
        ("fftlen", ctypes.c_int),
        ("steplen", ctypes.c_int),
        ("Pairs", ctypes.c_void_p),
        ("startend", ctypes.c_void_p),
        ("data", ctypes.c_void_p),
        ("ncfsr", ctypes.c_void_p),
        ("ncfsi", ctypes.c_void_p),
        ("ifonebit", ctypes.c_int),
        ("ifspecwhitenning", ctypes.c_int),
        ("nThreads", ctypes.c_int),
    ]


_lib.SIGNATURES["ccfj_cc_v1"] = (ctypes.c_int, [ctypes.POINTER(CcArgs), ctypes.c_void_p])
_lib.SIGNATURES["CrossCorrelation"] = (ctypes.c_int, [CcData])

_CTYPE_NAMES = {np.dtype(np.int64): "long", np.dtype(np.int16): "short",
                np.dtype(np.float64): "double", np.dtype(np.float32): "float",
                np.dtype(np.int32): "int", np.dtype(np.uint32): "unsigned int"}


def _buffer_1d(x, dtype, cname):
    """The check of a Cython typed memoryview `cname[:]`: a 1-D buffer of
    exactly that type. Returns a C-contiguous view (a copy when strided)."""
    return np.ascontiguousarray(_buffer_1d_checked(x, dtype, cname))


def _buffer_1d_checked(x, dtype, cname):
    """The same check, returning the array itself (never a copy)."""
    if not isinstance(x, np.ndarray):
        try:
            memoryview(x)
        except TypeError:
            raise TypeError("a bytes-like object is required, not '%s'" % type(x).__name__)
        x = np.asarray(x)
    if x.ndim != 1:
        raise ValueError("Buffer has wrong number of dimensions (expected 1, got %d)" % x.ndim)
    if x.dtype != dtype:
        raise ValueError("Buffer dtype mismatch, expected '%s' but got '%s'"
                         % (cname, _CTYPE_NAMES.get(x.dtype, str(x.dtype))))
    return x


def _prepare(npts, nsta, nf, fftlen, Pairs, startend, data, overlaprate=0.0, fstride=1,
             ifonebit=0, ifspecwhittenning=1):
    """The reference wrapper's argument handling: returns (args, arrays the
    args point into, output array)."""
    steplen = int(fftlen * (1 - overlaprate))
    npairs = int(len(Pairs) / 2)
    if data.dtype != np.float32:
        data = np.array(data, dtype=np.float32)
    pairs = _buffer_1d(Pairs, np.int32, "int")
    se = _buffer_1d(startend, np.int32, "int")
    flat = _buffer_1d(data, np.float32, "float")
    if len(se) < 2 * nsta:
        raise ValueError("startend holds %d values, %d stations need %d" % (len(se), nsta, 2 * nsta))
    if flat.size < nsta * npts:
        raise ValueError("data holds %d samples, %d stations of %d need %d"
                         % (flat.size, nsta, npts, nsta * npts))
    out = np.zeros((npairs, nf), dtype=np.complex64)
    a = CcArgs()
    a.struct_size = ctypes.sizeof(CcArgs)
    a.nsta, a.npts, a.nf, a.npairs = int(nsta), int(npts), int(nf), npairs
    a.fstride, a.fftlen, a.steplen = int(fstride), int(fftlen), steplen
    a.onebit = 1 if ifonebit else 0
    a.whiten = 1 if ifspecwhittenning else 0
    a.device_ptrs, a.accumulate, a.out_layout = 0, 0, 1
    a.pairs, a.startend = pairs.ctypes.data, se.ctypes.data
    a.data = flat.ctypes.data
    a.out_re, a.out_im = out.ctypes.data, None
    return a, (pairs, se, flat), out


def CC(npts, nsta, nf, fftlen, Pairs, startend, data, overlaprate=0.0, nThreads=8, fstride=1,
       ifonebit=0, ifspecwhittenning=1):
    """Cross-spectra of station pairs (reference `CC`): for every pair the
    mean over the windows both stations keep of conj(X_a) X_b, X the
    (one-bit, whitened) real FFT of a window at bins j*fstride, j < nf.
    Returns complex64 [npairs, nf]."""
    a, _keep, out = _prepare(npts, nsta, nf, fftlen, Pairs, startend, data, overlaprate,
                             fstride, ifonebit, ifspecwhittenning)
    _lib.check(_lib.load().ccfj_cc_v1(ctypes.byref(a), None))
    return out


_lib.SIGNATURES["ccfj_cc_fj_noise_v1"] = (ctypes.c_int, [ctypes.POINTER(CcArgs),
                                                          ctypes.POINTER(_lib.FjArgs),
                                                          ctypes.c_void_p])


def cc_fj_noise(npts, nsta, nf, fftlen, Pairs, startend, data, r, c, f, overlaprate=0.0,
                fstride=1, ifonebit=0, ifspecwhittenning=1, itype=1, func=0):
    """Records to a normalised F-J dispersion spectrum in one call: the
    reference's pipeline CC(...) followed by fj_noise(ncfs, r, c, f, itype,
    func) (examples/example_noise.py:6-11), with the cross-spectra kept on
    the device between the two steps. The records cross to the device once
    and the float32 [nc, nf] spectrum comes back once.

    The CC arguments are those of `CC` (one-bit is applied to the samples as
    they are read: `data` is not rewritten, unlike CC); r [npairs] holds the
    distance of each pair of Pairs, f the nf frequencies of the bins
    j*fstride, c the velocities; itype and func as in fj_noise (func 1 takes
    the Hilbert transform of each pair's spectrum along frequency)."""
    if func not in (0, 1):
        raise ValueError("func must be 0 (Bessel) or 1 (Hankel), got %r" % (func,))
    if itype not in (0, 1):
        raise ValueError("itype must be 0 or 1, got %r" % (itype,))
    a, keep, _ = _prepare(npts, nsta, nf, fftlen, Pairs, startend, data, overlaprate, fstride,
                          ifonebit, ifspecwhittenning)
    npairs = a.npairs
    r = np.asarray(r)
    if r.shape != (npairs,):
        raise ValueError("r must hold one distance per pair (%d), got shape %s"
                         % (npairs, r.shape))
    if len(f) != nf:
        raise ValueError("f must hold the nf=%d frequencies of the bins" % nf)
    indx = np.argsort(r)
    perm = np.ascontiguousarray(indx, dtype=np.int64)
    rs = np.ascontiguousarray(r[indx], dtype=np.float32)
    f32 = np.ascontiguousarray(f, dtype=np.float32)
    c32 = np.ascontiguousarray(c, dtype=np.float32)
    out = np.empty((len(c), nf), dtype=np.float32)
    fa = _lib.FjArgs()
    fa.struct_size = ctypes.sizeof(_lib.FjArgs)
    fa.nr, fa.nf, fa.nc = npairs, nf, len(c)
    fa.itype = int(itype)
    fa.mode = _lib.MODE_J if func == 0 else _lib.MODE_J_MINUS_Y
    fa.precision, fa.normalize, fa.device_ptrs = _lib.PREC_FP32, 1, 0
    fa.perm, fa.r, fa.f, fa.c = perm.ctypes.data, rs.ctypes.data, f32.ctypes.data, c32.ctypes.data
    fa.out = out.ctypes.data
    a.out_re = None
    _lib.check(_lib.load().ccfj_cc_fj_noise_v1(ctypes.byref(a), ctypes.byref(fa), None))
    del keep  # the records, pairs and ranges the call read
    return out
