"""ccfj -- CC-FJpy's frequency-Bessel (F-J) API over B200 CUDA kernels.

Drop-in for the F-J part of the reference's Python module (GPU build
src/ccfj-gpu.pyx:168-313, CPU build src/ccfj.pyx:148-268): the same
functions, argument meanings, return shapes and dtypes. The transform itself
runs in libccfj_b200.so (sm_100a); this module only validates and marshals
arrays, calls the C ABI with host pointers, and keeps the reference's
host-side conventions that decide bits of the answer:

* pair order is `np.argsort(r)` exactly as the reference calls it (the
  permutation is applied to the spectra on the device);
* inputs are read as float32 (a complex spectrum contributes its real part,
  with numpy's ComplexWarning), as `np.array(x, dtype=np.float32)` does;
* `fj_noise` / `fj_earthquake` return float32 [nc, nf]; `MWFJ` returns
  float64 [nwin, nc, nf];
* an unknown `func` prints the reference's message and returns 0.

`CC` (ambient-noise cross-correlation, src/CrossCorr.cpp) produces the
cross-spectra that fj_noise takes (ccfj/_cc.py).
"""
import ctypes
import os
import warnings

import numpy as np

from . import _lib
from ._lib import CcfjError  # noqa: F401

__all__ = ["fj_noise", "fj_earthquake", "MWFJ", "fj", "fhr", "fhi", "fh", "win",
           "GetStationPairs", "CC", "CcfjError", "fj_noise_batch", "fj_full", "fHr_full",
           "fHi_full", "fH_full", "CC_full"]

_FUNC_MSG = "set func as 0 for Bessel function 1 for Hankel function"


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _as_f32_vec(x):
    return np.ascontiguousarray(np.asarray(x), dtype=np.float32)


def _float_rows(uf):
    """Returns (float32 array, ld, es) describing the real part of the 2-D
    array `uf` element (i, j) at base[i*ld + j*es]: without a copy when the
    memory already holds float32 values (float32 rows, or interleaved
    complex64), else from a float32 copy."""
    uf = np.asarray(uf)
    if np.iscomplexobj(uf):
        warnings.warn("Casting complex values to real discards the imaginary part",
                      np.exceptions.ComplexWarning, stacklevel=4)
        if uf.dtype == np.complex64 and uf.strides[1] == 8 and uf.strides[0] > 0 \
                and uf.strides[0] % 4 == 0:
            return uf.real, uf.strides[0] // 4, 2
        uf = uf.real
    if uf.dtype == np.float32 and uf.strides[1] == 4 and uf.strides[0] > 0 \
            and uf.strides[0] % 4 == 0:
        return uf, uf.strides[0] // 4, 1
    c = np.ascontiguousarray(uf, dtype=np.float32)
    return c, c.shape[1], 1


def _transform(ufs, r, c, f, fstride, itype, mode, perm=None, hilbert=False, normalize=False,
               precision=_lib.PREC_FP32, cols=None):
    """Runs ccfj_fj_v1 on host arrays. `ufs` holds one or two 2-D spectra
    of the same shape whose rows are pairs; `r` is in pair order (sorted by
    the caller when perm is given: r[i] belongs to row perm[i]). `cols` =
    (a, b) computes only frequencies a .. b-1 of f (f, out cover those)."""
    lib = _lib.load()
    nr, nc, nf = len(r), len(c), len(f)
    a_col, b_col = (0, nf) if cols is None else cols
    u0 = np.asarray(ufs[0])
    if u0.ndim != 2:
        raise IndexError("too many indices for array: array is %d-dimensional, but 2 were indexed"
                         % u0.ndim)
    rows, ncols = u0.shape
    strided = len(range(0, ncols, fstride)) if fstride > 0 else 0
    if fstride <= 0:
        raise ValueError("slice step cannot be zero" if fstride == 0 else
                         "negative fstride is not supported")
    if rows * strided != nr * nf:
        raise ValueError("cannot reshape array of size %d into shape (%d,)"
                         % (rows * strided, nr * nf))
    if rows != nr or (perm is not None and rows < nr):
        # same element count but another row grouping: reproduce the
        # reference's flatten/reshape literally on a float32 copy
        flat = [np.ascontiguousarray(np.asarray(u)[:, ::fstride].real, dtype=np.float32)
                .reshape(nr, nf) for u in ufs]
        if perm is not None:
            flat = [x[perm] for x in flat]
        return _transform(flat, r, c, f, 1, itype, mode, None, hilbert, normalize, precision, cols)
    bases = [_float_rows(u) for u in ufs]
    r32, f32, c32 = _as_f32_vec(r), _as_f32_vec(np.asarray(f)[a_col:b_col]), _as_f32_vec(c)
    out = np.empty((nc, b_col - a_col), dtype=np.float32)
    a = _lib.FjArgs()
    a.struct_size = ctypes.sizeof(_lib.FjArgs)
    a.nr, a.nf, a.nc = nr, b_col - a_col, nc
    a.col_begin, a.nf_total = a_col, nf
    a.itype, a.mode, a.precision = int(itype), int(mode), int(precision)
    a.normalize = 1 if normalize else 0
    a.device_ptrs = 0
    a.hilbert = 1 if hilbert else 0
    a.u[0] = bases[0][0].ctypes.data
    a.u[1] = bases[1][0].ctypes.data if len(bases) > 1 else None
    ld, es = bases[0][1], bases[0][2]
    if len(bases) > 1 and (bases[1][1], bases[1][2]) != (ld, es):
        b1 = np.ascontiguousarray(bases[1][0], dtype=np.float32)
        b0 = np.ascontiguousarray(bases[0][0], dtype=np.float32)
        bases = [(b0, ncols, 1), (b1, ncols, 1)]
        a.u[0], a.u[1] = b0.ctypes.data, b1.ctypes.data
        ld, es = ncols, 1
    a.u_ld, a.u_es, a.u_ncols, a.u_rows, a.fstride = ld, es, ncols, rows, fstride
    perm64 = None
    if perm is not None:
        perm64 = np.ascontiguousarray(perm, dtype=np.int64)
        a.perm = perm64.ctypes.data
    a.r, a.f, a.c, a.out = r32.ctypes.data, f32.ctypes.data, c32.ctypes.data, out.ctypes.data
    _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), None))
    return out


def _itype_ok(itype):
    if itype in (0, 1):
        return True
    warnings.warn("itype=%r is neither 0 (trapezoid) nor 1 (linear integral); the reference "
                  "returns an all-zero transform for it" % (itype,), RuntimeWarning, stacklevel=3)
    return False


def _zeros_like_transform(uf, r, c, f, fstride):
    nr, nc, nf = len(r), len(c), len(f)
    u = np.asarray(uf)
    if u[:, ::fstride].size != nr * nf:
        raise ValueError("cannot reshape array of size %d into shape (%d,)"
                         % (u[:, ::fstride].size, nr * nf))
    return np.zeros((nc, nf), dtype=np.float32)


def _normalize_host(out):
    # only used for the all-zero result of an invalid itype: 0/0 -> NaN,
    # as the reference's normalisation of its zero output
    with np.errstate(invalid="ignore", divide="ignore"):
        for i in range(out.shape[1]):
            out[:, i] = out[:, i] / max(np.abs(out[:, i]))
    return out


# ------------------------------------------------------------- low level
def fj(uf, r, c, f, fstride=1, itype=1, nThread=None):
    """F-J transform with the Bessel basis (reference `fj`,
    src/ccfj-gpu.pyx:181-200 / src/ccfj.pyx:161-179). Rows of `uf` are in
    the order of `r` (no sorting here, as in the reference). nThread is the
    CPU build's OpenMP thread count and is ignored."""
    if not _itype_ok(itype):
        return _zeros_like_transform(uf, r, c, f, fstride)
    return _transform([uf], r, c, f, fstride, itype, _lib.MODE_J)


def fhr(uf, r, c, f, fstride=1, itype=1):
    """Real part of the Hankel-basis transform: the Bessel J basis
    (reference `fhr`, src/ccfj-gpu.pyx:202-219)."""
    if not _itype_ok(itype):
        return _zeros_like_transform(uf, r, c, f, fstride)
    return _transform([uf], r, c, f, fstride, itype, _lib.MODE_J)


def fhi(uf, r, c, f, fstride=1, itype=1):
    """Imaginary part of the Hankel-basis transform: the Bessel Y basis
    (reference `fhi`, src/ccfj-gpu.pyx:221-239)."""
    if not _itype_ok(itype):
        return _zeros_like_transform(uf, r, c, f, fstride)
    return _transform([uf], r, c, f, fstride, itype, _lib.MODE_Y)


def fh(uf, r, c, f, fstride=1, itype=1, nThread=None):
    """CPU build's name for the Y-basis transform (src/ccfj.pyx:181-198)."""
    return fhi(uf, r, c, f, fstride, itype)


# ------------------------------------------------------------ public API
def fj_noise(uf, r, c, f, fstride=1, itype=1, func=0, num=-1):
    """F-J dispersion spectrum of ambient-noise cross-spectra (reference
    `fj_noise`, src/ccfj-gpu.pyx:241-268).

    uf: [npairs, nf*fstride] spectra (real part used); r: [npairs] distances;
    c: [nc] phase velocities; f: [nf] frequencies; itype 1 = linear
    interpolation integral, 0 = trapezoid; func 0 = Bessel J basis,
    1 = Hankel (J(uf) - Y(hilbert(uf))). Returns float32 [nc, nf], each
    frequency column divided by its max |value|.
    """
    if num != -1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(int(num))
    r = np.asarray(r)
    indx = np.argsort(r)
    rs = r[indx]
    if func not in (0, 1):
        print(_FUNC_MSG)
        return 0
    if not _itype_ok(itype):
        return _normalize_host(_zeros_like_transform(uf, rs, c, f, fstride))
    if func == 0:
        return _transform([uf], rs, c, f, fstride, itype, _lib.MODE_J, perm=indx,
                          normalize=True)
    return _transform([uf], rs, c, f, fstride, itype, _lib.MODE_J_MINUS_Y, perm=indx,
                      hilbert=True, normalize=True)


def win(npts, Fs, T1, T2, taper=0.8):
    """Taper window (reference `win`, src/ccfj-gpu.pyx:168-178): zero outside
    [floor(T1 Fs), min(npts, floor(T2 Fs))), sine ramps of
    floor((n2-n1)(1-taper)/2) samples at both ends."""
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


def GetStationPairs(nsta):
    """Upper-triangle station pair list, int32 [2*npairs] (reference
    src/ccfj-gpu.pyx:137-144)."""
    ii, jj = np.triu_indices(nsta, k=1)
    return np.stack([ii, jj], axis=1).reshape(-1).astype(np.int32)



from ._eq import fj_earthquake, MWFJ  # noqa: E402
from ._batch import fj_noise_batch  # noqa: E402
from ._cc import CC, cc_fj_noise  # noqa: E402
from ._io import load_ncfs, pinned_empty  # noqa: E402
from ._pick import pick_curve  # noqa: E402
from ._shims import CC_full, fH_full, fHi_full, fHr_full, fj_full  # noqa: E402
from . import dist  # noqa: E402,F401
