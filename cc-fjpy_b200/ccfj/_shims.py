"""The reference module's low-level entry points (its cpdef shims), over the
same C ABI: fj_full, fHr_full, fHi_full (GPU build, src/ccfj-gpu.pyx:75-135),
fH_full (CPU build, src/ccfj.pyx:95-113) and CC_full (both builds,
src/ccfj.pyx:44-68). Each takes 1-D float32 (int32 for pairs and ranges)
buffers, as the reference's typed memoryviews do, and fills `out` (or
ncfsr / ncfsi) in place through the C entry the reference shim calls.

The reference hands C the address of element 0 of each memoryview, so a
strided view is read (and written) as if it were contiguous, past the
view's own elements. These shims reject a non-contiguous buffer with
ValueError instead.
"""
import ctypes

import numpy as np

from . import _cc, _lib

_fp = ctypes.POINTER(ctypes.c_float)


def _view(x, dtype, cname, name, writable=False):
    x = _cc._buffer_1d_checked(x, dtype, cname)
    if not x.flags.c_contiguous:
        raise ValueError("%s must be contiguous: the C entry reads it from its first element"
                         % name)
    if writable and not x.flags.writeable:
        raise ValueError("buffer source array is read-only")
    return x


def _fj_call(fn_name, U_f, r, f, out, c, nc, nr, nf, type_, extra=()):
    arrs = [_view(a, np.float32, "float", n, writable=(n == "out"))
            for a, n in ((U_f, "U_f"), (r, "r"), (f, "f"), (out, "out"), (c, "c"))]
    lib = _lib.load()
    ptrs = [a.ctypes.data_as(_fp) for a in arrs]
    _lib.check(getattr(lib, fn_name)(*ptrs, int(nc), int(nr), int(nf), int(type_), *extra))


def fj_full(U_f, r, f, out, c, nc, nr, nf, type, nThread=20):
    """FJ into out[nc*nf] (Bessel J basis; type 1 integral, 0 trapezoid).
    nThread (the CPU build's OpenMP count) is accepted and ignored."""
    _fj_call("FJ", U_f, r, f, out, c, nc, nr, nf, type)


def fHr_full(U_f, r, f, out, c, nc, nr, nf, type):
    """FHr into out[nc*nf] (the J basis, as the reference's FHr)."""
    _fj_call("FHr", U_f, r, f, out, c, nc, nr, nf, type)


def fHi_full(U_f, r, f, out, c, nc, nr, nf, type):
    """FHi into out[nc*nf] (the Y basis)."""
    _fj_call("FHi", U_f, r, f, out, c, nc, nr, nf, type)


def fH_full(U_f, r, f, out, c, nc, nr, nf, type, nThread=20):
    """The CPU build's FH (Y basis) into out[nc*nf]; nThread is ignored."""
    _fj_call("FH", U_f, r, f, out, c, nc, nr, nf, type, extra=(int(nThread),))


def CC_full(npts, nsta, nf, fstride, fftlen, steplen, ifonebit, ifspecwhitenning, nThreads,
            npairs, Pairs, startend, data, ncfsr, ncfsi):
    """CrossCorrelation with the reference's CC_data: sums accumulated into
    ncfsr / ncfsi [npairs*nf] and divided, data rewritten by one-bit."""
    pairs = _view(Pairs, np.int32, "int", "Pairs")
    se = _view(startend, np.int32, "int", "startend")
    d = _view(data, np.float32, "float", "data", writable=True)
    re = _view(ncfsr, np.float32, "float", "ncfsr", writable=True)
    im = _view(ncfsi, np.float32, "float", "ncfsi", writable=True)
    if len(pairs) < 2 * npairs or len(se) < 2 * nsta or d.size < nsta * npts \
            or re.size < npairs * nf or im.size < npairs * nf:
        raise ValueError("CC_full: a buffer is shorter than its sizes require")
    cd = _cc.CcData()
    cd.nsta, cd.npts, cd.nf, cd.npairs = int(nsta), int(npts), int(nf), int(npairs)
    cd.fstride, cd.fftlen, cd.steplen = int(fstride), int(fftlen), int(steplen)
    cd.Pairs, cd.startend, cd.data = pairs.ctypes.data, se.ctypes.data, d.ctypes.data
    cd.ncfsr, cd.ncfsi = re.ctypes.data, im.ctypes.data
    cd.ifonebit, cd.ifspecwhitenning, cd.nThreads = int(ifonebit), int(ifspecwhitenning), \
        int(nThreads)
    _lib.check(_lib.load().CrossCorrelation(cd))
