"""fj_noise over many subarrays in one persistent launch (ccfj_fj_batch_v1).

No counterpart in the reference, which is called once per subarray; the
result equals [fj_noise(uf_b, r_b, c, f, ...) for each subarray b].
"""
import ctypes
import warnings

import numpy as np

from . import _lib


class BatchArgs(ctypes.Structure):
    """Mirror of struct ccfj_batch_args (include/ccfj_b200.h)."""

    _fields_ = [
        ("struct_size", ctypes.c_int),
        ("nsets", ctypes.c_int),
        ("nf", ctypes.c_int),
        ("nc", ctypes.c_int),
        ("itype", ctypes.c_int),
        ("mode", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("normalize", ctypes.c_int),
        ("device_ptrs", ctypes.c_int),
        ("hilbert", ctypes.c_int),
        ("use_graph", ctypes.c_int),
        ("variant", ctypes.c_int),
        ("offsets", ctypes.c_void_p),
        ("total_pairs", ctypes.c_longlong),
        ("r", ctypes.c_void_p),
        ("u", ctypes.c_void_p * 2),
        ("u_ld", ctypes.c_longlong),
        ("u_rows", ctypes.c_longlong),
        ("u_es", ctypes.c_int),
        ("u_ncols", ctypes.c_int),
        ("fstride", ctypes.c_int),
        ("perm", ctypes.c_void_p),
        ("f", ctypes.c_void_p),
        ("c", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("tau", ctypes.c_float),
    ]


_lib.SIGNATURES["ccfj_fj_batch_v1"] = (ctypes.c_int, [ctypes.POINTER(BatchArgs), ctypes.c_void_p])
_lib.SIGNATURES["ccfj_batch_graph_cache_clear"] = (ctypes.c_int, [])
_lib.SIGNATURES["ccfj_autotune_batch_v1"] = (ctypes.c_int, [ctypes.POINTER(BatchArgs),
                                                             ctypes.c_void_p,
                                                             ctypes.POINTER(ctypes.c_int),
                                                             ctypes.POINTER(ctypes.c_float)])


def _consecutive_complex64(parts):
    """True when every part is a C-contiguous complex64 block that starts
    right where the previous one ends in memory."""
    if not all(p.dtype == np.complex64 and p.flags.c_contiguous for p in parts):
        return False
    return all(parts[b + 1].ctypes.data == parts[b].ctypes.data + parts[b].nbytes
               for b in range(len(parts) - 1))


def fj_noise_batch(ufs, rs, c, f, fstride=1, itype=1, func=0, variant=0):
    """fj_noise on every (uf_b, r_b) of the lists `ufs`, `rs` (shared c and
    f) in one launch. Each uf_b is [npairs_b, nf*fstride] (real part used).
    Returns a list of float32 [nc, nf] arrays, normalised per frequency."""
    if func not in (0, 1):
        raise ValueError("func must be 0 (Bessel) or 1 (Hankel), got %r" % (func,))
    if itype not in (0, 1):
        raise ValueError("itype must be 0 or 1, got %r" % (itype,))
    lib = _lib.load()
    nsets = len(ufs)
    if nsets == 0 or nsets != len(rs):
        raise ValueError("ufs and rs must be non-empty lists of the same length")
    nc, nf = len(c), len(f)
    counts = np.array([len(r) for r in rs], dtype=np.int64)
    if np.any(counts < 1):
        raise ValueError("every subarray needs at least one pair")
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    ncols = np.asarray(ufs[0]).shape[1]
    if len(range(0, ncols, fstride)) != nf:
        raise ValueError("cannot reshape array: %d columns with fstride %d do not give %d "
                         "frequencies" % (ncols, fstride, nf))
    perm = np.empty(offsets[-1], dtype=np.int64)
    rsorted = np.empty(offsets[-1], dtype=np.float32)
    for b, r in enumerate(rs):
        r = np.asarray(r)
        indx = np.argsort(r)
        perm[offsets[b]:offsets[b + 1]] = offsets[b] + indx
        rsorted[offsets[b]:offsets[b + 1]] = r[indx]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", np.exceptions.ComplexWarning)
        parts = [np.asarray(u) for u in ufs]
        for b, p in enumerate(parts):
            if p.ndim != 2 or p.shape[0] != counts[b] or p.shape[1] != ncols:
                raise ValueError("every uf_b must be [len(r_b), %d]" % ncols)
        if _consecutive_complex64(parts):
            # the subarrays are consecutive rows of one complex64 array (for
            # example views of a pinned buffer): read them in place
            U = parts
            base_ptr, ld, es = parts[0].ctypes.data, 2 * ncols, 2
        elif all(p.dtype == np.complex64 for p in parts):
            U = np.concatenate(parts, axis=0)
            base_ptr, ld, es = U.ctypes.data, 2 * ncols, 2
        else:
            U = np.concatenate([np.real(p).astype(np.float32) for p in parts], axis=0)
            base_ptr, ld, es = U.ctypes.data, ncols, 1
    f32 = np.ascontiguousarray(f, dtype=np.float32)
    c32 = np.ascontiguousarray(c, dtype=np.float32)
    out = np.empty((nsets, nc, nf), dtype=np.float32)
    a = BatchArgs()
    a.struct_size = ctypes.sizeof(BatchArgs)
    a.nsets, a.nf, a.nc = nsets, nf, nc
    a.itype = int(itype)
    a.mode = _lib.MODE_J if func == 0 else _lib.MODE_J_MINUS_Y
    a.precision, a.normalize, a.device_ptrs = _lib.PREC_FP32, 1, 0
    a.hilbert = 1 if func == 1 else 0
    a.use_graph, a.variant = 0, int(variant)
    a.offsets, a.total_pairs = offsets.ctypes.data, int(offsets[-1])
    a.r = rsorted.ctypes.data
    a.u[0] = base_ptr
    a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = ld, int(offsets[-1]), es, ncols, fstride
    a.perm = perm.ctypes.data
    a.f, a.c, a.out = f32.ctypes.data, c32.ctypes.data, out.ctypes.data
    _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(a), None))
    return [out[b] for b in range(nsets)]
