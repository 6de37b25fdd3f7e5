"""Dispersion-curve picking on the device (ccfj_pick_v1): for every
frequency, the phase velocity of the spectrum's largest value inside a
velocity band, refined between grid velocities. No counterpart in the
reference, whose users pick the curves from the plotted spectrum."""
import ctypes

import numpy as np

from . import _lib

_lib.SIGNATURES["ccfj_pick_v1"] = (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_int,
                                                   ctypes.c_void_p])


def _band(v, nf, name):
    if v is None:
        return None
    b = np.broadcast_to(np.asarray(v, dtype=np.float32), (nf,))
    if not np.all(np.isfinite(b) | np.isinf(b)):
        raise ValueError("%s holds NaN" % name)
    return np.ascontiguousarray(b)


def pick_curve(spec, c, cmin=None, cmax=None):
    """spec: [nc, nf] spectrum (e.g. fj_noise's output), c: [nc] velocities,
    cmin / cmax: scalars or [nf] arrays bounding the search per frequency.
    Returns (c_pick [nf], amplitude [nf]) as float32; NaN where a column
    holds NaN in the band or the band holds no velocity."""
    spec = np.ascontiguousarray(spec, dtype=np.float32)
    if spec.ndim != 2:
        raise ValueError("spec must be [nc, nf]")
    nc, nf = spec.shape
    c32 = np.ascontiguousarray(c, dtype=np.float32)
    if c32.shape != (nc,):
        raise ValueError("c must hold the %d velocities of spec's rows" % nc)
    lo, hi = _band(cmin, nf, "cmin"), _band(cmax, nf, "cmax")
    cp = np.empty(nf, dtype=np.float32)
    amp = np.empty(nf, dtype=np.float32)
    _lib.check(_lib.load().ccfj_pick_v1(spec.ctypes.data, nc, nf, c32.ctypes.data,
                                        lo.ctypes.data if lo is not None else None,
                                        hi.ctypes.data if hi is not None else None,
                                        cp.ctypes.data, amp.ctypes.data, 0, None))
    return cp, amp
