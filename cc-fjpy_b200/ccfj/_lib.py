"""ctypes binding of libccfj_b200.so (the C ABI declared in include/ccfj_b200.h).

The library is built in-tree by ccfj._build; loading fails loudly when it is
missing: there is no CPU implementation of the transform in this package.
"""
import ctypes
import os

from . import _build

CCFJ_OK = 0
CCFJ_ERR_INVALID = 1
CCFJ_ERR_CUDA = 2
CCFJ_ERR_ALLOC = 3
CCFJ_ERR_UNSUPPORTED = 4
CCFJ_ERR_TIMEOUT = 5

MODE_J, MODE_Y, MODE_J_MINUS_Y, MODE_ABS_J, MODE_ABS_H = 0, 1, 2, 3, 4
PREC_FP32, PREC_FP64, PREC_FP64_PLAIN = 0, 1, 2

_fp = ctypes.POINTER(ctypes.c_float)
_i64p = ctypes.POINTER(ctypes.c_longlong)


class FjArgs(ctypes.Structure):
    """Mirror of struct ccfj_fj_args (include/ccfj_b200.h)."""

    _fields_ = [
        ("struct_size", ctypes.c_int),
        ("nr", ctypes.c_int),
        ("nf", ctypes.c_int),
        ("nc", ctypes.c_int),
        ("itype", ctypes.c_int),
        ("mode", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("normalize", ctypes.c_int),
        ("device_ptrs", ctypes.c_int),
        ("hilbert", ctypes.c_int),
        ("u", ctypes.c_void_p * 2),
        ("u_ld", ctypes.c_longlong),
        ("u_rows", ctypes.c_longlong),
        ("u_es", ctypes.c_int),
        ("u_ncols", ctypes.c_int),
        ("fstride", ctypes.c_int),
        ("perm", ctypes.c_void_p),
        ("r", ctypes.c_void_p),
        ("f", ctypes.c_void_p),
        ("c", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("tau", ctypes.c_float),
        ("col_begin", ctypes.c_int),
        ("nf_total", ctypes.c_int),
    ]


# name -> (restype, argtypes) of every exported symbol
SIGNATURES = {
    "FJ": (ctypes.c_int, [_fp, _fp, _fp, _fp, _fp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int]),
    "FHr": (ctypes.c_int, [_fp, _fp, _fp, _fp, _fp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                           ctypes.c_int]),
    "FHi": (ctypes.c_int, [_fp, _fp, _fp, _fp, _fp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                           ctypes.c_int]),
    "FH": (ctypes.c_int, [_fp, _fp, _fp, _fp, _fp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, ctypes.c_int]),
    "ccfj_fj_v1": (ctypes.c_int, [ctypes.POINTER(FjArgs), ctypes.c_void_p]),
    "ccfj_fj_noalloc_v1": (ctypes.c_int, [ctypes.POINTER(FjArgs), ctypes.c_void_p]),
    "ccfj_autotune_fj_v1": (ctypes.c_int, [ctypes.POINTER(FjArgs), ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_float)]),
    "ccfj_set_fj_variant": (ctypes.c_int, [ctypes.c_int]),
    "ccfj_set_fj_split": (ctypes.c_int, [ctypes.c_int]),
    "ccfj_set_tune_cache": (ctypes.c_int, [ctypes.c_char_p]),
    "ccfj_tuned_choice_fj": (ctypes.c_int, [ctypes.POINTER(FjArgs), ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]),
    "ccfj_last_error": (ctypes.c_char_p, []),
    "ccfj_version": (ctypes.c_char_p, []),
    "ccfj_launch_count": (ctypes.c_longlong, []),
    "ccfj_set_allocator": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ccfj_profile_enable": (ctypes.c_int, [ctypes.c_int]),
    "ccfj_last_transform_ms": (ctypes.c_float, []),
    "ccfj_profile_total_ms": (ctypes.c_double, [ctypes.POINTER(ctypes.c_int)]),
    "ccfj_fp32_peak_probe": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
}

# the unit tests' probe library (include/ccfj_b200_probe.h)
PROBE_SIGNATURES = {
    "ccfj_special_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong,
                                         ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_double)]),
    "ccfj_special_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "ccfj_paired_probe": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]),
}

_LIB = None


def lib_path():
    return _build.LIB


def _bind(lib, signatures):
    for name, (res, args) in signatures.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def load():
    """Returns the loaded library, building it first if it is absent or was
    built from other sources than the ones in this tree."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.environ.get("CCFJ_LIB_PATH") or _build.LIB
    if path == _build.LIB:
        if not _build.up_to_date():
            _build.build()
    elif not os.path.exists(path):
        raise FileNotFoundError("CCFJ_LIB_PATH=%s does not exist" % path)
    _LIB = _bind(ctypes.CDLL(path), SIGNATURES)
    return _LIB


_PROBE = None


def load_probe():
    """The unit tests' special-function probe library (not the product)."""
    global _PROBE
    if _PROBE is None:
        if not _build.up_to_date(_build.PROBE_LIB, _build.probe_sources()):
            _build.build()
        _PROBE = _bind(ctypes.CDLL(_build.PROBE_LIB), PROBE_SIGNATURES)
    return _PROBE


class CcfjError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("ccfj_b200 error %d: %s" % (status, msg))
        self.status = status


def check(status):
    if status != CCFJ_OK:
        raise CcfjError(status, load().ccfj_last_error().decode())
    return status
