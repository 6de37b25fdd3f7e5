"""The C-ABI library: builds, loads, exports every declared symbol, and
rejects bad arguments before touching the device (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO


def declared_symbols(header="ccfj_b200.h", macro="CCFJ_API"):
    text = open(os.path.join(REPO, "include", header)).read()
    return re.findall(macro + r"\s+[\w\s\*]+?\b(\w+)\s*\(", text)


def test_header_declares_entry_points():
    syms = declared_symbols()
    for name in ("FJ", "FHr", "FHi", "FH", "ccfj_fj_v1", "ccfj_fj_earthquake_v1",
                 "ccfj_last_error", "ccfj_set_allocator", "ccfj_fj_noalloc_v1"):
        assert name in syms


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_probe_library_is_separate(lib, probe):
    """The special-function probes live in the test library only."""
    syms = declared_symbols("ccfj_b200_probe.h", "CCFJ_PROBE_API")
    assert set(syms) == {"ccfj_special_host", "ccfj_special_device", "ccfj_paired_probe"}
    for name in syms:
        assert hasattr(probe, name), name
    import subprocess
    from ccfj import _build
    dyn = subprocess.run(["nm", "-D", "--defined-only", _build.LIB], capture_output=True,
                         text=True).stdout
    assert "ccfj_special_host" not in dyn and "ccfj_special_device" not in dyn


def test_library_digest_matches_sources():
    """The loaded library was built from the sources in this tree."""
    from ccfj import _build
    assert _build.up_to_date()


def test_version(lib):
    assert b"sm_100a" in lib.ccfj_version()


def _args(**kw):
    from ccfj import _lib
    a = _lib.FjArgs()
    a.struct_size = ctypes.sizeof(_lib.FjArgs)
    a.nr, a.nf, a.nc = 4, 3, 2
    a.itype, a.mode, a.precision = 1, 0, 0
    a.u_ld, a.u_es, a.u_ncols, a.u_rows, a.fstride = 3, 1, 3, 4, 1
    buf = np.zeros(64, dtype=np.float32)
    a.u[0] = buf.ctypes.data
    a.r = a.f = a.c = a.out = buf.ctypes.data
    for k, v in kw.items():
        setattr(a, k, v)
    return a, buf


@pytest.mark.parametrize("field,value,needle", [
    ("struct_size", 8, "struct_size"),
    ("itype", 2, "itype"),
    ("mode", 9, "mode"),
    ("precision", 7, "precision"),
    ("nr", 0, "nr="),
    ("fstride", 0, "fstride"),
    ("u_ncols", 5, "frequencies"),
    ("u_rows", 2, "u_rows"),
])
def test_invalid_arguments_are_rejected(lib, field, value, needle):
    a, _buf = _args(**{field: value})
    st = lib.ccfj_fj_v1(ctypes.byref(a), None)
    assert st == 1  # CCFJ_ERR_INVALID
    assert needle in lib.ccfj_last_error().decode()


def test_two_input_mode_needs_second_input(lib):
    a, _buf = _args(mode=2)
    assert lib.ccfj_fj_v1(ctypes.byref(a), None) == 1
    assert "two inputs" in lib.ccfj_last_error().decode()


def test_compat_entry_rejects_bad_type(lib):
    fp = ctypes.POINTER(ctypes.c_float)
    b = np.zeros(16, dtype=np.float32)
    p = b.ctypes.data_as(fp)
    assert lib.FJ(p, p, p, p, p, 2, 2, 2, 5) == 1


def test_allocator_hook_validation(lib):
    cb = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p)(
        lambda n, s, u: None)
    assert lib.ccfj_set_allocator(ctypes.cast(cb, ctypes.c_void_p), None, None) == 1
    assert lib.ccfj_set_allocator(None, None, None) == 0


def test_earthquake_rejects_more_fft_rows_than_a_grid_holds(lib):
    """One FFT row (and CTA) per (window, trace): nwin * ntr above 2^31 - 1
    is rejected before any device work."""
    from ccfj import _eq
    a = _eq.EqArgs()
    a.struct_size = ctypes.sizeof(a)
    a.ntr, a.npts, a.nf, a.nc = 40000, 64, 8, 4
    a.itype, a.func, a.fstride, a.nwin = 1, 0, 1, 60000
    a.u_ld, a.u_rows = 64, 40000
    buf = np.zeros(64, dtype=np.float32)
    a.u = a.r = a.f = a.c = a.out = buf.ctypes.data
    a.win_n1 = a.win_n2 = a.win_delta = buf.ctypes.data
    assert lib.ccfj_fj_earthquake_v1(ctypes.byref(a), None) == 1
    assert "exceed 2^31-1" in lib.ccfj_last_error().decode()


@pytest.mark.parametrize("out_f64,device_ptrs,needle", [(2, 0, "out_f64 must be 0 or 1"),
                                                         (1, 1, "out_f64 needs host pointers")])
def test_earthquake_double_output_validation(lib, out_f64, device_ptrs, needle):
    """A double result (MWFJ's type) is converted while the library copies it
    out, so it exists for host pointers only."""
    from ccfj import _eq
    a = _eq.EqArgs()
    a.struct_size = ctypes.sizeof(a)
    a.ntr, a.npts, a.nf, a.nc = 4, 64, 8, 4
    a.itype, a.func, a.fstride, a.nwin = 1, 0, 1, 0
    a.u_ld, a.u_rows = 64, 4
    a.out_f64, a.device_ptrs = out_f64, device_ptrs
    buf = np.zeros(64, dtype=np.float32)
    a.u = a.r = a.f = a.c = a.out = buf.ctypes.data
    assert lib.ccfj_fj_earthquake_v1(ctypes.byref(a), None) == 1
    assert needle in lib.ccfj_last_error().decode()


def test_batch_autotuner_needs_device_pointers(lib):
    """ccfj_autotune_batch_v1 validates like the batch entry and times only
    device-resident batches (host-memory calls would time the copies)."""
    from ccfj import _batch
    a = _batch.BatchArgs()
    a.struct_size = ctypes.sizeof(a)
    a.nsets, a.nf, a.nc, a.itype, a.mode = 1, 4, 2, 1, 0
    buf = np.zeros(64, dtype=np.float32)
    offsets = np.array([0, 3], dtype=np.int64)
    a.offsets = offsets.ctypes.data
    a.r = a.f = a.c = a.out = buf.ctypes.data
    a.u[0] = buf.ctypes.data
    a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = 4, 3, 1, 4, 1
    best, ms = ctypes.c_int(), ctypes.c_float()
    assert lib.ccfj_autotune_batch_v1(ctypes.byref(a), None, ctypes.byref(best),
                                      ctypes.byref(ms)) == 1
    assert "device pointers" in lib.ccfj_last_error().decode()
    a.variant = 3
    assert lib.ccfj_autotune_batch_v1(ctypes.byref(a), None, ctypes.byref(best),
                                      ctypes.byref(ms)) == 1
    assert "variant" in lib.ccfj_last_error().decode()
