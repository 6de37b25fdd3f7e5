"""Failure paths that leave the device usable: a device-side bounded wait
that runs out (the tensor-core kernel's self-test), and a device allocation
that fails (injected through the allocator hook). Neither faults, traps or
hangs the GPU."""
import ctypes
import warnings

import numpy as np
import pytest

import cases
import fj_oracle as O

pytestmark = pytest.mark.gpu


def _small_noise(ccfj):
    case = cases.noise_case("noise_small")
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        y = ccfj.fj_noise(case["uf"], case["r"], case["c"], case["f"])
    assert O.rel_error(y, O.fj_noise(case["uf"], case["r"], case["c"], case["f"])) <= 1e-4


def test_bounded_wait_times_out_and_device_stays_usable(lib):
    import ccfj
    assert lib.ccfj_self_test_wait_timeout(None) == 0, lib.ccfj_last_error()
    assert lib.ccfj_device_status(None) == 0  # the flag was cleared
    _small_noise(ccfj)


def test_failed_allocation_is_reported(lib):
    import ccfj
    from ccfj import _lib
    ALLOC = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p)
    FREE = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)
    calls = []

    def refuse(n, stream, user):
        calls.append(n)
        return None

    alloc, free = ALLOC(refuse), FREE(lambda p, s, u: None)
    assert lib.ccfj_set_allocator(ctypes.cast(alloc, ctypes.c_void_p),
                                  ctypes.cast(free, ctypes.c_void_p), None) == 0
    try:
        case = cases.noise_case("noise_small")
        with pytest.raises(_lib.CcfjError) as e, warnings.catch_warnings():
            warnings.simplefilter("ignore")
            ccfj.fj_noise(case["uf"], case["r"], case["c"], case["f"])
        assert e.value.status == _lib.CCFJ_ERR_ALLOC
        assert calls
    finally:
        assert lib.ccfj_set_allocator(None, None, None) == 0
    _small_noise(ccfj)
