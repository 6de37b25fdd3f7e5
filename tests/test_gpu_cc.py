"""Cross-correlation on the device (ccfj.CC, CrossCorrelation) against the
FP64 oracle (oracle/cc_oracle.py), on the cases the host replay of the same
kernels is checked on (tests/test_cc_emul.py)."""
import ctypes

import numpy as np
import pytest

import cc_oracle as C
from test_cc_emul import CASES, TOL, _case

pytestmark = pytest.mark.gpu


def _copy(args):
    return [np.copy(x) if isinstance(x, np.ndarray) else x for x in args]


@pytest.mark.parametrize("name", CASES)
def test_cc_matches_oracle(name):
    import ccfj
    args, kw = _case(name)
    got = ccfj.CC(*_copy(args), **kw)
    ref = C.CC(*_copy(args), **kw)
    assert got.dtype == np.complex64 and got.shape == ref.shape
    scale = np.abs(ref).max(axis=1, keepdims=True)
    zero = scale[:, 0] == 0
    assert np.all(got[zero] == 0)
    err = (np.abs(got - ref)[~zero] / scale[~zero]).max() if (~zero).any() else 0.0
    assert err <= TOL, err


def test_reference_entry_accumulates_and_rewrites_onebit(lib):
    """CrossCorrelation with the reference's CC_data: sums added to the
    caller's ncfsr / ncfsi before the division, pairs without a common
    window left as they were, and one-bit samples written back to data."""
    from ccfj import _cc
    args, kw = _case("tiles")
    npts, nsta, nf, fftlen, pairs, se, data = _copy(args)
    steplen = int(fftlen * (1 - kw["overlaprate"]))
    npairs = len(pairs) // 2
    rng = np.random.default_rng(3)
    re0 = rng.standard_normal((npairs, nf)).astype(np.float32)
    im0 = rng.standard_normal((npairs, nf)).astype(np.float32)
    re, im = re0.copy(), im0.copy()
    d = _cc.CcData()
    d.nsta, d.npts, d.nf, d.npairs = nsta, npts, nf, npairs
    d.fstride, d.fftlen, d.steplen = 1, fftlen, steplen
    d.Pairs, d.startend, d.data = pairs.ctypes.data, se.ctypes.data, data.ctypes.data
    d.ncfsr, d.ncfsi = re.ctypes.data, im.ctypes.data
    d.ifonebit, d.ifspecwhitenning, d.nThreads = 1, 1, 8
    signed = np.sign(data)
    assert lib.CrossCorrelation(d) == 0, lib.ccfj_last_error().decode()
    assert np.array_equal(data, signed)
    mean, counts = C.cross_correlation(signed.copy(), npts, nsta, nf, 1, fftlen, steplen,
                                       pairs, se, ifonebit=0)
    init = re0 + 1j * im0.astype(np.complex128)
    n = np.maximum(counts, 1)[:, None]
    expect = np.where(counts[:, None] > 0, init / n + mean, init)
    assert np.allclose(re + 1j * im, expect, rtol=0, atol=TOL * np.abs(expect).max())
    assert np.array_equal((re + 1j * im)[counts == 0], init[counts == 0].astype(np.complex64))


def test_cc_onebit_rewrites_the_callers_float32_array():
    import ccfj
    args, kw = _case("odd_window")
    npts, nsta, nf, fftlen, pairs, se, data = _copy(args)
    expect = C.CC(npts, nsta, nf, fftlen, pairs, se, np.sign(data), **kw)
    got = ccfj.CC(npts, nsta, nf, fftlen, pairs, se, data, ifonebit=1, **kw)
    assert np.array_equal(data, np.sign(args[6]))
    scale = np.abs(expect).max(axis=1, keepdims=True)
    assert (np.abs(got - expect) / scale).max() <= TOL
