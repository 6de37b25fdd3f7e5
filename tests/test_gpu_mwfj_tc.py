"""MWFJ's window contraction on the tensor cores (tcgen05, scaled FP16x3) against
the CUDA-core path and the FP64 oracle."""
import ctypes
import warnings

import numpy as np
import pytest

import cases
import fj_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _case(seed, ntr, nwin, npts=256, Fs=10.0, nf=24, nc=33):
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(np.log(5e3), np.log(1.5e5), ntr))
    u = cases.ricker_records(rng, r, npts, Fs)
    L = rng.integers(40, 200, size=(nwin, ntr))
    start = rng.integers(0, npts - L)
    f = Fs * np.arange(nf) / npts
    c = np.linspace(1500, 5000, nc)
    return u, r, c, f, Fs, nwin, start / Fs, (start + L) / Fs


def _run(path, case, **kw):
    import ccfj
    from ccfj import _lib
    lib = _lib.load()
    assert lib.ccfj_set_mwfj_path(path) == 0
    try:
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            return ccfj.MWFJ(*case, taper=0.9, **kw)
    finally:
        lib.ccfj_set_mwfj_path(0)


@pytest.mark.parametrize("ntr,nwin,nc", [(14, 10, 33), (70, 64, 300), (40, 8, 257)])
def test_tensor_path_matches_cuda_core_and_oracle(ntr, nwin, nc):
    case = _case(51 + ntr, ntr, nwin, nc=nc)
    y_tc = _run(2, case)
    y_cc = _run(1, case)
    assert np.isfinite(y_tc[:, :, 1:]).all()
    for w in range(nwin):
        assert O.rel_error(y_tc[w], y_cc[w]) <= TOL
    # the oracle on a few windows
    u, r, c, f, Fs, nw, winl, winr = case
    for w in sorted({0, nwin // 2, nwin - 1}):
        y64 = O.MWFJ(u, r, c, f, Fs, 1, winl[w:w + 1], winr[w:w + 1], taper=0.9,
                     normalize=False)[0]
        assert O.rel_error(y_tc[w], O._normalize(y64)) <= TOL


@pytest.mark.parametrize("ntr,nwin,nc", [(70, 64, 300), (41, 8, 257)])
def test_paired_generator_agrees_with_one_interval_at_a_time(ntr, nwin, nc):
    """The A operand formed with paired FP32 instructions (two stations per
    instruction where both have x >= 8; an odd pair count leaves a last
    interval alone) against the one-interval-at-a-time generator (path 3):
    the same arithmetic up to rounding."""
    case = _case(91 + ntr, ntr, nwin, nc=nc)
    y2 = _run(2, case)
    y3 = _run(3, case)
    assert np.array_equal(np.isnan(y2), np.isnan(y3))
    for w in range(nwin):
        assert O.rel_error(y2[w], y3[w]) <= 1e-5


def test_tensor_path_f0_column_is_nan():
    case = _case(77, 20, 16)
    y = _run(2, case)
    assert np.isnan(y[:, :, 0]).all()  # k = 0, as the reference


def test_device_status_ok(lib):
    from ccfj import _lib
    assert lib.ccfj_device_status(None) == 0
