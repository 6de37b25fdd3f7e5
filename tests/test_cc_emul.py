"""The cross-correlation path without a GPU: its plan (cc_plan.h) and
per-thread arithmetic (cc_core.cuh), replayed on the host in the kernels'
loop structure by tests/cc_emul.cpp, against numpy's rfft and the FP64
oracle (oracle/cc_oracle.py); the Python wrapper's argument handling; and
the library's argument errors, which it returns before any device work."""
import ctypes
import os
import shutil
import subprocess
import zlib

import numpy as np
import pytest

import cc_oracle as C
from conftest import REPO

CSRC = os.path.join(REPO, "cc-fjpy_b200", "csrc")
# FP32 FFT and accumulation against the FP64 oracle, relative to each
# pair's largest value
TOL = 2e-5


def _pairs(nsta):
    from ccfj import GetStationPairs
    return GetStationPairs(nsta)


def _emul_cc(emul, *args, **kw):
    """ccfj.CC's marshalling with the host replay in place of the library."""
    from ccfj import _cc
    a, _keep, out = _cc._prepare(*args, **kw)
    st = emul.cc_emul_v1(ctypes.byref(a))
    assert st == 0, emul.cc_emul_error().decode()
    return out


def _records(rng, nsta, npts):
    return rng.standard_normal(nsta * npts).astype(np.float32)


def test_fft_plan(emul):
    radix = (ctypes.c_int * 24)()
    for M in (2, 3, 4, 5, 8, 12, 30, 64, 90, 360, 1800, 3600, 7200, 8192, 6000, 3125, 2187):
        n = emul.cc_emul_fft_plan(M, radix)
        rs = list(radix[:n])
        assert n > 0 and np.prod(rs) == M and set(rs) <= {2, 3, 4, 5, 8}, (M, rs)
        # the kernel's order: 8s, at most one 4 or 2, then 3s, then 5s
        order = [{8: 0, 4: 1, 2: 1, 3: 2, 5: 3}[r] for r in rs]
        assert order == sorted(order) and sum(r in (2, 4) for r in rs) <= 1
    for M in (1, 7, 14, 49, 2 * 17, 11 * 8):
        assert emul.cc_emul_fft_plan(M, radix) == 0


def test_shift_range_matches_the_window_rule(emul):
    rng = np.random.default_rng(1)
    lo, hi = ctypes.c_longlong(), ctypes.c_longlong()
    for _ in range(3000):
        npts = int(rng.integers(1, 400))
        fftlen = int(rng.integers(1, 450))
        steplen = int(rng.integers(1, 60))
        F, nshifts = C.cc_shifts(npts, fftlen, steplen)
        start = int(rng.integers(-50, npts + 20))
        end = int(rng.integers(-50, npts + 60))
        se = [start, end]
        kept = [k for k in range(nshifts) if C.cc_active(k, steplen, F, se, 0)]
        emul.cc_emul_shift_range(nshifts, steplen, F, start, end, ctypes.byref(lo),
                                 ctypes.byref(hi))
        assert list(range(lo.value, hi.value + 1)) == kept, (npts, fftlen, steplen, start, end)


@pytest.mark.parametrize("F,path", [(16, 1), (24, 1), (60, 1), (128, 1), (250, 1), (360, 1),
                                    (1000, 1), (2048, 1), (3600, 1), (14400, 1), (16384, 1),
                                    (15, 0), (101, 0), (98, 0), (224, 0), (16390, 0),
                                    (20000, 0)])
def test_window_spectra_match_numpy(emul, F, path):
    """Stockham path (1) for even lengths up to 16384 whose half has no
    prime factor above 5, the direct transform (0) otherwise."""
    from ccfj import _cc
    rng = np.random.default_rng(F)
    nsta, nf, fstride = 2, min(F // 2 + 1, 300), 1
    if F > 4000:
        fstride = (F // 2) // (nf - 1)
    data = _records(rng, nsta, F)
    se = np.array([0, F + 1] * nsta, dtype=np.int32)
    a, _keep, _out = _cc._prepare(F, nsta, nf, F, _pairs(nsta), se, data, fstride=fstride,
                                  ifspecwhittenning=0)
    ldj, nsh, stock = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_int()
    assert emul.cc_emul_spectra(ctypes.byref(a), None, ctypes.byref(ldj), ctypes.byref(nsh),
                                ctypes.byref(stock)) == 0
    assert stock.value == path and nsh.value == 1
    X = np.zeros(nsh.value * nsta * ldj.value * 2, dtype=np.float32)
    assert emul.cc_emul_spectra(ctypes.byref(a), X.ctypes.data, ctypes.byref(ldj),
                                ctypes.byref(nsh), ctypes.byref(stock)) == 0
    X = X.view(np.complex64).reshape(nsh.value, nsta, ldj.value)[0, :, :nf]
    ref = np.fft.rfft(data.astype(np.float64).reshape(nsta, F), axis=1)[:, ::fstride][:, :nf]
    err = np.abs(X - ref).max() / np.abs(ref).max()
    assert err <= 1e-5, err


def _case(name):
    """(args of CC, kwargs): seeded records with the reference example's
    shapes scaled down."""
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "tiles":           # 40 stations: three station tiles, ragged
        nsta, npts, fftlen = 40, 3000, 400
        se = np.tile([0, npts], nsta).astype(np.int32)
        se[2 * 5:2 * 5 + 2] = [700, 2600]       # part of the record
        se[2 * 17:2 * 17 + 2] = [0, 300]        # keeps no window
        se[2 * 33:2 * 33 + 2] = [1200, 3100]
        return (npts, nsta, 64, fftlen, _pairs(nsta), se, _records(rng, nsta, npts)), \
            dict(overlaprate=0.5)
    if name == "onebit_plain_fstride":
        nsta, npts, fftlen = 6, 2400, 360
        se = np.tile([0, npts + 1], nsta).astype(np.int32)
        return (npts, nsta, 40, fftlen, _pairs(nsta), se, _records(rng, nsta, npts)), \
            dict(overlaprate=0.75, fstride=4, ifonebit=1, ifspecwhittenning=0)
    if name == "odd_window":      # 401 samples: the direct transform
        nsta, npts, fftlen = 5, 2000, 401
        se = np.tile([0, npts], nsta).astype(np.int32)
        return (npts, nsta, 50, fftlen, _pairs(nsta), se, _records(rng, nsta, npts)), \
            dict(overlaprate=0.3)
    if name == "factor7":         # 224 = 2 * 112, 112 = 16 * 7: direct
        nsta, npts, fftlen = 4, 1500, 224
        se = np.tile([0, npts], nsta).astype(np.int32)
        return (npts, nsta, 30, fftlen, _pairs(nsta), se, _records(rng, nsta, npts)), \
            dict(overlaprate=0.5, ifspecwhittenning=0)
    if name == "one_window":      # fftlen >= npts
        nsta, npts = 7, 600
        se = np.tile([0, npts + 1], nsta).astype(np.int32)
        se[2 * 3 + 1] = npts                     # ends at npts: never kept
        return (npts, nsta, 100, 5000, _pairs(nsta), se, _records(rng, nsta, npts)), dict()
    if name == "pair_list":       # reversed, self, repeated, cross-tile pairs
        nsta, npts, fftlen = 36, 1200, 200
        se = np.tile([0, npts], nsta).astype(np.int32)
        se[2 * 30:2 * 30 + 2] = [500, 1200]
        pairs = np.array([3, 35, 35, 3, 7, 7, 3, 35, 0, 1, 30, 2, 17, 16, 34, 0, 3, 35],
                         dtype=np.int32)
        return (npts, nsta, 48, fftlen, pairs, se, _records(rng, nsta, npts)), \
            dict(overlaprate=0.6, ifspecwhittenning=0)
    if name == "example_shape":   # the reference example at 1/8 of the samples
        nsta, Fs = 12, 4
        npts, fftlen = 86400 * Fs // 8, 3600 * Fs // 2
        se = np.tile([0, npts], nsta).astype(np.int32)
        return (npts, nsta, 250, fftlen, _pairs(nsta), se, _records(rng, nsta, npts)), \
            dict(overlaprate=0.9, fstride=3)
    raise KeyError(name)


CASES = ["tiles", "onebit_plain_fstride", "odd_window", "factor7", "one_window", "pair_list",
         "example_shape"]


@pytest.mark.parametrize("name", CASES)
def test_replay_matches_oracle(emul, name):
    args, kw = _case(name)
    got = _emul_cc(emul, *[np.copy(x) if isinstance(x, np.ndarray) else x for x in args], **kw)
    ref = C.CC(*[np.copy(x) if isinstance(x, np.ndarray) else x for x in args], **kw)
    assert got.dtype == np.complex64 and got.shape == ref.shape
    scale = np.abs(ref).max(axis=1, keepdims=True)
    zero = scale[:, 0] == 0
    assert np.all(got[zero] == 0)            # pairs with no common window
    err = (np.abs(got - ref)[~zero] / scale[~zero]).max() if (~zero).any() else 0.0
    assert err <= TOL, err


def test_accumulate_semantics_of_the_reference_entry(emul):
    """accumulate = 1, separate planes (the reference's CrossCorrelation):
    (initial + sum) / count where the pair has common windows, the initial
    values untouched where it has none."""
    from ccfj import _cc
    args, kw = _case("tiles")
    npts, nsta, nf, fftlen, pairs, se, data = args
    a, _keep, _out = _cc._prepare(*args, **kw)
    rng = np.random.default_rng(3)
    npairs = len(pairs) // 2
    re0 = rng.standard_normal((npairs, nf)).astype(np.float32)
    im0 = rng.standard_normal((npairs, nf)).astype(np.float32)
    re, im = re0.copy(), im0.copy()
    a.accumulate, a.out_layout = 1, 0
    a.out_re, a.out_im = re.ctypes.data, im.ctypes.data
    assert emul.cc_emul_v1(ctypes.byref(a)) == 0
    mean, counts = C.cross_correlation(data.copy(), npts, nsta, nf, 1, fftlen,
                                       int(fftlen * (1 - kw["overlaprate"])), pairs, se)
    init = re0 + 1j * im0.astype(np.complex128)
    n = np.maximum(counts, 1)[:, None]
    expect = np.where(counts[:, None] > 0, init / n + mean, init)
    assert (counts == 0).any() and (counts > 0).any()
    assert np.allclose(re + 1j * im, expect, rtol=0, atol=TOL * np.abs(expect).max())


def test_onebit_plumbing_uses_the_callers_float32_array():
    """The library rewrites the samples it is given; _prepare hands it the
    caller's own float32 array (as the reference's wrapper does) and a copy
    of any other dtype."""
    from ccfj import _cc
    se = np.array([0, 100, 0, 100], dtype=np.int32)
    d32 = np.ones(200, dtype=np.float32)
    a, keep, _ = _cc._prepare(100, 2, 5, 50, _pairs(2), se, d32, ifonebit=1)
    assert a.data == d32.ctypes.data
    d64 = np.ones(200)
    a, keep, _ = _cc._prepare(100, 2, 5, 50, _pairs(2), se, d64, ifonebit=1)
    assert a.data != d64.ctypes.data and keep[2].dtype == np.float32


def test_wrapper_argument_errors():
    import ccfj
    se = np.array([0, 100, 0, 100], dtype=np.int32)
    d = np.zeros(200, dtype=np.float32)
    with pytest.raises(ValueError, match="Buffer dtype mismatch, expected 'int' but got 'long'"):
        ccfj.CC(100, 2, 5, 50, ccfj.GetStationPairs(2).astype(np.int64), se, d)
    with pytest.raises(ValueError, match="wrong number of dimensions"):
        ccfj.CC(100, 2, 5, 50, ccfj.GetStationPairs(2), se, d.reshape(2, 100))
    with pytest.raises(ValueError, match="data holds 150 samples"):
        ccfj.CC(100, 2, 5, 50, ccfj.GetStationPairs(2), se, d[:150])
    with pytest.raises(TypeError):
        ccfj.CC(100, 2, 5, 50, [0, 1], se, d)


@pytest.mark.parametrize("field,value,needle", [
    ("nf", 27, "past the last real-FFT bin"),     # bins 0..25 of a 50-sample window
    ("steplen", 0, "steplen=0"),
    ("nsta", 0, "nsta=0"),
    ("fstride", 0, "fstride=0"),
    ("out_layout", 3, "out_layout"),
    ("struct_size", 8, "struct_size"),
])
def test_library_rejects_bad_plans(lib, field, value, needle):
    from ccfj import _cc
    se = np.array([0, 100, 0, 100], dtype=np.int32)
    d = np.zeros(200, dtype=np.float32)
    a, _keep, _out = _cc._prepare(100, 2, 5, 50, _pairs(2), se, d)
    setattr(a, field, value)
    assert lib.ccfj_cc_v1(ctypes.byref(a), None) == 1
    assert needle in lib.ccfj_last_error().decode()


def test_library_rejects_pairs_outside_the_stations(lib):
    from ccfj import _cc
    se = np.array([0, 100, 0, 100], dtype=np.int32)
    d = np.zeros(200, dtype=np.float32)
    a, _keep, _out = _cc._prepare(100, 2, 5, 50, np.array([0, 2], dtype=np.int32), se, d)
    assert lib.ccfj_cc_v1(ctypes.byref(a), None) == 1
    assert "outside 0..1" in lib.ccfj_last_error().decode()


def _smooth(m):
    """No prime factor above 5: 2m is a length the shared-memory FFT takes."""
    for p in (2, 3, 5):
        while m % p == 0:
            m //= p
    return m == 1


def _fuzz_case(seed):
    rng = np.random.default_rng(1000 + seed)
    nsta = int(rng.integers(2, 40))
    npts = int(rng.integers(64, 1500))
    if rng.random() < 0.6:   # the Stockham path
        lens = [2 * m for m in range(2, (npts + 50) // 2 + 1) if _smooth(m)]
        fftlen = int(rng.choice(lens))
    else:                    # any length: mostly the direct transform
        fftlen = int(rng.integers(8, npts + 50))
    overlap = float(rng.choice([0.0, 0.25, 0.5, 0.75, 0.9]))
    if fftlen < npts and int(fftlen * (1 - overlap)) < 1:
        overlap = 0.0
    F = min(fftlen, npts)
    fstride = int(rng.integers(1, 4))
    nf = int(rng.integers(1, (F // 2) // fstride + 2))
    se = np.empty(2 * nsta, dtype=np.int32)   # most records cover most of the day
    se[0::2] = rng.integers(-20, npts // 4 + 1, nsta)
    se[1::2] = se[0::2] + rng.integers(npts // 2, npts + 40, nsta)
    npairs = int(rng.integers(1, 3 * nsta))
    pairs = rng.integers(0, nsta, 2 * npairs).astype(np.int32)
    kw = dict(overlaprate=overlap, fstride=fstride, ifonebit=int(rng.integers(0, 2)),
              ifspecwhittenning=int(rng.integers(0, 2)))
    return (npts, nsta, nf, fftlen, pairs, se, _records(rng, nsta, npts)), kw


def _fuzz_bounds(args, kw):
    """Per (pair, bin): the scale of the sum's terms -- the mean over the
    pair's common windows of |X_a| |X_b| (after one-bit and whitening), an
    upper bound of the result that does not shrink when the terms cancel --
    and the cells that cannot be checked: with whitening, a window whose
    spectral value is within 1e-3 sqrt(F) of zero (one-bit samples give exact
    zeros), which FP32 and FP64 normalise to unrelated phases."""
    npts, nsta, nf, fftlen, pairs, se, data = args
    steplen = int(fftlen * (1 - kw.get("overlaprate", 0.0)))
    F, nsh = C.cc_shifts(npts, fftlen, steplen)
    fstride, whiten = kw.get("fstride", 1), kw.get("ifspecwhittenning", 1)
    x = data.astype(np.float64).reshape(nsta, npts)
    if kw.get("ifonebit"):
        x = np.sign(x)
    mag = np.zeros((nsh, nsta, nf))
    kept = np.zeros((nsh, nsta), dtype=bool)
    small = np.zeros((nsta, nf), dtype=bool)
    for i in range(nsta):
        for k in range(nsh):
            if C.cc_active(k, steplen, F, se, i):
                X = np.abs(np.fft.rfft(x[i, k * steplen:k * steplen + F])[::fstride][:nf])
                kept[k, i] = True
                small[i] |= X < 1e-3 * np.sqrt(F)
                mag[k, i] = np.minimum(X / np.maximum(X, 1e-8), 1.0) if whiten else X
    # bin 0 and (even F) bin F/2 are sums of the samples with signs, exact in
    # FP32 for one-bit samples: their zeros are zeros on both sides
    b = np.arange(nf) * fstride
    small &= ~((b == 0) | ((F % 2 == 0) & (b == F // 2)))[None, :]
    pr = np.asarray(pairs)[:2 * (len(pairs) // 2)].reshape(-1, 2)
    both = kept[:, pr[:, 0]] & kept[:, pr[:, 1]]                  # [nsh, npairs]
    terms = (mag[:, pr[:, 0]] * mag[:, pr[:, 1]]) * both[:, :, None]
    scale = terms.sum(axis=0) / np.maximum(both.sum(axis=0), 1)[:, None]
    skip = (small[pr[:, 0]] | small[pr[:, 1]]) if whiten else np.zeros_like(scale, dtype=bool)
    return scale.max(axis=1, keepdims=True), skip


@pytest.mark.parametrize("seed", range(40))
def test_replay_matches_oracle_fuzz(emul, seed):
    """Random window lengths (both transforms), steps, ragged valid ranges,
    pair lists with repeats, reversals and self-pairs, fstride, one-bit and
    whitening: FP32 error within TOL of each pair's term scale."""
    args, kw = _fuzz_case(seed)
    got = _emul_cc(emul, *[np.copy(x) if isinstance(x, np.ndarray) else x for x in args], **kw)
    ref = C.CC(*[np.copy(x) if isinstance(x, np.ndarray) else x for x in args], **kw)
    scale, skip = _fuzz_bounds(args, kw)
    none = scale[:, 0] == 0                    # no common window
    assert np.all(got[none] == 0) and np.all(ref[none] == 0)
    err = np.abs(got - ref) / np.where(scale > 0, scale, 1.0)
    assert skip.mean() < 0.5                   # most cells are checked
    assert err[~skip].max() <= TOL, (err[~skip].max(), kw)


def test_calls_without_output_touch_no_device(lib):
    """No pairs (or no bins): the library returns at once -- after one-bit
    has rewritten the caller's samples, as the reference's loop does before
    anything else -- so this runs without a GPU."""
    import ccfj
    se = np.array([0, 100, 0, 100], dtype=np.int32)
    d = np.array(np.linspace(-1, 1, 200), dtype=np.float32)
    out = ccfj.CC(100, 2, 5, 50, np.zeros(0, dtype=np.int32), se, d, ifonebit=1)
    assert out.shape == (0, 5) and out.dtype == np.complex64
    assert np.array_equal(d, np.sign(np.linspace(-1, 1, 200)).astype(np.float32))
    out = ccfj.CC(100, 2, 0, 50, ccfj.GetStationPairs(2), se, d)
    assert out.shape == (1, 0)
