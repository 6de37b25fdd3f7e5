"""The cross-correlation oracle (oracle/cc_oracle.py) against properties
that follow from the reference's CrossCorrelation (src/CrossCorr.cpp:33-159)
and CC wrapper (src/ccfj.pyx:125-147). FFTW is absent here, so the
reference's cross-correlator cannot be built or run; these checks use
hand-counted windows and closed-form spectra instead. No GPU."""
import numpy as np
import pytest

import cc_oracle as C


def _pairs(nsta):
    return np.array([(a, b) for a in range(nsta) for b in range(a + 1, nsta)],
                    dtype=np.int32).reshape(-1)


def test_shift_count():
    assert C.cc_shifts(1000, 100, 50) == (100, 19)
    assert C.cc_shifts(100, 200, 0) == (100, 1)         # fftlen >= npts: one shift
    assert C.cc_shifts(100, 100, 7) == (100, 1)
    # one day at 4 Hz, one-hour windows, 90 % overlap: the wrapper's
    # steplen is int(14400 * (1 - 0.9)) = 1439, not 1440
    steplen = int(14400 * (1 - 0.9))
    assert steplen == 1439
    assert C.cc_shifts(345600, 14400, steplen) == (14400, 231)
    with pytest.raises(ValueError):
        C.cc_shifts(1000, 100, 0)


def test_window_rule_counts():
    """npts 1000, windows of 100 every 50 samples (starts 0..900). A
    station valid over [0, 1000) misses the last window, which ends exactly
    at 1000 (the end test is strict): shifts 0-17. [120, 500) gives shifts
    3-7. [0, 100) gives none."""
    npts, fftlen, steplen = 1000, 100, 50
    rng = np.random.default_rng(1)
    data = rng.standard_normal(3 * npts).astype(np.float32)
    startend = np.array([0, 1000, 120, 500, 0, 100], dtype=np.int32)
    assert [k for k in range(19) if C.cc_active(k, steplen, fftlen, startend, 0)] == \
        list(range(18))
    assert [k for k in range(19) if C.cc_active(k, steplen, fftlen, startend, 1)] == \
        list(range(3, 8))
    assert not any(C.cc_active(k, steplen, fftlen, startend, 2) for k in range(19))
    ncfs, counts = C.cross_correlation(data, npts, 3, 20, 1, fftlen, steplen, _pairs(3),
                                       startend)
    assert counts.tolist() == [5, 0, 0]                 # pairs (0,1), (0,2), (1,2)
    assert np.all(ncfs[1:] == 0) and np.all(ncfs[0] != 0)


def test_single_window_is_the_cross_spectrum():
    """fftlen >= npts: one window over the whole record; without
    whitening each pair is conj(X_a) X_b at bins j * fstride."""
    npts, nsta, nf, fstride = 240, 3, 30, 3
    rng = np.random.default_rng(2)
    data = rng.standard_normal(nsta * npts).astype(np.float32)
    startend = np.tile(np.array([0, npts + 1], dtype=np.int32), nsta)
    ncfs, counts = C.cross_correlation(data.copy(), npts, nsta, nf, fstride, 4096, 0,
                                       _pairs(nsta), startend, ifspecwhitenning=0)
    X = np.fft.rfft(data.astype(np.float64).reshape(nsta, npts), axis=1)[:, ::fstride][:, :nf]
    for p, (a, b) in enumerate(_pairs(nsta).reshape(-1, 2)):
        assert np.allclose(ncfs[p], np.conj(X[a]) * X[b], rtol=1e-12, atol=1e-9)
    assert counts.tolist() == [1, 1, 1]
    # a record that ends at npts fails the strict end test: nothing is correlated
    startend[1::2] = npts
    ncfs, counts = C.cross_correlation(data.copy(), npts, nsta, nf, fstride, 4096, 0,
                                       _pairs(nsta), startend)
    assert counts.tolist() == [0, 0, 0] and np.all(ncfs == 0)


def test_whitened_delay_is_a_phase_ramp():
    """Station b is station a delayed circularly by d samples inside the one
    window: whitened, conj(X_a) X_b = exp(-2 pi i k d / N) at every bin."""
    npts, d, nf = 256, 7, 100
    rng = np.random.default_rng(3)
    a = rng.standard_normal(npts).astype(np.float32)
    data = np.concatenate([a, np.roll(a, d)])
    startend = np.array([0, npts + 1, 0, npts + 1], dtype=np.int32)
    ncfs, _ = C.cross_correlation(data, npts, 2, nf, 1, npts, npts, _pairs(2), startend)
    k = np.arange(nf)
    assert np.allclose(ncfs[0], np.exp(-2j * np.pi * k * d / npts), atol=1e-9)


def test_average_over_windows():
    """Two identical stations: whitened, every bin averages to 1; without
    whitening, to the mean power over the windows both take part in."""
    npts, fftlen, steplen, nf = 900, 120, 60, 40
    rng = np.random.default_rng(4)
    a = rng.standard_normal(npts).astype(np.float32)
    data = np.concatenate([a, a])
    startend = np.array([0, npts, 100, 700], dtype=np.int32)
    ncfs, counts = C.cross_correlation(data.copy(), npts, 2, nf, 1, fftlen, steplen,
                                       _pairs(2), startend)
    starts = [s for s in range(0, npts - fftlen + 1, steplen) if s >= 100 and s + fftlen < 700]
    assert counts[0] == len(starts) == 8
    assert np.allclose(ncfs[0], 1.0, atol=1e-12)
    ncfs, _ = C.cross_correlation(data.copy(), npts, 2, nf, 1, fftlen, steplen, _pairs(2),
                                  startend, ifspecwhitenning=0)
    power = np.mean([np.abs(np.fft.rfft(a[s:s + fftlen].astype(np.float64))[:nf]) ** 2
                     for s in starts], axis=0)
    assert np.allclose(ncfs[0], power, rtol=1e-12)


def test_whitening_floor():
    """An all-zero window whitens to 0 / max(0, 1e-8) = 0, not NaN."""
    npts, nf = 64, 10
    data = np.zeros(2 * npts, dtype=np.float32)
    data[npts:] = 1.0
    startend = np.array([0, npts + 1, 0, npts + 1], dtype=np.int32)
    ncfs, counts = C.cross_correlation(data, npts, 2, nf, 1, npts, npts, _pairs(2), startend)
    assert counts[0] == 1 and np.all(ncfs == 0)


def test_onebit_is_applied_to_the_callers_float32_array():
    npts, nsta, nf, fftlen = 300, 3, 20, 100
    rng = np.random.default_rng(5)
    d64 = rng.standard_normal(nsta * npts)
    d32 = d64.astype(np.float32)
    startend = np.tile(np.array([0, npts], dtype=np.int32), nsta)
    pairs = _pairs(nsta)
    expect = C.CC(npts, nsta, nf, fftlen, pairs, startend, np.sign(d32), overlaprate=0.5)
    got = C.CC(npts, nsta, nf, fftlen, pairs, startend, d32, overlaprate=0.5, ifonebit=1)
    assert np.array_equal(got, expect)
    assert np.array_equal(d32, np.sign(d64).astype(np.float32))   # modified in place
    before = d64.copy()
    C.CC(npts, nsta, nf, fftlen, pairs, startend, d64, overlaprate=0.5, ifonebit=1)
    assert np.array_equal(d64, before)                              # the cast copied it


def test_wrapper_shapes_and_types():
    npts, nsta, nf, fftlen = 400, 4, 25, 128
    rng = np.random.default_rng(6)
    data = rng.standard_normal(nsta * npts).astype(np.float32)
    startend = np.tile(np.array([0, npts], dtype=np.int32), nsta)
    pairs = _pairs(nsta)
    out = C.CC(npts, nsta, nf, fftlen, pairs, startend, data, overlaprate=0.25)
    assert out.dtype == np.complex64 and out.shape == (6, nf)
    # an odd-length pair list drops its last index, as int(len(Pairs) / 2) does
    out2 = C.CC(npts, nsta, nf, fftlen, np.append(pairs, 3).astype(np.int32), startend, data,
                overlaprate=0.25)
    assert np.array_equal(out, out2)
    # bins 0..fftlen/2 exist (65 of them for 128); the reference reads past them
    assert C.CC(npts, nsta, 65, fftlen, pairs, startend, data, overlaprate=0.25).shape == (6, 65)
    with pytest.raises(ValueError):
        C.CC(npts, nsta, 66, fftlen, pairs, startend, data, overlaprate=0.25)
    with pytest.raises(ValueError):
        C.CC(npts, nsta, 34, fftlen, pairs, startend, data, overlaprate=0.25, fstride=2)
