"""FP64 CPU restatement of CC-FJpy's ambient-noise cross-correlator -- TEST
INFRASTRUCTURE ONLY.

This module is a checker: only tests/ may import it. The product
(cc-fjpy_b200/ccfj) never imports it.

What it restates (reference file:line):

* CC -- the Python wrapper of src/ccfj.pyx:125-147 (the same code in
  src/ccfj-gpu.pyx:146-167): steplen = int(fftlen * (1 - overlaprate)),
  npairs = int(len(Pairs) / 2), a float32 cast of `data` that copies only
  when the dtype differs, float32 accumulators, and a complex64 result
  [npairs, nf].
* cross_correlation -- CrossCorrelation of src/CrossCorr.cpp:33-159:
    - nshifts: fftlen >= npts clamps fftlen to npts with one shift, else
      nshifts = 1 + (npts - fftlen) / steplen in integer division (:47-53);
    - one-bit: data = sign(data) in place, over the caller's array when no
      cast copied it (:72-81);
    - station i takes part in shift k when k*steplen >= startend[2i] and
      k*steplen + fftlen < startend[2i+1] (:88-95);
    - its spectrum is the unnormalised forward real FFT (FFTW r2c) of the
      window, bins j*fstride for j < nf (:97-100), whitened to
      X / max(|X|, 1e-8) when ifspecwhitenning (:101-115);
    - pair (a, b) gets conj(X_a) X_b added when both take part, and a count
      (:118-131); each pair with a nonzero count is divided by it (:133-144).

Pinning: FFTW is not in this image, so src/CrossCorr.cpp is compiled
unmodified against oracle/fftw_shim (this project's FP64 stand-in for the
few FFTW calls it makes) into oracle/_ref, and tests/golden/
make_cc_golden.py records the reference's CC outputs on six seeded cases
(tests/golden/cc_reference_outputs.npz). tests/test_cc_golden.py holds
this restatement to them within 2e-5 of each pair's largest value;
tests/test_cc_oracle.py adds properties that follow from the code above.

Arithmetic: float64 on the float32 (one-bit: sign) samples with numpy's
rfft; the reference works in float32 with FFTW.
"""
import numpy as np

__all__ = ["cc_shifts", "cc_active", "cross_correlation", "CC"]

WHITEN_FLOOR = float(np.float32(1e-8))  # max(absv, 1e-8f), src/CrossCorr.cpp:106


def cc_shifts(npts, fftlen, steplen):
    """(fftlen, nshifts) after src/CrossCorr.cpp:47-53."""
    if fftlen >= npts:
        return npts, 1
    if steplen <= 0:
        # the reference divides by steplen (or loops over a negative count)
        raise ValueError("steplen=%d must be positive when fftlen < npts" % steplen)
    return fftlen, 1 + (npts - fftlen) // steplen


def cc_active(k, steplen, fftlen, startend, i):
    """Whether station i takes part in shift k (src/CrossCorr.cpp:88-95)."""
    s = k * steplen
    return s >= startend[2 * i] and s + fftlen < startend[2 * i + 1]


def cross_correlation(data, npts, nsta, nf, fstride, fftlen, steplen, pairs, startend,
                      ifonebit=0, ifspecwhitenning=1):
    """CrossCorrelation on float32 `data` [nsta * npts] (modified in place
    when ifonebit). Returns (ncfs complex128 [npairs, nf], counts int64
    [npairs])."""
    pairs = np.asarray(pairs).reshape(-1, 2)
    startend = np.asarray(startend)
    fftlen, nshifts = cc_shifts(npts, fftlen, steplen)
    if nf > 0 and (nf - 1) * fstride > fftlen // 2:
        # FFTW's r2c writes bins 0..fftlen/2; the reference reads past them
        raise ValueError("bin (nf-1)*fstride=%d exceeds fftlen/2=%d"
                         % ((nf - 1) * fstride, fftlen // 2))
    if ifonebit:
        data[:nsta * npts] = np.sign(data[:nsta * npts])
    x = np.asarray(data[:nsta * npts], dtype=np.float64).reshape(nsta, npts)
    bins = np.arange(nf) * fstride
    acc = np.zeros((len(pairs), nf), dtype=np.complex128)
    counts = np.zeros(len(pairs), dtype=np.int64)
    for k in range(nshifts):
        act = np.array([cc_active(k, steplen, fftlen, startend, i) for i in range(nsta)])
        if not act.any():
            continue
        s = k * steplen
        X = np.zeros((nsta, nf), dtype=np.complex128)
        idx = np.nonzero(act)[0]
        X[idx] = np.fft.rfft(x[idx, s:s + fftlen], axis=1)[:, bins]
        if ifspecwhitenning:
            X[idx] /= np.maximum(np.abs(X[idx]), WHITEN_FLOOR)
        both = act[pairs[:, 0]] & act[pairs[:, 1]]
        p = np.nonzero(both)[0]
        acc[p] += np.conj(X[pairs[p, 0]]) * X[pairs[p, 1]]
        counts[p] += 1
    nz = counts > 0
    acc[nz] /= counts[nz, None]
    return acc, counts


def CC(npts, nsta, nf, fftlen, Pairs, startend, data, overlaprate=0.0, nThreads=8, fstride=1,
       ifonebit=0, ifspecwhittenning=1):
    """src/ccfj.pyx:125-147: complex64 [npairs, nf]."""
    steplen = int(fftlen * (1 - overlaprate))
    npairs = int(len(Pairs) / 2)
    if data.dtype != np.float32:
        data = np.array(data, dtype=np.float32)
    ncfs, _ = cross_correlation(data, npts, nsta, nf, fstride, fftlen, steplen,
                                np.asarray(Pairs)[:2 * npairs], startend, ifonebit,
                                ifspecwhittenning)
    return ncfs.astype(np.complex64)
