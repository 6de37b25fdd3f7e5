#!/usr/bin/env python3
"""Regenerates tests/golden/cc_reference_outputs.npz by running the
REFERENCE's own cross-correlator -- its `CC` wrapper (src/ccfj.pyx:125-147)
over CrossCorrelation (src/CrossCorr.cpp:33-159), built unmodified by
`make -C oracle` into oracle/_ref/ against oracle/fftw_shim (FFTW itself is
not installed) -- on small seeded cases.

The reference ships no tests or data for the cross-correlator, so these
files are the record of its outputs; tests/ pins the FP64 oracle, the host
replay of the kernels and the CUDA path against them. Run in a container
that has the reference sources and the oracle/_ref build:

    make -C oracle && python tests/golden/make_cc_golden.py

Each case stores its inputs (the float32 records before the call -- the
reference's one-bit step rewrites them in place -- the pair list and the
valid ranges), its parameters and the reference's complex64 output.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle", "_ref"))

import ccfj_ref  # noqa: E402  (the reference's Cython module)


def all_pairs(nsta):
    return np.asarray(ccfj_ref.GetStationPairs(nsta), dtype=np.int32)


def cases():
    """(name, nsta, npts, nf, fftlen, pairs, startend, data, overlaprate,
    fstride, ifonebit, ifspecwhittenning)"""
    out = []
    rng = np.random.default_rng(101)
    nsta, npts = 5, 3000
    out.append(("cc_basic", nsta, npts, 120, 512, all_pairs(nsta),
                np.tile([0, npts], nsta).astype(np.int32),
                rng.standard_normal(nsta * npts).astype(np.float32), 0.5, 2, 0, 1))
    rng = np.random.default_rng(102)
    nsta, npts = 4, 2500
    se = np.array([0, 2500, 300, 2500, 0, 1900, 650, 2200], dtype=np.int32)
    out.append(("cc_onebit_raw_ragged", nsta, npts, 201, 400, all_pairs(nsta), se,
                rng.standard_normal(nsta * npts).astype(np.float32), 0.25, 1, 1, 0))
    rng = np.random.default_rng(103)
    nsta, npts = 3, 700
    out.append(("cc_single_window", nsta, npts, 351, 1000, all_pairs(nsta),
                np.tile([0, 701], nsta).astype(np.int32),
                rng.standard_normal(nsta * npts).astype(np.float32), 0.0, 1, 0, 1))
    rng = np.random.default_rng(104)
    nsta, npts = 6, 2600
    pairs = np.array([0, 1, 3, 1, 2, 2, 0, 4, 0, 4, 5, 0, 1, 5, 4, 3], dtype=np.int32)
    se = np.array([0, 2600, 100, 2600, 0, 2600, 0, 2000, 500, 2600, 0, 300], dtype=np.int32)
    out.append(("cc_pairs_irregular_onebit", nsta, npts, 50, 441, pairs, se,
                rng.standard_normal(nsta * npts).astype(np.float32), 0.3, 3, 1, 1))
    rng = np.random.default_rng(105)
    nsta, npts = 4, 2000
    out.append(("cc_odd_length", nsta, npts, 60, 375, all_pairs(nsta),
                np.tile([0, npts], nsta).astype(np.int32),
                rng.standard_normal(nsta * npts).astype(np.float32), 0.6, 3, 0, 1))
    rng = np.random.default_rng(106)
    nsta, npts = 4, 7200
    out.append(("cc_example_shape", nsta, npts, 200, 1440, all_pairs(nsta),
                np.tile([0, npts], nsta).astype(np.int32),
                rng.standard_normal(nsta * npts).astype(np.float32), 0.9, 3, 0, 1))
    return out


def main():
    store = {}
    for (name, nsta, npts, nf, fftlen, pairs, se, data, ov, fstride, onebit,
         whiten) in cases():
        d = data.copy()  # the reference rewrites float32 records in place (one-bit)
        res = ccfj_ref.CC(npts, nsta, nf, fftlen, pairs, se, d, overlaprate=ov, nThreads=4,
                          fstride=fstride, ifonebit=onebit, ifspecwhittenning=whiten)
        store[name + "__data"] = data
        store[name + "__pairs"] = pairs
        store[name + "__startend"] = se
        store[name + "__params"] = np.array([nsta, npts, nf, fftlen, fstride, onebit, whiten],
                                            dtype=np.int64)
        store[name + "__overlaprate"] = np.array([ov])
        store[name + "__out"] = np.asarray(res, dtype=np.complex64)
        store[name + "__data_after"] = d
    path = os.path.join(HERE, "cc_reference_outputs.npz")
    np.savez_compressed(path, **store)
    print("wrote", path, "cases:", sorted({k.split("__")[0] for k in store}))


if __name__ == "__main__":
    main()
