"""The cross-correlator pinned to the reference itself.

tests/golden/cc_reference_outputs.npz holds the outputs of the reference's
own CC / CrossCorrelation (src/ccfj.pyx:125-147, src/CrossCorr.cpp:33-159),
compiled unmodified against this project's stand-in for the few FFTW calls
it makes (oracle/fftw_shim), on six seeded cases: whitened and raw spectra,
one-bit records, ragged valid ranges, a single window (fftlen >= npts),
bins up to fftlen/2, odd and factor-7 window lengths, reversed, self and
duplicate pairs, a station that never takes part, and the reference
example's window shape (0.9 overlap, fstride 3). make_cc_golden.py made it.

Checked here without a GPU: the FP64 oracle and the host replay of the CUDA
kernels (tests/cc_emul.cpp); on a GPU (marked gpu): ccfj.CC and the
reference-layout CrossCorrelation entry. Tolerance: 2e-5 of each pair's
largest value (FP32 transforms and sums); pairs without a common window are
exactly zero; one-bit records are rewritten in place exactly as the
reference rewrites them.
"""
import ctypes
import os

import numpy as np
import pytest

import cc_oracle as C
from conftest import REPO

TOL = 2e-5
GOLDEN = os.path.join(REPO, "tests", "golden", "cc_reference_outputs.npz")


def _load():
    with np.load(GOLDEN) as z:
        d = {k: z[k] for k in z.files}
    names = sorted({k.split("__")[0] for k in d})
    return names, d


NAMES, G = _load()


def _case(name):
    nsta, npts, nf, fftlen, fstride, onebit, whiten = (int(v) for v in G[name + "__params"])
    kw = dict(overlaprate=float(G[name + "__overlaprate"][0]), fstride=fstride, ifonebit=onebit,
              ifspecwhittenning=whiten)
    args = (npts, nsta, nf, fftlen, G[name + "__pairs"].copy(), G[name + "__startend"].copy(),
            G[name + "__data"].copy())
    return args, kw


def _err(got, ref):
    scale = np.abs(ref).max(axis=1, keepdims=True)
    zero = scale[:, 0] == 0
    assert np.all(got[zero] == 0)
    if not (~zero).any():
        return 0.0
    return float((np.abs(got - ref)[~zero] / scale[~zero]).max())


def test_golden_cases_cover_the_reference_semantics():
    assert len(NAMES) == 6
    irr = G["cc_pairs_irregular_onebit__out"]
    assert np.all(irr[5] == 0) and np.all(irr[6] == 0)        # station 5 never takes part
    assert np.array_equal(irr[3], irr[4])                       # a duplicate pair
    for name in NAMES:                                          # one-bit rewrote the records
        onebit = int(G[name + "__params"][5])
        after = G[name + "__data_after"]
        assert np.array_equal(after, np.sign(G[name + "__data"]) if onebit else G[name + "__data"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference(name):
    args, kw = _case(name)
    data = args[6]
    got = C.CC(*args, **kw)
    assert _err(got, G[name + "__out"]) <= TOL
    assert np.array_equal(data, G[name + "__data_after"])     # same in-place one-bit


@pytest.mark.parametrize("name", NAMES)
def test_host_replay_of_the_kernels_matches_reference(name, emul):
    from test_cc_emul import _emul_cc
    args, kw = _case(name)
    got = _emul_cc(emul, *args, **kw)
    assert _err(got, G[name + "__out"]) <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_device_matches_reference(name):
    import ccfj
    args, kw = _case(name)
    data = args[6]
    got = ccfj.CC(*args, **kw)
    assert got.dtype == np.complex64 and got.shape == G[name + "__out"].shape
    assert _err(got, G[name + "__out"]) <= TOL
    assert np.array_equal(data, G[name + "__data_after"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cc_basic", "cc_pairs_irregular_onebit"])
def test_reference_layout_entry_matches_reference(lib, name):
    """CrossCorrelation with the reference's CC_data layout, on zeroed
    outputs as the reference's CC wrapper passes them."""
    from ccfj import _cc
    args, kw = _case(name)
    npts, nsta, nf, fftlen, pairs, se, data = args
    npairs = len(pairs) // 2
    re = np.zeros(npairs * nf, dtype=np.float32)
    im = np.zeros(npairs * nf, dtype=np.float32)
    d = _cc.CcData()
    d.nsta, d.npts, d.nf, d.npairs = nsta, npts, nf, npairs
    d.fstride, d.fftlen = kw["fstride"], fftlen
    d.steplen = int(fftlen * (1 - kw["overlaprate"]))
    d.Pairs, d.startend, d.data = pairs.ctypes.data, se.ctypes.data, data.ctypes.data
    d.ncfsr, d.ncfsi = re.ctypes.data, im.ctypes.data
    d.ifonebit, d.ifspecwhitenning, d.nThreads = kw["ifonebit"], kw["ifspecwhittenning"], 8
    assert lib.CrossCorrelation(d) == 0, lib.ccfj_last_error().decode()
    got = (re + 1j * im).reshape(npairs, nf)
    assert _err(got, G[name + "__out"]) <= TOL
    assert np.array_equal(data, G[name + "__data_after"])
