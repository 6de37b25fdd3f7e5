"""The reference module's low-level shims (fj_full, fHr_full, fHi_full,
fH_full, CC_full) without a GPU: with the library replaced by a recorder,
each passes the caller's own buffers (so results land in the caller's
`out`) and sizes to the C entry the reference shim calls, and rejects what
the reference's typed memoryviews reject."""
import ctypes

import numpy as np
import pytest


class _Rec:
    def __init__(self):
        self.calls = []

    def _fj(self, name, *args):
        ptrs = [ctypes.cast(p, ctypes.c_void_p).value for p in args[:5]]
        self.calls.append((name, ptrs, list(args[5:])))
        ctypes.cast(args[3], ctypes.POINTER(ctypes.c_float))[0] = 42.0   # out[0]
        return 0

    def FJ(self, *a):
        return self._fj("FJ", *a)

    def FHr(self, *a):
        return self._fj("FHr", *a)

    def FHi(self, *a):
        return self._fj("FHi", *a)

    def FH(self, *a):
        return self._fj("FH", *a)

    def CrossCorrelation(self, d):
        self.calls.append(("CrossCorrelation", d))
        ctypes.cast(d.ncfsr, ctypes.POINTER(ctypes.c_float))[0] = 7.0
        return 0

    def ccfj_last_error(self):
        return b""


@pytest.fixture
def rec(monkeypatch):
    from ccfj import _lib
    r = _Rec()
    monkeypatch.setattr(_lib, "load", lambda: r)
    return r


def _arrays(nr=4, nf=3, nc=2):
    rng = np.random.default_rng(0)
    return (rng.standard_normal(nr * nf).astype(np.float32), np.arange(1, nr + 1, dtype=np.float32),
            np.linspace(0.1, 1, nf).astype(np.float32), np.zeros(nc * nf, dtype=np.float32),
            np.linspace(1000, 2000, nc).astype(np.float32))


@pytest.mark.parametrize("shim,entry,extra", [("fj_full", "FJ", []), ("fHr_full", "FHr", []),
                                              ("fHi_full", "FHi", []), ("fH_full", "FH", [20])])
def test_fj_shims_pass_the_callers_buffers(rec, shim, entry, extra):
    import ccfj
    U, r, f, out, c = _arrays()
    getattr(ccfj, shim)(U, r, f, out, c, 2, 4, 3, 1)
    name, ptrs, ints = rec.calls[-1]
    assert name == entry
    assert ptrs == [x.ctypes.data for x in (U, r, f, out, c)]
    assert ints == [2, 4, 3, 1] + extra
    assert out[0] == 42.0            # written in place


def test_fj_shim_buffer_checks(rec):
    import ccfj
    U, r, f, out, c = _arrays()
    with pytest.raises(ValueError, match="expected 'float' but got 'double'"):
        ccfj.fj_full(U.astype(np.float64), r, f, out, c, 2, 4, 3, 1)
    with pytest.raises(ValueError, match="wrong number of dimensions"):
        ccfj.fj_full(U.reshape(4, 3), r, f, out, c, 2, 4, 3, 1)
    with pytest.raises(ValueError, match="contiguous"):
        ccfj.fj_full(np.repeat(U, 2)[::2], r, f, out, c, 2, 4, 3, 1)
    ro = out.copy()
    ro.setflags(write=False)
    with pytest.raises(ValueError, match="read-only"):
        ccfj.fj_full(U, r, f, ro, c, 2, 4, 3, 1)
    assert rec.calls == []


def test_cc_full_fills_the_reference_struct(rec):
    import ccfj
    nsta, npts, nf = 3, 100, 5
    pairs = ccfj.GetStationPairs(nsta)
    se = np.tile(np.array([0, npts], dtype=np.int32), nsta)
    data = np.ones(nsta * npts, dtype=np.float32)
    re = np.zeros(3 * nf, dtype=np.float32)
    im = np.zeros(3 * nf, dtype=np.float32)
    ccfj.CC_full(npts, nsta, nf, 2, 40, 20, 1, 0, 8, 3, pairs, se, data, re, im)
    name, d = rec.calls[-1]
    assert name == "CrossCorrelation"
    assert (d.nsta, d.npts, d.nf, d.npairs, d.fstride, d.fftlen, d.steplen) == \
        (nsta, npts, nf, 3, 2, 40, 20)
    assert (d.ifonebit, d.ifspecwhitenning, d.nThreads) == (1, 0, 8)
    assert (d.Pairs, d.startend, d.data, d.ncfsr, d.ncfsi) == tuple(
        x.ctypes.data for x in (pairs, se, data, re, im))
    assert re[0] == 7.0
    with pytest.raises(ValueError, match="expected 'int' but got 'long'"):
        ccfj.CC_full(npts, nsta, nf, 2, 40, 20, 1, 0, 8, 3, pairs.astype(np.int64), se, data,
                     re, im)
    with pytest.raises(ValueError, match="shorter"):
        ccfj.CC_full(npts, nsta, nf, 2, 40, 20, 1, 0, 8, 3, pairs, se, data, re[:5], im)
