"""The Python layer's hand-off to ccfj_fj_v1 without a GPU: with the library
replaced by a recorder, every element the argument struct says the device
reads (u[0][row*u_ld + col*u_es], through the raw pointer) must equal the
value the reference reads for that pair and frequency
(float32(Re(uf[perm[i], j*fstride])), src/ccfj-gpu.pyx:181-200), for the
memory layouts callers pass: complex64 read in place, float32 rows with
any row stride, float64 / complex128 / Fortran-order copies, and the
reference's flatten-and-reshape when the rows do not match the pairs.
Likewise for ccfj_fj_earthquake_v1: the spectra its struct describes
(traces, permutation, MWFJ window parameters with the device's taper rule)
equal the reference's host spectra (src/ccfj-gpu.pyx:270-313)."""
import ctypes
import warnings

import numpy as np
import pytest


class _Recorder:
    """Stands in for the loaded library: ccfj_fj_v1 reads the input through
    the struct's pointers and strides, as the device does."""

    def __init__(self):
        self.seen = None

    def ccfj_fj_v1(self, aref, stream):
        a = aref._obj
        nf, nr = a.nf, a.nr
        perm = None
        if a.perm:
            perm = np.ctypeslib.as_array(ctypes.cast(a.perm, ctypes.POINTER(ctypes.c_longlong)),
                                         shape=(nr,)).copy()
        fp = ctypes.cast(a.u[0], ctypes.POINTER(ctypes.c_float))
        vals = np.empty((nr, nf), dtype=np.float32)
        for i in range(nr):
            row = perm[i] if perm is not None else i
            assert 0 <= row < a.u_rows
            for j in range(nf):
                col = (a.col_begin + j) * a.fstride
                assert col < a.u_ncols
                vals[i, j] = fp[row * a.u_ld + col * a.u_es]
        self.seen = dict(vals=vals, es=a.u_es, ld=a.u_ld, ptr=a.u[0], fstride=a.fstride,
                         perm=perm, mode=a.mode, hilbert=a.hilbert, normalize=a.normalize)
        out = ctypes.cast(a.out, ctypes.POINTER(ctypes.c_float))
        for k in range(a.nc * nf):
            out[k] = 0.0
        return 0

    def ccfj_last_error(self):
        return b""


@pytest.fixture
def rec(monkeypatch):
    from ccfj import _lib
    r = _Recorder()
    monkeypatch.setattr(_lib, "load", lambda: r)
    return r


def _expected(uf, r, nf, fstride, sort=True):
    idx = np.argsort(r) if sort else np.arange(len(r))
    u = np.asarray(uf)[idx][:, ::fstride].reshape(len(r) * nf)
    if np.iscomplexobj(u):
        u = u.real
    return u.astype(np.float32).reshape(len(r), nf)


def _case(dtype, nr=7, nf=5, fstride=1, order="C", row_step=1):
    rng = np.random.default_rng(0)
    ncols = nf * fstride
    base = rng.standard_normal((nr * row_step, ncols)) + 1j * rng.standard_normal(
        (nr * row_step, ncols))
    if not np.issubdtype(np.dtype(dtype), np.complexfloating):
        base = base.real
    uf = np.asarray(base, dtype=dtype, order=order)[::row_step]
    r = rng.uniform(1e3, 5e4, nr)
    return uf, r, np.linspace(1000, 4000, 3), np.linspace(0.1, 1.0, nf)


@pytest.mark.parametrize("dtype,order,row_step,fstride,in_place", [
    (np.complex64, "C", 1, 1, True),     # interleaved complex: real parts in place
    (np.complex64, "C", 2, 3, True),     # every other row, every third column
    (np.float32, "C", 1, 2, True),
    (np.float32, "C", 3, 1, True),       # row stride 3 rows
    (np.float64, "C", 1, 1, False),      # copied to float32
    (np.complex128, "C", 1, 2, False),
    (np.float32, "F", 1, 1, False),      # column-major: copied
])
def test_fj_noise_reads_what_the_reference_reads(rec, dtype, order, row_step, fstride, in_place):
    import ccfj
    uf, r, c, f = _case(dtype, fstride=fstride, order=order, row_step=row_step)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ccfj.fj_noise(uf, r, c, f, fstride=fstride)
    s = rec.seen
    assert np.array_equal(s["vals"], _expected(uf, r, len(f), fstride))
    assert np.array_equal(s["perm"], np.argsort(r))
    assert s["normalize"] == 1 and s["hilbert"] == 0
    base = np.asarray(uf)
    if in_place:   # no copy: the device reads the caller's memory
        assert s["ptr"] == base.ctypes.data
        assert s["es"] == (2 if np.iscomplexobj(base) else 1)
    else:
        assert s["ptr"] != base.ctypes.data


def test_func1_asks_for_the_device_hilbert_transform(rec):
    import ccfj
    from ccfj import _lib
    uf, r, c, f = _case(np.complex64)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ccfj.fj_noise(uf, r, c, f, func=1)
    assert rec.seen["mode"] == _lib.MODE_J_MINUS_Y and rec.seen["hilbert"] == 1


def test_rows_that_do_not_match_the_pairs_follow_the_reference_reshape(rec):
    """uf with 2*nr rows of nf/2 columns holds nr*nf values: the reference's
    uf[:, ::1].reshape(nr*nf) regroups them into nr rows of nf."""
    import ccfj
    rng = np.random.default_rng(1)
    nr, nf = 6, 4
    uf = rng.standard_normal((2 * nr, nf // 2)).astype(np.float32)
    r = rng.uniform(1e3, 5e4, nr)
    ccfj.fj(uf, r, np.linspace(1000, 4000, 3), np.linspace(0.1, 1.0, nf))
    assert np.array_equal(rec.seen["vals"], uf.reshape(nr, nf))
    assert rec.seen["perm"] is None


def test_low_level_fj_keeps_the_callers_pair_order(rec):
    import ccfj
    uf, r, c, f = _case(np.float32)
    ccfj.fhi(uf, r, c, f)
    assert rec.seen["perm"] is None
    assert np.array_equal(rec.seen["vals"], _expected(uf, r, len(f), 1, sort=False))


class _EqRecorder:
    """Stands in for the library's ccfj_fj_earthquake_v1: reads the traces,
    the permutation and the window parameters through the struct the way
    the device does (sorted trace i is row perm[i]; window w of that trace
    takes parameters [w][perm[i]] and the device's per-sample taper rule)
    and records the spectra the transform would see."""

    def __init__(self):
        self.spec = None

    def ccfj_fj_earthquake_v1(self, aref, stream):
        from test_host_logic import _device_rule
        a = aref._obj
        fp = ctypes.cast(a.u, ctypes.POINTER(ctypes.c_float))
        perm = np.ctypeslib.as_array(ctypes.cast(a.perm, ctypes.POINTER(ctypes.c_longlong)),
                                     shape=(a.ntr,))
        nw = max(a.nwin, 1)
        wins = None
        if a.nwin > 0:
            wins = [np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_int)),
                                          shape=(a.nwin, a.u_rows))
                    for p in (a.win_n1, a.win_n2, a.win_delta)]
        spec = np.empty((nw, a.ntr, a.nf), dtype=np.complex128)
        for w in range(nw):
            for i in range(a.ntr):
                row = int(perm[i])
                x = np.array([fp[row * a.u_ld + n] for n in range(a.npts)], dtype=np.float64)
                if wins is not None:
                    x = x * _device_rule(a.npts, *(int(v[w, row]) for v in wins))
                spec[w, i] = np.fft.rfft(x)[0:a.nf * a.fstride:a.fstride]
        self.spec = spec
        out = ctypes.cast(a.out, ctypes.POINTER(ctypes.c_float))
        for k in range(nw * a.nc * a.nf):
            out[k] = 0.0
        return 0

    def ccfj_last_error(self):
        return b""


@pytest.fixture
def eqrec(monkeypatch):
    from ccfj import _lib
    r = _EqRecorder()
    monkeypatch.setattr(_lib, "load", lambda: r)
    return r


def _traces(nr=6, npts=96, extra_rows=0, row_step=1, dtype=np.float32):
    rng = np.random.default_rng(2)
    u = rng.standard_normal(((nr + extra_rows) * row_step, npts)).astype(dtype)[::row_step]
    return u, rng.uniform(1e3, 5e4, nr)


@pytest.mark.parametrize("row_step,dtype", [(1, np.float32), (2, np.float32), (1, np.float64)])
def test_fj_earthquake_spectra_are_the_references(eqrec, row_step, dtype):
    import ccfj
    u, r = _traces(row_step=row_step, dtype=dtype)
    nf = 20
    f = np.arange(nf) * 10.0 / u.shape[1]
    ccfj.fj_earthquake(u, r, np.linspace(1000, 4000, 3), f)
    idx = np.argsort(r)
    ref = np.fft.rfft(u[idx].astype(np.float32).astype(np.float64))[:, 0:nf]
    assert np.allclose(eqrec.spec[0], ref, rtol=0, atol=1e-9 * np.abs(ref).max())


def test_mwfj_windows_follow_the_callers_trace_order(eqrec):
    """MWFJ tapers trace j of window i by win(npts, Fs, winl[i][j],
    winr[i][j], taper) before fj_earthquake sorts the traces
    (src/ccfj-gpu.pyx:297-313); the device sorts first, so it must look the
    window up by the trace's original row."""
    import ccfj
    u, r = _traces(nr=5, npts=120, extra_rows=2)
    nwin, Fs, taper, nf = 3, 10.0, 0.7, 16
    rng = np.random.default_rng(4)
    winl = rng.uniform(-1.0, 5.0, (nwin, len(r)))
    winr = winl + rng.uniform(2.0, 9.0, (nwin, len(r)))
    f = np.arange(nf) * Fs / u.shape[1]
    ccfj.MWFJ(u, r, np.linspace(1000, 4000, 3), f, Fs, nwin, winl, winr, taper=taper)
    idx = np.argsort(r)
    for i in range(nwin):
        u1 = np.array([u[j] * ccfj.win(u.shape[1], Fs, winl[i][j], winr[i][j], taper)
                       for j in range(len(r))])
        ref = np.fft.rfft(u1[idx].astype(np.float32).astype(np.float64))[:, 0:nf]
        assert np.allclose(eqrec.spec[i], ref, rtol=0, atol=1e-6 * np.abs(ref).max()), i


class _BatchRecorder:
    """ccfj_fj_batch_v1 stand-in: per set, the values and distances the
    device reads for its sorted pairs."""

    def __init__(self):
        self.sets = None

    def ccfj_fj_batch_v1(self, aref, stream):
        a = aref._obj
        P = ctypes.POINTER
        off = np.ctypeslib.as_array(ctypes.cast(a.offsets, P(ctypes.c_longlong)),
                                    shape=(a.nsets + 1,))
        perm = np.ctypeslib.as_array(ctypes.cast(a.perm, P(ctypes.c_longlong)),
                                     shape=(a.total_pairs,))
        r = np.ctypeslib.as_array(ctypes.cast(a.r, P(ctypes.c_float)), shape=(a.total_pairs,))
        fp = ctypes.cast(a.u[0], P(ctypes.c_float))
        self.sets = []
        for b in range(a.nsets):
            vals = np.array([[fp[int(perm[i]) * a.u_ld + j * a.fstride * a.u_es]
                              for j in range(a.nf)] for i in range(off[b], off[b + 1])],
                            dtype=np.float32)
            self.sets.append((vals, r[off[b]:off[b + 1]].copy()))
        out = ctypes.cast(a.out, P(ctypes.c_float))
        for k in range(a.nsets * a.nc * a.nf):
            out[k] = 0.0
        return 0

    def ccfj_last_error(self):
        return b""


@pytest.mark.parametrize("dtype", [np.complex64, np.float64])
def test_batch_sets_read_their_own_sorted_pairs(monkeypatch, dtype):
    import ccfj
    from ccfj import _lib
    rec = _BatchRecorder()
    monkeypatch.setattr(_lib, "load", lambda: rec)
    rng = np.random.default_rng(5)
    nf, fstride = 4, 2
    ufs, rs = [], []
    for n in (3, 1, 6):
        x = rng.standard_normal((n, nf * fstride)) + 1j * rng.standard_normal((n, nf * fstride))
        ufs.append(x.astype(dtype) if dtype == np.complex64 else x.real.astype(dtype))
        rs.append(rng.uniform(1e3, 5e4, n))
    ccfj.fj_noise_batch(ufs, rs, np.linspace(1000, 4000, 3), np.linspace(0.1, 1, nf),
                        fstride=fstride)
    for (vals, rsorted), uf, r in zip(rec.sets, ufs, rs):
        assert np.array_equal(vals, _expected(uf, r, nf, fstride))
        assert np.array_equal(rsorted, np.sort(r).astype(np.float32))


def test_earthquake_result_type_is_float32_or_float64():
    """MWFJ's float64 result comes from the library's copy-out; any other
    result type is refused before the call."""
    from ccfj import _eq
    rng = np.random.default_rng(0)
    u = rng.standard_normal((3, 64)).astype(np.float32)
    r = np.array([1e3, 2e3, 3e3])
    with pytest.raises(ValueError, match="float32 or float64"):
        _eq._run(u, r, np.array([2000.0, 3000.0]), np.array([0.1, 0.2]), 1, 1, 0,
                 dtype=np.int32)
