"""Parity of the CUDA path (through the public API and the C ABI) with the
FP64 oracle and with the reference's own outputs (golden fixtures).

Tolerance: the error metric is max over (c, f) of |y - y64| / max_c |y64|
(the absolute error of the normalised spectrum). The CUDA path must be within
1e-4 of the FP64 oracle, and within (the reference's own error against the
oracle) + 1e-4 of the reference's outputs.
"""
import ctypes
import warnings

import numpy as np
import pytest

import cases
import fj_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-4


@pytest.fixture(scope="module")
def ccfj():
    import ccfj as m
    return m


def _quiet(fn, *a, **k):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return fn(*a, **k)


@pytest.mark.parametrize("name", ["noise_small", "noise_ties", "noise_fstride2", "noise_real64"])
@pytest.mark.parametrize("itype", [0, 1])
@pytest.mark.parametrize("func", [0, 1])
def test_fj_noise(ccfj, golden, name, itype, func):
    case = cases.noise_case(name)
    args = (case["uf"], case["r"], case["c"], case["f"])
    y = _quiet(ccfj.fj_noise, *args, fstride=case["fstride"], itype=itype, func=func)
    assert y.dtype == np.float32 and y.shape == (len(case["c"]), len(case["f"]))
    y64 = O._normalize(_quiet(O.fj_noise, *args, fstride=case["fstride"], itype=itype, func=func,
                              normalize=False))
    err = O.rel_error(y, y64)
    assert err <= TOL, err
    ref = golden["%s_i%d_f%d" % (name, itype, func)]
    ref_err = O.rel_error(ref, y64)
    assert O.rel_error(y, ref) <= ref_err + TOL


@pytest.mark.parametrize("itype", [0, 1])
@pytest.mark.parametrize("func", [0, 1])
def test_fj_earthquake(ccfj, golden, itype, func):
    case = cases.eq_case("eq_small")
    args = (case["u"], case["r"], case["c"], case["f"])
    y = _quiet(ccfj.fj_earthquake, *args, itype=itype, func=func)
    assert y.dtype == np.float32
    y64 = O._normalize(O.fj_earthquake(*args, itype=itype, func=func, normalize=False))
    assert O.rel_error(y, y64) <= TOL
    ref = golden["eq_small_i%d_f%d" % (itype, func)]
    assert O.rel_error(y, ref) <= O.rel_error(ref, y64) + TOL
    # f = 0: k = 0, the reference's column is NaN for the integral form
    if itype == 1:
        assert np.isnan(ref[:, 0]).all() and np.isnan(y[:, 0]).all()


@pytest.mark.parametrize("func", [0, 1])
def test_mwfj(ccfj, golden, func):
    case = cases.mwfj_case("mwfj_small")
    y = _quiet(ccfj.MWFJ, case["u"], case["r"], case["c"], case["f"], case["Fs"], case["nwin"],
               case["winl"], case["winr"], taper=case["taper"], func=func)
    assert y.dtype == np.float64 and y.shape == (case["nwin"], len(case["c"]), len(case["f"]))
    y64 = np.stack([O._normalize(o) for o in O.MWFJ(
        case["u"], case["r"], case["c"], case["f"], case["Fs"], case["nwin"], case["winl"],
        case["winr"], taper=case["taper"], func=func, normalize=False)])
    ref = golden["mwfj_small_i1_f%d" % func]
    for w in range(case["nwin"]):
        assert O.rel_error(y[w], y64[w]) <= TOL
        assert O.rel_error(y[w], ref[w]) <= O.rel_error(ref[w], y64[w]) + TOL


@pytest.mark.parametrize("fname,basis", [("FJ", "J"), ("FHr", "J"), ("FHi", "Y"), ("FH", "Y")])
@pytest.mark.parametrize("itype", [0, 1])
def test_reference_c_abi(ccfj, lib, golden, fname, basis, itype):
    """The reference's own entry points with host pointers (raw, unsorted
    pairs in the given order, no normalisation)."""
    case = cases.noise_case("raw_small")
    U = np.ascontiguousarray(np.real(case["uf"]), dtype=np.float32)
    r32, f32, c32 = (np.ascontiguousarray(case[k], dtype=np.float32) for k in ("r", "f", "c"))
    nr, nf, nc = len(r32), len(f32), len(c32)
    out = np.full(nc * nf, np.nan, dtype=np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    P = lambda a: a.ctypes.data_as(fp)  # noqa: E731
    extra = (8,) if fname == "FH" else ()
    st = getattr(lib, fname)(P(U), P(r32), P(f32), P(out), P(c32), nc, nr, nf, itype, *extra)
    assert st == 0, lib.ccfj_last_error()
    out = out.reshape(nc, nf)
    y64 = O.fj_transform(U, r32, f32, c32, itype, basis)
    assert O.rel_error(out, y64) <= TOL
    ref = golden["raw_%s_i%d" % ("FJ" if basis == "J" else "FH", itype)]
    assert O.rel_error(out, ref) <= O.rel_error(ref, y64) + TOL


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("itype", [0, 1])
@pytest.mark.parametrize("mode", [0, 1])
def test_fp64_forms_match_oracle(ccfj, prec, itype, mode):
    """The FP64 station-amortised form and the FP64 comparator with the
    reference's loop structure agree with the oracle to ~1e-9."""
    case = cases.noise_case("noise_small")
    idx = np.argsort(case["r"])
    U = np.ascontiguousarray(np.real(case["uf"]), dtype=np.float32)
    rs = case["r"][idx]
    y = ccfj._transform([U], rs, case["c"], case["f"], 1, itype, mode, perm=idx, precision=prec)
    y64 = O.fj_transform(U[idx], rs.astype(np.float32), case["f"].astype(np.float32),
                         case["c"].astype(np.float32), itype, "JY"[mode])
    assert O.rel_error(y, y64) <= 1e-6


def test_unsorted_pairs_follow_reference_order(ccfj):
    """fj() does not sort (src/ccfj-gpu.pyx:181-200): reversed intervals are
    integrated as given, like the reference."""
    case = cases.noise_case("noise_small")
    U = np.ascontiguousarray(np.real(case["uf"]), dtype=np.float32)
    y = ccfj.fj(U, case["r"], case["c"], case["f"], itype=1)
    y64 = O.fj_transform(U, case["r"].astype(np.float32), case["f"].astype(np.float32),
                         case["c"].astype(np.float32), 1, "J")
    assert O.rel_error(y, y64) <= TOL


def test_deterministic(ccfj):
    case = cases.noise_case("noise_small")
    a = _quiet(ccfj.fj_noise, case["uf"], case["r"], case["c"], case["f"], func=1)
    b = _quiet(ccfj.fj_noise, case["uf"], case["r"], case["c"], case["f"], func=1)
    assert np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("nr", [1, 2, 3])
def test_tiny_pair_counts(ccfj, nr):
    rng = np.random.default_rng(nr)
    r = rng.uniform(1e3, 2e4, nr)
    f = np.linspace(0.05, 0.5, 12)
    c = np.linspace(1000, 4000, 9)
    uf = cases.noise_spectra(rng, r, f)
    for itype in (0, 1):
        y = _quiet(ccfj.fj_noise, uf, r, c, f, itype=itype, normalize=False) \
            if False else _quiet(ccfj._transform, [np.real(uf)], np.sort(r), c, f, 1, itype, 0,
                                 perm=np.argsort(r))
        y64 = O.fj_transform(np.real(uf)[np.argsort(r)], np.sort(r).astype(np.float32),
                             f.astype(np.float32), c.astype(np.float32), itype, "J")
        if nr == 1:
            assert np.all(y == 0)
        else:
            assert O.rel_error(y, y64) <= TOL


def test_invalid_func_and_shape(ccfj, capsys):
    case = cases.noise_case("noise_small")
    assert ccfj.fj_noise(case["uf"], case["r"], case["c"], case["f"], func=3) == 0
    assert "set func as 0" in capsys.readouterr().out
    with pytest.raises(ValueError, match="cannot reshape"):
        ccfj.fj_noise(case["uf"][:, :-1], case["r"], case["c"], case["f"])
    eq = cases.eq_case("eq_small")
    with pytest.raises(ValueError, match="cannot reshape"):
        ccfj.fj_earthquake(eq["u"], eq["r"], eq["c"], eq["f"], fstride=2)


@pytest.mark.parametrize("itype", [0, 1])
@pytest.mark.parametrize("func", [0, 1])
def test_mwfj_window_tiles(ccfj, itype, func):
    """10 windows: one full tile of 8 windows and a partial tile of 2 share
    each station evaluation; every window matches the FP64 oracle and the
    single-window transform of the windowed traces."""
    rng = np.random.default_rng(41)
    npts, Fs, ntr, nwin = 256, 10.0, 14, 10
    r = np.exp(rng.uniform(np.log(5e3), np.log(1.5e5), ntr))
    u = cases.ricker_records(rng, r, npts, Fs)
    L = rng.integers(40, 200, size=(nwin, ntr))
    start = rng.integers(0, npts - L)
    winl, winr = start / Fs, (start + L) / Fs
    f = Fs * np.arange(24) / npts
    c = np.linspace(1500, 5000, 33)
    y = _quiet(ccfj.MWFJ, u, r, c, f, Fs, nwin, winl, winr, taper=0.9, itype=itype, func=func)
    y64 = O.MWFJ(u, r, c, f, Fs, nwin, winl, winr, taper=0.9, itype=itype, func=func,
                 normalize=False)
    for w in range(nwin):
        assert O.rel_error(y[w], O._normalize(y64[w])) <= TOL
        uw = np.stack([u[j] * ccfj.win(npts, Fs, winl[w, j], winr[w, j], 0.9) for j in range(ntr)])
        single = _quiet(ccfj.fj_earthquake, uw, r, c, f, itype=itype, func=func)
        assert O.rel_error(y[w], single) <= TOL


@pytest.mark.parametrize("func", [0, 1])
@pytest.mark.parametrize("itype", [0, 1])
def test_frequency_window_equals_full_transform(ccfj, func, itype):
    """Computing frequencies a..b-1 only (the sharded path's unit) gives the
    same bits as those columns of the full transform (the Hilbert transform
    still runs along the full rows)."""
    from ccfj import dist
    case = cases.noise_case("noise_fstride2")
    args = (case["uf"], case["r"], case["c"], case["f"], case["fstride"], itype, func)
    full = _quiet(ccfj.fj_noise, *args[:4], fstride=case["fstride"], itype=itype, func=func)
    nf = len(case["f"])
    for a, b in ((0, 7), (7, 13), (13, nf), (3, 4)):
        part = dist._cuda_columns(*args, (a, b))
        assert np.array_equal(part, full[:, a:b], equal_nan=True)


@pytest.mark.parametrize("mode,merged,nr,nf", [(0, True, 2600, 4096), (3, True, 2600, 4096),
                                               (3, False, 2600, 4096), (0, True, 10000, 8192)])
def test_host_blocks_equal_device_path(ccfj, lib, mode, merged, nr, nf):
    """A host-memory transform large enough to run in frequency blocks (the
    upload of one block overlapping the transform of the previous one)
    gives the same bits as the same transform on device-resident inputs.
    2600 x 4096 complex spectra make 2 blocks; 10000 x 8192 make 16."""
    import torch
    from ccfj import _lib
    rng = np.random.default_rng(41)
    nc = 24
    r = np.sort(rng.uniform(1e3, 3e5, nr)).astype(np.float32)
    f = np.linspace(0.01, 1.5, nf).astype(np.float32)
    c = np.linspace(800.0, 4500.0, nc).astype(np.float32)
    uf = np.empty((nr, nf), dtype=np.complex64)
    uf.real = rng.standard_normal((nr, nf), dtype=np.float32)
    uf.imag = rng.standard_normal((nr, nf), dtype=np.float32)
    perm = rng.permutation(nr).astype(np.int64)
    flat = uf.view(np.float32)                       # (nr, 2 nf): Re, Im interleaved
    if merged:
        ins = [flat, flat[:, 1:]]                    # one region, Re and Im
        ld, es = 2 * nf, 2
    else:
        ins = [np.ascontiguousarray(flat[:, 0::2]), np.ascontiguousarray(flat[:, 1::2])]
        ld, es = nf, 1

    def args(us, rp, fp, cp, pp, outp, device):
        a = _lib.FjArgs()
        a.struct_size = ctypes.sizeof(a)
        a.nr, a.nf, a.nc = nr, nf, nc
        a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = 1, mode, 0, 1, int(device)
        a.u[0] = us[0]
        a.u[1] = us[1] if mode == 3 else None
        a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = ld, nr, es, nf, 1
        a.perm, a.r, a.f, a.c, a.out = pp, rp, fp, cp, outp
        return a

    out_h = np.empty((nc, nf), dtype=np.float32)
    a = args([x.ctypes.data for x in ins], r.ctypes.data, f.ctypes.data, c.ctypes.data,
             perm.ctypes.data, out_h.ctypes.data, False)
    _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), None))
    T = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda()
         for k, v in dict(r=r, f=f, c=c, perm=perm).items()}
    if merged:
        dflat = torch.from_numpy(flat).cuda()
        us = [dflat.data_ptr(), dflat.data_ptr() + 4]
        keep = [dflat]
    else:
        keep = [torch.from_numpy(x).cuda() for x in ins]
        us = [t.data_ptr() for t in keep]
    out_d = torch.empty((nc, nf), device="cuda")
    a = args(us, T["r"].data_ptr(), T["f"].data_ptr(), T["c"].data_ptr(), T["perm"].data_ptr(),
             out_d.data_ptr(), True)
    _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), None))
    torch.cuda.synchronize()
    assert np.array_equal(out_h, out_d.cpu().numpy(), equal_nan=True)


@pytest.mark.parametrize("func", [0, 1])
@pytest.mark.parametrize("zero_pair", [False, True])
def test_wide_velocity_range(ccfj, func, zero_pair):
    """Velocities over two decades (100-10000 m/s) at up to 2 Hz: k dr spans
    the Hermite rule, folded intervals with closed-form corrections and
    intervals left out of the fold, in one transform. With zero_pair, one
    pair sits at zero distance (the J basis is finite there; the Y basis of
    func 1 is singular at r = 0 and left out of that case)."""
    if zero_pair and func == 1:
        pytest.skip("Y0 is singular at r = 0")
    rng = np.random.default_rng(77)
    r = np.sort(rng.uniform(50.0, 8e4, 90))
    if zero_pair:
        r[0] = 0.0
    f = np.linspace(0.02, 2.0, 36)
    c = np.geomspace(100.0, 1e4, 70)
    uf = cases.noise_spectra(rng, r, f, sigma=0.2, overtone=True)
    y = _quiet(ccfj.fj_noise, uf, r, c, f, itype=1, func=func)
    y64 = _quiet(O.fj_noise, uf, r, c, f, itype=1, func=func)
    assert np.array_equal(np.isnan(y), np.isnan(y64))
    assert O.rel_error(y, y64) <= TOL


@pytest.mark.parametrize("npts", [1024, 2048, 4096, 16384])
def test_fj_earthquake_long_traces(ccfj, npts):
    """Traces long enough for the 16-points-per-thread Stockham FFT (512 to
    8192 complex points; the radix-16 passes end in a radix-2, 4, 8 or 16
    pass): the spectra feed a transform that matches the FP64 oracle, whose
    front end is numpy's rfft."""
    rng = np.random.default_rng(npts)
    Fs, ntr = 10.0, 12
    r = np.exp(rng.uniform(np.log(2e4), np.log(4e5), ntr))
    u = cases.ricker_records(rng, r, npts, Fs)
    nf = 40
    f = Fs * np.arange(nf) / npts
    c = np.linspace(2000, 5000, 30)
    y = _quiet(ccfj.fj_earthquake, u, r, c, f, itype=1, func=0)
    y64 = O._normalize(O.fj_earthquake(u, r, c, f, itype=1, func=0, normalize=False))
    assert np.array_equal(np.isnan(y), np.isnan(y64))
    assert O.rel_error(y, y64) <= TOL


@pytest.mark.parametrize("func", [0, 1])
def test_mwfj_long_traces(ccfj, func):
    """MWFJ on 16384-sample traces (the Stockham FFT of every tapered window;
    func 0 takes the tensor-core contraction, func 1 the CUDA-core one)."""
    rng = np.random.default_rng(91)
    npts, Fs, ntr, nwin = 16384, 10.0, 8, 8
    r = np.exp(rng.uniform(np.log(5e3), np.log(1.5e6), ntr))
    L = rng.integers(200, 2001, size=(nwin, ntr))
    start = rng.integers(0, npts - L)
    winl, winr = start / Fs, (start + L) / Fs
    u = cases.ricker_records(rng, r, npts, Fs)
    f = Fs * np.arange(32) / npts
    c = np.linspace(1500, 5000, 24)
    y = _quiet(ccfj.MWFJ, u, r, c, f, Fs, nwin, winl, winr, taper=0.9, func=func)
    y64 = np.stack([O._normalize(o) for o in O.MWFJ(u, r, c, f, Fs, nwin, winl, winr,
                                                   taper=0.9, func=func, normalize=False)])
    for w in range(nwin):
        assert np.array_equal(np.isnan(y[w]), np.isnan(y64[w]))
        assert O.rel_error(y[w], y64[w]) <= TOL


@pytest.mark.parametrize("ncols,fstride", [(1024, 1), (2048, 2), (600, 1)])
def test_func1_long_rows(ccfj, ncols, fstride):
    """fj_noise func=1 on rows of 1024 and 2048 columns (the Hilbert
    transform by FFT, two rows per CTA; 21 pairs leave the last row without
    a partner) and of 600 columns (the direct convolution), against the
    FP64 oracle built on scipy.fftpack.hilbert."""
    rng = np.random.default_rng(ncols)
    nr = 21
    r = rng.uniform(2e3, 6e4, nr)
    ff = np.linspace(0.01, 1.2, ncols)
    uf = cases.noise_spectra(rng, r, ff, sigma=0.2)
    f = ff[::fstride]
    c = np.linspace(1200, 4800, 8)
    y = _quiet(ccfj.fj_noise, uf, r, c, f, fstride=fstride, itype=1, func=1)
    y64 = _quiet(O.fj_noise, uf, r, c, f, fstride=fstride, itype=1, func=1)
    assert np.array_equal(np.isnan(y), np.isnan(y64))
    assert O.rel_error(y, y64) <= TOL


@pytest.mark.parametrize("taper", [1.2, -1.5])
def test_mwfj_degenerate_windows(ccfj, taper):
    """Windows that end before they start (one before 0 s) with tapers
    outside [0, 1]: the reference's win then writes ramp values outside the
    window, and from a negative end at the end of the array. The device
    taper reproduces them; every window matches the FP64 oracle (whose win
    is the reference's)."""
    from ccfj import _eq
    rng = np.random.default_rng(61)
    npts, Fs, ntr, nwin = 256, 10.0, 10, 3
    r = np.exp(rng.uniform(np.log(5e3), np.log(1.5e5), ntr))
    winl = rng.uniform(8.0, 16.0, (nwin, ntr))
    winr = winl + rng.uniform(-6.0, 4.0, (nwin, ntr))
    winr[0, 0] = -0.8                                 # ends before 0 s
    for _ in range(100):                              # keep only windows win accepts
        try:
            _eq._win_params(npts, Fs, winl, winr, taper)
            break
        except IndexError:
            winr = winl + rng.uniform(-6.0, 4.0, (nwin, ntr))
    u = cases.ricker_records(rng, r, npts, Fs)
    f = Fs * np.arange(24) / npts
    c = np.linspace(1500, 5000, 20)
    y = _quiet(ccfj.MWFJ, u, r, c, f, Fs, nwin, winl, winr, taper=taper)
    y64 = np.stack([O._normalize(o) for o in O.MWFJ(u, r, c, f, Fs, nwin, winl, winr,
                                                   taper=taper, normalize=False)])
    for w in range(nwin):
        assert np.array_equal(np.isnan(y[w]), np.isnan(y64[w]))
        assert O.rel_error(y[w], y64[w]) <= TOL
