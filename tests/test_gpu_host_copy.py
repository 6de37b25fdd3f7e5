"""Large results and inputs copied between host memory and the device
(csrc/host_copy.cu).

Results of 16 MiB and more go to pageable host memory through pinned
staging buffers on several host threads; MWFJ's float64 result is converted
on the way. Checked here: the staged copy equals the device result read by
torch bit for bit, MWFJ's float64 result is exactly its float32 result
widened (staged and unstaged sizes), two calls that overlap on the host
(one takes the staging buffers, the other the plain route) both come back
right, a batch of 256 MB or more of host spectra, run in groups of sets
with the copies overlapping the transforms, equals one device-resident pass,
and large pageable inputs, staged the other way round, give the same bits as
pinned ones.
"""
import ctypes
import threading
import warnings

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def _noise_batch(nsets=8, nf=600, nc=1000, seed=21):
    rng = np.random.default_rng(seed)
    f = np.linspace(0.02, 0.8, nf)
    c = np.linspace(1500.0, 4500.0, nc)
    rs = [rng.uniform(1e3, 4e4, n) for n in rng.integers(5, 40, nsets)]
    ufs = [cases.noise_spectra(rng, r, f) for r in rs]
    return ufs, rs, c, f


def _device_batch(lib, ufs, rs, c, f):
    """The batch with every array on the device (one pass), read back by torch."""
    import torch
    from ccfj import _batch, _lib
    off = np.concatenate([[0], np.cumsum([len(r) for r in rs])]).astype(np.int64)
    perm = np.concatenate([off[b] + np.argsort(r) for b, r in enumerate(rs)]).astype(np.int64)
    rsorted = np.concatenate([np.sort(r) for r in rs]).astype(np.float32)
    U = np.concatenate(ufs, axis=0).astype(np.complex64)
    T = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
        u=U.view(np.float32), off=off, perm=perm, r=rsorted, f=f.astype(np.float32),
        c=c.astype(np.float32)).items()}
    out = torch.empty((len(rs), len(c), len(f)), device="cuda")
    a = _batch.BatchArgs()
    a.struct_size = ctypes.sizeof(a)
    a.nsets, a.nf, a.nc = len(rs), len(f), len(c)
    a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = 1, 0, 0, 1, 1
    a.offsets, a.total_pairs = T["off"].data_ptr(), int(off[-1])
    a.r, a.u[0] = T["r"].data_ptr(), T["u"].data_ptr()
    a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = 2 * len(f), U.shape[0], 2, len(f), 1
    a.perm, a.f, a.c, a.out = T["perm"].data_ptr(), T["f"].data_ptr(), T["c"].data_ptr(), \
        out.data_ptr()
    torch.cuda.synchronize()
    _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(a), None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_staged_copy_equals_device_result(lib):
    """19.2 MB of batch output: the host-memory call (staged copy) against the
    device-pointer call read back by torch."""
    import ccfj
    ufs, rs, c, f = _noise_batch()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        host = np.stack(ccfj.fj_noise_batch(ufs, rs, c, f))
    assert host.nbytes >= 16 << 20
    assert np.array_equal(_device_batch(lib, ufs, rs, c, f), host, equal_nan=True)


def test_pipelined_host_batch_equals_device_batch(lib):
    """328 MB of complex64 spectra from host memory run in groups of sets,
    the next group's copy overlapping the current group's transform; equal
    bit for bit to one device-resident pass over all sets."""
    import ccfj
    rng = np.random.default_rng(23)
    nf, nc = 1024, 16
    f = np.linspace(0.01, 1.0, nf)
    c = np.linspace(1500.0, 4500.0, nc)
    counts = rng.integers(1000, 4000, 16)
    counts[-1] += 40000 - counts.sum() if counts.sum() < 40000 else 0
    rs = [rng.uniform(1e3, 4e4, n) for n in counts]
    ufs = [cases.noise_spectra(rng, r, f) for r in rs]
    assert sum(u.nbytes for u in ufs) >= 256 << 20
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        host = np.stack(ccfj.fj_noise_batch(ufs, rs, c, f))
    assert np.array_equal(_device_batch(lib, ufs, rs, c, f), host, equal_nan=True)


@pytest.mark.parametrize("nwin,nc", [(16, 600), (8, 40)])
def test_mwfj_double_result_is_the_float_result_widened(nwin, nc):
    """(16, 600): 19.7 MB of float32 result, staged; (8, 40): plain."""
    import ccfj
    from ccfj import _eq
    rng = np.random.default_rng(7)
    ntr, npts, Fs, nf = 40, 2048, 10.0, 512
    r = np.exp(rng.uniform(np.log(5e3), np.log(2e5), ntr))
    u = cases.ricker_records(rng, r, npts, Fs)
    f = Fs * np.arange(nf) / npts
    c = np.linspace(1500.0, 5000.0, nc)
    L = rng.integers(200, 1001, size=(nwin, ntr))
    start = rng.integers(0, npts - L)
    winl, winr = start / Fs, (start + L) / Fs
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        y = ccfj.MWFJ(u, r, c, f, Fs, nwin, winl, winr, 0.9)
        n1, n2, dl = _eq._win_params(npts, Fs, winl, winr, 0.9)
        wins = tuple(np.ascontiguousarray(x, dtype=np.int32) for x in (n1, n2, dl))
        y32 = _eq._run(u, r, c, f, 1, 1, 0, nwin=nwin, wins=wins)
    assert y.dtype == np.float64 and y32.dtype == np.float32 and y.shape == (nwin, nc, nf)
    assert np.array_equal(y, y32.astype(np.float64), equal_nan=True)


def test_staged_input_equals_pinned_input():
    """20 MB of pageable traces reach the device through the threads'
    pinned staging; the same traces in pinned memory go in one plain copy.
    fj_earthquake gives the same bits either way."""
    import ccfj
    rng = np.random.default_rng(31)
    ntr, npts, Fs = 640, 8192, 20.0
    r = np.exp(rng.uniform(np.log(1e4), np.log(2e6), ntr))
    u = cases.ricker_records(rng, r, npts, Fs)
    assert u.dtype == np.float32 and u.nbytes >= 8 << 20
    f = Fs * np.arange(256) / npts
    c = np.linspace(2000.0, 5000.0, 64)
    pinned = ccfj.pinned_empty(u.shape, np.float32)
    pinned[...] = u
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        y_pageable = ccfj.fj_earthquake(u, r, c, f)
        y_pinned = ccfj.fj_earthquake(pinned, r, c, f)
    assert np.array_equal(y_pageable, y_pinned, equal_nan=True)


def test_overlapping_host_calls():
    """Four threads copy large results out at the same time: one holds the
    staging buffers, the others take the plain route; all are right."""
    import ccfj
    ufs, rs, c, f = _noise_batch(seed=22)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ref = np.stack(ccfj.fj_noise_batch(ufs, rs, c, f))
    got, errs = [None] * 4, []

    def work(i):
        try:
            with warnings.catch_warnings():
                warnings.simplefilter("ignore")
                got[i] = np.stack(ccfj.fj_noise_batch(ufs, rs, c, f))
        except Exception as e:  # reported below
            errs.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errs, errs
    for g in got:
        assert np.array_equal(g, ref, equal_nan=True)
