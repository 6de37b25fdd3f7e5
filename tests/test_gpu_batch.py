"""The ragged batch (many subarrays, one persistent launch) equals fj_noise
called once per subarray, and matches the FP64 oracle.

The batch and the single-set kernels run the same cell loop but are
separate kernels, and the code generator may fuse a multiply and an add
into one FMA in one of them and not in the other; so they agree to FP32
rounding (SAME_TOL on the normalised spectra, with identical NaN
positions), not bit for bit."""
import ctypes
import warnings

import numpy as np
import pytest

import cases
import fj_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-4
SAME_TOL = 2e-6


def _sets(seed, nsets, lo, hi, f):
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), nsets)).astype(int)
    ufs, rs = [], []
    for n in counts:
        r = rng.uniform(500.0, 3e5, n)
        rs.append(r)
        ufs.append(cases.noise_spectra(rng, r, f, sigma=0.2, overtone=True))
    return ufs, rs


@pytest.mark.parametrize("itype", [0, 1])
@pytest.mark.parametrize("func", [0, 1])
def test_batch_equals_per_set_calls(itype, func):
    import ccfj
    f = np.linspace(0.01, 1.0, 24)
    c = np.linspace(1000, 5000, 20)
    ufs, rs = _sets(5, 9, 2, 300, f)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        outs = ccfj.fj_noise_batch(ufs, rs, c, f, itype=itype, func=func)
        for uf, r, y in zip(ufs, rs, outs):
            single = ccfj.fj_noise(uf, r, c, f, itype=itype, func=func)
            assert np.array_equal(np.isnan(y), np.isnan(single))
            assert np.nanmax(np.abs(y.astype(np.float64) - single)) <= SAME_TOL
            y64 = O.fj_noise(uf, r, c, f, itype=itype, func=func)
            assert O.rel_error(y, y64) <= TOL


@pytest.mark.parametrize("variant", [1, 2, 4])
def test_batch_variants_and_single_pair_set(variant):
    import ccfj
    f = np.linspace(0.02, 0.8, 40)
    c = np.linspace(1500, 4500, 37)
    ufs, rs = _sets(7, 6, 3, 120, f)
    ufs.append(ufs[0][:1])
    rs.append(rs[0][:1])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        outs = ccfj.fj_noise_batch(ufs, rs, c, f, variant=variant)
    for uf, r, y in zip(ufs[:-1], rs[:-1], outs[:-1]):
        assert O.rel_error(y, O.fj_noise(uf, r, c, f)) <= TOL
    # one pair: no interval, the reference's 0/0 normalisation gives NaN
    assert np.isnan(outs[-1]).all()


def test_batch_device_graph_replay(lib):
    """Device pointers with use_graph: the captured graph is replayed on a
    second call and gives the same bits as the host-memory call."""
    import torch
    import ccfj
    from ccfj import _batch, _lib
    f = np.linspace(0.01, 1.0, 32)
    c = np.linspace(1000, 5000, 25)
    ufs, rs = _sets(9, 11, 5, 200, f)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ref = np.stack(ccfj.fj_noise_batch(ufs, rs, c, f))
    counts = np.array([len(r) for r in rs])
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    perm = np.concatenate([off[b] + np.argsort(r) for b, r in enumerate(rs)]).astype(np.int64)
    rsorted = np.concatenate([np.sort(r) for r in rs]).astype(np.float32)
    U = np.concatenate(ufs, axis=0)
    T = {k: torch.from_numpy(v).cuda() for k, v in dict(
        u=U.view(np.float32), off=off, perm=perm, r=rsorted, f=f.astype(np.float32),
        c=c.astype(np.float32)).items()}
    a = _batch.BatchArgs()
    a.struct_size = ctypes.sizeof(a)
    a.nsets, a.nf, a.nc = len(rs), len(f), len(c)
    a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = 1, 0, 0, 1, 1
    a.use_graph = 1
    a.offsets, a.total_pairs = T["off"].data_ptr(), int(off[-1])
    a.r = T["r"].data_ptr()
    a.u[0] = T["u"].data_ptr()
    a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = 2 * len(f), U.shape[0], 2, len(f), 1
    a.perm, a.f, a.c = T["perm"].data_ptr(), T["f"].data_ptr(), T["c"].data_ptr()
    s = torch.cuda.Stream()
    out = torch.empty((len(rs), len(c), len(f)), device="cuda")
    a.out = out.data_ptr()
    outs = []
    for _ in range(2):  # same arguments: the second call replays the cached graph
        with torch.cuda.stream(s):
            out.fill_(float("nan"))
            _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(a), ctypes.c_void_p(s.cuda_stream)))
        s.synchronize()
        outs.append(out.cpu().numpy())
    assert lib.ccfj_batch_graph_cache_clear() == 0
    for y in outs:
        assert np.array_equal(y, ref, equal_nan=True)
