"""Kernel variants and the autotuners on the device.

* Every velocities-per-thread variant (1, 2, 4) of the single-set kernel,
  for itype 0 and 1 and func 0 and 1, gives the default variant's result
  (the parity tests run only the defaults).
* ccfj_autotune_fj_v1 and ccfj_autotune_batch_v1 return a variant and a
  time, and a later variant-0 batch call gives the untuned result.
* The batch graph cache keeps 16 graphs: 18 distinct argument sets evict
  the oldest, and an evicted set is captured again, every output equal to
  the host-memory call bit for bit.
"""
import ctypes
import os
import warnings

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu
VAR_TOL = 2e-5
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _err(y, ref):
    assert np.array_equal(np.isnan(y), np.isnan(ref))
    return float(np.nanmax(np.abs(y - ref)) / np.nanmax(np.abs(ref)))


@pytest.mark.parametrize("itype", [0, 1])
@pytest.mark.parametrize("func", [0, 1])
@pytest.mark.parametrize("nc", [None, 37])
def test_single_set_variants_agree(lib, itype, func, nc):
    """nc = 37 leaves a partial velocity tile for every variant (37 is not a
    multiple of 8 rows x 1, 2 or 4 velocities per thread)."""
    import ccfj
    case = cases.noise_case("noise_small")
    c = case["c"] if nc is None else np.linspace(900.0, 4800.0, nc)
    args = (case["uf"], case["r"], c, case["f"])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        base = ccfj.fj_noise(*args, itype=itype, func=func)
        try:
            for v in (1, 2, 4):
                assert lib.ccfj_set_fj_variant(v) == 0
                assert _err(ccfj.fj_noise(*args, itype=itype, func=func), base) <= VAR_TOL, v
        finally:
            lib.ccfj_set_fj_variant(0)


def _device_batch(torch):
    """A seven-set batch (2 to 120 pairs) on the device, and the host-memory
    call's result for it."""
    import ccfj
    from ccfj import _batch
    rng = np.random.default_rng(3)
    f = np.linspace(0.02, 0.8, 40)
    c = np.linspace(1500, 4500, 37)
    ufs, rs = [], []
    for n in (50, 3, 120, 7, 64, 2, 31):
        r = rng.uniform(1e3, 4e4, n)
        ufs.append(cases.noise_spectra(rng, r, f))
        rs.append(r)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ref = np.stack(ccfj.fj_noise_batch(ufs, rs, c, f))
    off = np.concatenate([[0], np.cumsum([len(r) for r in rs])]).astype(np.int64)
    perm = np.concatenate([off[b] + np.argsort(r) for b, r in enumerate(rs)]).astype(np.int64)
    rsorted = np.concatenate([np.sort(r) for r in rs]).astype(np.float32)
    U = np.concatenate(ufs, axis=0)
    T = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
        u=U.view(np.float32), off=off, perm=perm, r=rsorted, f=f.astype(np.float32),
        c=c.astype(np.float32)).items()}
    torch.cuda.synchronize()

    def args(out, use_graph=0, variant=0):
        a = _batch.BatchArgs()
        a.struct_size = ctypes.sizeof(a)
        a.nsets, a.nf, a.nc = len(rs), len(f), len(c)
        a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = 1, 0, 0, 1, 1
        a.use_graph, a.variant = use_graph, variant
        a.offsets, a.total_pairs = T["off"].data_ptr(), int(off[-1])
        a.r, a.u[0] = T["r"].data_ptr(), T["u"].data_ptr()
        a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = 2 * len(f), U.shape[0], 2, len(f), 1
        a.perm, a.f, a.c, a.out = T["perm"].data_ptr(), T["f"].data_ptr(), T["c"].data_ptr(), \
            out.data_ptr()
        return a

    return args, ref, T


def test_batch_graph_cache_evicts_and_recaptures(lib):
    import torch
    from ccfj import _lib
    args, ref, _T = _device_batch(torch)
    outs = [torch.empty(ref.shape, device="cuda") for _ in range(18)]
    torch.cuda.synchronize()
    try:
        for o in outs:                       # 18 argument sets: two are evicted
            _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(args(o, use_graph=1)), None))
        _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(args(outs[0], use_graph=1)), None))
        torch.cuda.synchronize()
        for o in outs:
            assert np.array_equal(o.cpu().numpy(), ref, equal_nan=True)
    finally:
        torch.cuda.synchronize()
        assert lib.ccfj_batch_graph_cache_clear() == 0


def test_batch_graph_null_stream_is_ordered(lib):
    """A graph replay requested on the legacy default stream (NULL) runs
    after the default-stream work queued before the call and before the
    work queued after it, with no host synchronisation in between."""
    import torch
    from ccfj import _lib
    assert torch.cuda.current_stream().cuda_stream == 0
    args, ref, T = _device_batch(torch)
    out = torch.empty(ref.shape, device="cuda")
    try:
        _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(args(out, use_graph=1)), None))  # capture
        torch.cuda.synchronize()
        u_true = T["u"].clone()
        T["u"].zero_()
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        for _ in range(3):
            torch.cuda._sleep(20_000_000)        # default stream busy for several ms
            T["u"].copy_(u_true)                 # the inputs arrive only after that
            _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(args(out, use_graph=1)), None))
            got = out.clone()                    # default-stream work after the call
            T["u"].zero_()
            torch.cuda.synchronize()
            assert np.array_equal(got.cpu().numpy(), ref, equal_nan=True)
    finally:
        torch.cuda.synchronize()
        assert lib.ccfj_batch_graph_cache_clear() == 0


def test_batch_autotuner(lib):
    import torch
    from ccfj import _lib
    args, ref, _T = _device_batch(torch)
    out = torch.empty(ref.shape, device="cuda")
    best, ms = ctypes.c_int(), ctypes.c_float()
    _lib.check(lib.ccfj_autotune_batch_v1(ctypes.byref(args(out)), None, ctypes.byref(best),
                                          ctypes.byref(ms)))
    assert best.value in (1, 2, 4) and ms.value > 0
    for v in (0, 1, 2, 4):                   # 0: the tuned choice
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        _lib.check(lib.ccfj_fj_batch_v1(ctypes.byref(args(out, variant=v)), None))
        torch.cuda.synchronize()
        assert _err(out.cpu().numpy(), ref) <= VAR_TOL, v


def test_single_set_autotuner(lib):
    import torch
    from ccfj import _lib
    case = cases.noise_case("noise_small")
    idx = np.argsort(case["r"])
    nr, nf, nc = len(case["r"]), len(case["f"]), len(case["c"])
    T = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
        u=np.ascontiguousarray(case["uf"]).view(np.float32), perm=idx.astype(np.int64),
        r=case["r"][idx].astype(np.float32), f=case["f"].astype(np.float32),
        c=case["c"].astype(np.float32)).items()}
    out = torch.empty((nc, nf), device="cuda")
    torch.cuda.synchronize()
    a = _lib.FjArgs()
    a.struct_size = ctypes.sizeof(a)
    a.nr, a.nf, a.nc = nr, nf, nc
    a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = 1, _lib.MODE_J, 0, 1, 1
    a.u[0] = T["u"].data_ptr()
    a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = 2 * nf, nr, 2, nf, 1
    a.perm, a.r, a.f, a.c = (T[k].data_ptr() for k in ("perm", "r", "f", "c"))
    a.out = out.data_ptr()
    best, ms = ctypes.c_int(), ctypes.c_float()
    _lib.check(lib.ccfj_autotune_fj_v1(ctypes.byref(a), None, ctypes.byref(best),
                                       ctypes.byref(ms)))
    assert best.value in (1, 2, 4) and ms.value > 0


def _mid_case():
    """300 pairs (1-50 km) x 64 f x 70 c: few CTAs, enough stations for
    8 ranges of 32."""
    rng = np.random.default_rng(21)
    r = rng.uniform(1e3, 5e4, 300)
    f = np.linspace(0.02, 1.0, 64)
    c = np.linspace(1000.0, 5000.0, 70)
    return cases.noise_spectra(rng, r, f, sigma=0.1), r, c, f


@pytest.mark.parametrize("itype,func", [(1, 0), (1, 1), (0, 0)])
@pytest.mark.parametrize("nsplit", [2, 3, 8])
def test_split_launch_matches_unsplit_and_oracle(lib, itype, func, nsplit):
    """Station ranges summed in a fixed order: the same spectrum as the
    unsplit launch (to rounding), within 1e-4 of the FP64 oracle, and the
    same bits on a second run."""
    import ccfj
    import fj_oracle as O
    uf, r, c, f = _mid_case()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        try:
            assert lib.ccfj_set_fj_split(1) == 0
            base = ccfj.fj_noise(uf, r, c, f, itype=itype, func=func)
            assert lib.ccfj_set_fj_split(nsplit) == 0
            y = ccfj.fj_noise(uf, r, c, f, itype=itype, func=func)
            y2 = ccfj.fj_noise(uf, r, c, f, itype=itype, func=func)
        finally:
            lib.ccfj_set_fj_split(0)
        y64 = O.fj_noise(uf, r, c, f, itype=itype, func=func)
    assert _err(y, base) <= 1e-5
    assert O.rel_error(y, y64) <= 1e-4
    assert np.array_equal(y, y2)


def test_tuned_choice_is_reused_by_another_process(tmp_path):
    """The autotuner writes its choice to the table named by
    CCFJ_TUNE_CACHE; a second process reads it back for the same class."""
    import subprocess
    import sys
    cache = tmp_path / "tune.txt"
    prog = r'''
import ctypes, sys, numpy as np, torch
sys.path[:0] = [%r, %r]
import cases
from ccfj import _lib
lib = _lib.load()
rng = np.random.default_rng(21)
r = np.sort(rng.uniform(1e3, 5e4, 300)); f = np.linspace(0.02, 1.0, 64)
c = np.linspace(1000.0, 5000.0, 70); uf = cases.noise_spectra(rng, r, f, sigma=0.1)
T = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(
    u=uf.view(np.float32), r=r.astype(np.float32), f=f.astype(np.float32),
    c=c.astype(np.float32)).items()}
out = torch.empty((70, 64), device="cuda")
a = _lib.FjArgs(); a.struct_size = ctypes.sizeof(a)
a.nr, a.nf, a.nc, a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = 300, 64, 70, 1, 0, 0, 1, 1
a.u[0] = T["u"].data_ptr(); a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = 128, 300, 2, 64, 1
a.r, a.f, a.c, a.out = T["r"].data_ptr(), T["f"].data_ptr(), T["c"].data_ptr(), out.data_ptr()
cpt, ns = ctypes.c_int(), ctypes.c_int()
if sys.argv[1] == "tune":
    ms = ctypes.c_float()
    _lib.check(lib.ccfj_autotune_fj_v1(ctypes.byref(a), None, ctypes.byref(cpt), ctypes.byref(ms)))
_lib.check(lib.ccfj_tuned_choice_fj(ctypes.byref(a), ctypes.byref(cpt), ctypes.byref(ns)))
print(cpt.value, ns.value)
''' % (os.path.join(REPO, "cc-fjpy_b200"), os.path.join(REPO, "tests"))
    env = dict(os.environ, CCFJ_TUNE_CACHE=str(cache))
    first = subprocess.run([sys.executable, "-c", prog, "tune"], env=env, capture_output=True,
                           text=True, timeout=600)
    assert first.returncode == 0, first.stderr
    second = subprocess.run([sys.executable, "-c", prog, "query"], env=env, capture_output=True,
                            text=True, timeout=600)
    assert second.returncode == 0, second.stderr
    assert first.stdout.split() == second.stdout.split()
    line = [ln for ln in cache.read_text().splitlines() if ln.startswith("ccfj-tune-v1 ")]
    assert len(line) == 1 and " fj " in line[0]
    cpt, ns = (int(v) for v in second.stdout.split())
    assert int(line[0].split()[4]) == cpt + 8 * ns
