"""Parity at the benchmark's full sizes.

The other GPU tests use small seeded cases; these run the benchmark
workloads themselves through the public API and check
  * sampled frequency columns of the large-array workload (19,900 pairs x
    2048 f x 1000 c) and of the earthquake workload (500 traces x 8192
    samples, 1024 bins x 800 c) against the FP64 oracle, and against the
    reference's own FJcpu.cpp where its CPU build (make -C oracle) is present;
  * every window of the MWFJ workload (1000 traces x 16384 samples, 64
    windows, 1024 bins x 2000 c; tensor cores, scaled FP16x3) against the FP64 GPU
    form, and two (window, bin) columns against the oracle;
  * every subarray of a 64-subarray ragged batch against the FP64 GPU form.
Every frequency column is independent of the others (its normalisation
included), so a column of the full call can be checked alone. Tolerance:
1e-4 of each column's largest value against FP64 forms; against FJcpu.cpp,
FJcpu's own error against the oracle plus 1e-4.
"""
import multiprocessing
import os
import sys
import warnings

import numpy as np
import pytest

import fj_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-4
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    import bench
    return bench


@pytest.fixture(scope="module")
def pool():
    # spawned workers hold no CUDA state (a fork after CUDA initialisation hangs)
    with multiprocessing.get_context("spawn").Pool(4) as p:
        yield p


def _reference():
    try:
        return _bench().reference_module()
    except ImportError:
        return None


def _check_fjcpu(y_cols, ref_cols, oracle_cols):
    own = max(O.rel_error(ref_cols[:, [j]], o) for j, o in enumerate(oracle_cols))
    err = O.rel_error(y_cols, ref_cols)
    assert err <= own + TOL, (err, own)


def test_large_array_columns(pool):
    import ccfj
    b = _bench()
    uf, r, f, c = b.workload()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        y = ccfj.fj_noise(uf, r, c, f)
    cols = np.linspace(0, b.NF - 1, 4).round().astype(int)
    jobs = [("noise", dict(uf=uf[:, [k]], r=r, c=c, f=f[[k]])) for k in cols]
    outs = pool.map(b._oracle_job, jobs)
    for k, o in zip(cols, outs):
        assert O.rel_error(y[:, [k]], o) <= TOL, k
    ref = _reference()
    if ref is not None:
        _, ro = b.ref_noise_cols(ref, uf, r, c, f, cols, os.cpu_count() or 1)
        _check_fjcpu(y[:, cols], ro, outs)


def test_earthquake_columns(pool):
    import ccfj
    b = _bench()
    u, r, f, c = b.workload_eq()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        y = ccfj.fj_earthquake(u, r, c, f)
    assert np.all(np.isnan(y[:, 0])) and not np.any(np.isnan(y[:, 1:]))  # f = 0: k = 0
    cols = np.linspace(1, len(f) - 1, 4).round().astype(int)
    jobs = [("eq", dict(u=u, r=r, c=c, f=f, cols=[k])) for k in cols]
    outs = pool.map(b._oracle_job, jobs)
    for k, o in zip(cols, outs):
        assert O.rel_error(y[:, [k]], o) <= TOL, k
    ref = _reference()
    if ref is not None:
        _, _, ro = b.ref_eq_cols(ref, u, r, c, f, cols, os.cpu_count() or 1)
        _check_fjcpu(y[:, cols], ro, outs)


def test_mwfj_every_window(pool):
    """Scaled FP16x3 tensor-core MWFJ: all 64 windows against the FP64 form."""
    import ccfj
    from ccfj import _eq, _lib
    b = _bench()
    wl = b.workload_mwfj()
    u, r, f, c = wl["u"], wl["r"], wl["f"], wl["c"]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        y = ccfj.MWFJ(u, r, c, f, wl["Fs"], wl["nwin"], wl["winl"], wl["winr"], wl["taper"])
        n1, n2, dl = _eq._win_params(u.shape[1], wl["Fs"], wl["winl"], wl["winr"], wl["taper"])
        wins = tuple(np.ascontiguousarray(x, dtype=np.int32) for x in (n1, n2, dl))
        y64 = _eq._run(u, r, c, f, 1, 1, 0, nwin=wl["nwin"], wins=wins,
                       precision=_lib.PREC_FP64)
    assert y.shape == (64, 2000, 1024) and y.dtype == np.float64
    errs = [O.rel_error(y[w], y64[w]) for w in range(wl["nwin"])]
    assert max(errs) <= TOL, (int(np.argmax(errs)), max(errs))
    assert np.array_equal(np.isnan(y), np.isnan(y64))
    picks = [(7, 100), (50, 900)]
    jobs = [("mwfj", dict(u=u, r=r, c=c, f=f, Fs=wl["Fs"], winl=wl["winl"][w],
                          winr=wl["winr"][w], cols=[k], taper=wl["taper"])) for w, k in picks]
    for (w, k), o in zip(picks, pool.map(b._oracle_job, jobs)):
        assert O.rel_error(y[w][:, [k]], o) <= TOL, (w, k)


def test_ragged_batch_every_subarray():
    """64 subarrays (50-20,000 pairs each, log-uniform) in one persistent
    launch: every subarray against the FP64 form of the single-set
    transform."""
    import cases
    import ccfj
    from ccfj import _lib
    b = _bench()
    counts, off = b.batch_counts(seed=15, nsets=64)
    rng = np.random.default_rng(15)
    f = np.linspace(0.01, 1.0, 256)
    c = np.linspace(1000.0, 5000.0, 500)
    rs = [rng.uniform(500.0, 3e5, int(n)) for n in counts]
    ufs = [cases.noise_spectra(rng, rb, f, sigma=0.2, overtone=True) for rb in rs]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ys = ccfj.fj_noise_batch(ufs, rs, c, f)
        for rb, ub, yb in zip(rs, ufs, ys):
            idx = np.argsort(rb)
            y64 = ccfj._transform([ub], rb[idx], c, f, 1, 1, _lib.MODE_J, perm=idx,
                                  normalize=True, precision=_lib.PREC_FP64)
            assert O.rel_error(yb, y64) <= TOL, len(rb)
