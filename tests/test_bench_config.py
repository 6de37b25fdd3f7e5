"""The benchmark's headline workload is the large-array configuration the
metric is quoted on: 19,900 pairs (all pairs of 200 stations placed
uniformly in a 300 x 300 km box), 2048 frequencies over 0.005-2 Hz, 1000
velocities over 500-5000 m/s, complex64 spectra from the c(f) law with a
first overtone and sigma = 0.2 noise. No GPU: the generator is numpy."""
import importlib
import os
import sys

import numpy as np

from conftest import REPO


def _bench():
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    return importlib.import_module("bench")


def test_headline_workload_shapes_and_grids():
    bench = _bench()
    uf, r, f, c = bench.workload()
    assert (bench.NPAIRS, bench.NF, bench.NC) == (19900, 2048, 1000)
    assert uf.shape == (19900, 2048) and uf.dtype == np.complex64
    assert r.shape == (19900,) and r.dtype == np.float64
    assert 0 < r.min() and r.max() <= np.hypot(3e5, 3e5)
    assert np.array_equal(f, np.linspace(0.005, 2.0, 2048))
    assert np.array_equal(c, np.linspace(500.0, 5000.0, 1000))
    # 200 stations: every distance is a pair of the same 200 points
    n = int((1 + np.sqrt(1 + 8 * len(r))) / 2)
    assert n * (n - 1) // 2 == len(r) == 19900


def test_headline_workload_is_seeded():
    bench = _bench()
    a, b = bench.workload(), bench.workload()
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_config_names_the_workload():
    cfg = _bench().config_dict()
    assert (cfg["npairs"], cfg["nf"], cfg["nc"], cfg["itype"], cfg["func"]) == (19900, 2048, 1000,
                                                                                 1, 0)
    assert "workload" in cfg and "l2" in cfg
    assert os.path.exists(os.path.join(REPO, "bench.py"))


def _ref_module():
    import pytest
    bench = _bench()
    try:
        return bench, bench.reference_module()
    except ImportError:
        pytest.skip("the reference's CPU build (make -C oracle) is not present")


def test_reference_column_samples_equal_full_calls():
    """The CPU baseline's column samples reproduce the reference's own full
    calls on those columns: fj_noise, fj_earthquake and one MWFJ window."""
    import cases
    bench, ref = _ref_module()
    import warnings
    warnings.simplefilter("ignore")
    n = cases.noise_case("noise_small")
    full = ref.fj_noise(n["uf"], n["r"], n["c"], n["f"], num=2)
    cols = np.array([3, 9, 30])
    _, o = bench.ref_noise_cols(ref, n["uf"], n["r"], n["c"], n["f"], cols, 2)
    assert np.array_equal(o, full[:, cols], equal_nan=True)
    e = cases.eq_case("eq_small")
    full = ref.fj_earthquake(e["u"], e["r"], e["c"], e["f"], num=2)
    cols = np.array([0, 5, 17, 39])                      # bin 0: the NaN column
    _, _, o = bench.ref_eq_cols(ref, e["u"], e["r"], e["c"], e["f"], cols, 2)
    assert np.array_equal(o, full[:, cols], equal_nan=True)
    m = cases.mwfj_case("mwfj_small")
    full = ref.MWFJ(m["u"], m["r"], m["c"], m["f"], m["Fs"], m["nwin"], m["winl"], m["winr"],
                    m["taper"], num=2)
    wl = {k: m[k] for k in ("u", "r", "c", "f", "Fs", "winl", "winr", "taper")}
    cols = np.array([1, 7, 20])
    _, _, o = bench.ref_mwfj_window_cols(ref, wl, 2, cols, 2)
    assert np.allclose(o, full[2][:, cols], rtol=0, atol=0)


def test_column_sets_cover_the_band_evenly():
    bench = _bench()
    sets = bench.column_sets(2048, 16, 20)
    allc = np.sort(np.concatenate(sets))
    assert len(sets) == 20 and all(len(s) == 16 for s in sets)
    assert len(np.unique(allc)) == 320 and allc[0] == 0 and allc[-1] == 2047
    gaps = np.diff(allc)
    assert gaps.max() - gaps.min() <= 1                  # evenly spaced
    for s in sets:                                      # each step spans the band
        assert s.min() < 128 and s.max() > 1900


def test_oracle_column_helpers_equal_full_oracle():
    import cases
    import fj_oracle as O
    e = cases.eq_case("eq_small")
    full = O.fj_earthquake(e["u"], e["r"], e["c"], e["f"])
    cols = [0, 3, 17, 39]
    sub = O.fj_earthquake_columns(e["u"], e["r"], e["c"], e["f"], cols)
    assert np.array_equal(sub, full[:, cols], equal_nan=True)
    m = cases.mwfj_case("mwfj_small")
    full = O.MWFJ(m["u"], m["r"], m["c"], m["f"], m["Fs"], m["nwin"], m["winl"], m["winr"],
                  m["taper"])
    sub = O.mwfj_window_columns(m["u"], m["r"], m["c"], m["f"], m["Fs"], m["winl"][1],
                                m["winr"][1], [2, 5, 9], m["taper"])
    assert np.array_equal(sub, full[1][:, [2, 5, 9]], equal_nan=True)


def test_batch_fjcpu_check_uses_the_compared_columns():
    """Configuration 5's check of FJcpu.cpp: our columns are compared with
    FJcpu's on the CPU sample's columns, so FJcpu's own error is taken on the
    same columns (against the FP64 form) as well as on the oracle's."""
    bench = _bench()
    rng = np.random.default_rng(0)
    # normalised columns, as the transforms return them (largest |value| 1)
    y64 = rng.uniform(-0.5, 0.5, (5, 6))
    y64[0] = 1.0
    ours = y64 + 1e-7
    fjcpu = y64.copy()
    fjcpu[1] += 0.3  # FJcpu off by 0.3 of the column's largest value

    class Run:
        pass

    run = Run()
    run.res = {"accuracy": {}}
    run.gpu_cols, run.ref_out, run.y64_cols = ours, fjcpu, y64
    # one oracle column on which FJcpu happens to be accurate
    run.oracle_jobs = [(None, (slice(None), [2]))]
    oracle = [y64[:, [2]]]
    run.ref_out = run.ref_out.copy()
    run.ref_out[:, 2] = y64[:, 2]
    acc = bench.finish_batch(run, oracle)["accuracy"]
    assert acc["fjcpu_err_vs_oracle"] < 1e-12
    assert abs(acc["fjcpu_err_vs_fp64"] - 0.3) < 1e-9
    assert acc["fjcpu_check"].endswith("True")
