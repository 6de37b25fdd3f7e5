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
