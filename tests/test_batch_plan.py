"""The grouping of a large host-memory batch (csrc/batch_plan.h) without a
GPU: groups of consecutive sets ending at the first set boundary past 1/16,
1/4, 1/2, 3/4 and all of the pairs, rows disjoint and increasing; one pass
for small inputs, two-part inputs, a single set, or a permutation that mixes
sets. The device side (the pipelined batch equal to one device-resident
pass) is in tests/test_gpu_host_copy.py."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import REPO

BIG = 300 << 20  # input bytes above the pipelining size


@pytest.fixture(scope="module")
def bp(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    so = str(tmp_path_factory.mktemp("bp") / "libbp.so")
    subprocess.run([cxx, "-O1", "-std=c++17", "-shared", "-fPIC",
                    "-I", os.path.join(REPO, "cc-fjpy_b200", "csrc"),
                    os.path.join(REPO, "tests", "batch_plan_check.cpp"), "-o", so], check=True)
    lib = ctypes.CDLL(so)
    lib.bp_plan.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong,
                            ctypes.c_int, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_int]
    lib.bp_plan.restype = ctypes.c_int
    return lib


def _plan(bp, counts, perm=None, nin=1, ubytes=BIG):
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    out = np.zeros(4 * 16, dtype=np.int64)
    p = None if perm is None else np.ascontiguousarray(perm, dtype=np.int64)
    n = bp.bp_plan(off.ctypes.data, len(counts), None if p is None else p.ctypes.data,
                   int(off[-1]), nin, ubytes, out.ctypes.data, 16)
    return [tuple(int(v) for v in out[4 * i:4 * i + 4]) for i in range(n)], off


def test_equal_sets(bp):
    groups, _ = _plan(bp, [100] * 16)
    assert [(b0, b1) for b0, b1, _, _ in groups] == [(0, 1), (1, 4), (4, 8), (8, 12), (12, 16)]
    assert [(lo, hi) for _, _, lo, hi in groups] == [(0, 99), (100, 399), (400, 799),
                                                     (800, 1199), (1200, 1599)]


def test_one_large_set_first(bp):
    groups, _ = _plan(bp, [10000, 10, 10])
    assert [(b0, b1) for b0, b1, _, _ in groups] == [(0, 1), (1, 2), (2, 3)]


@pytest.mark.parametrize("seed", range(5))
def test_groups_cover_every_set_once_with_increasing_rows(bp, seed):
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(50), np.log(20000), 64)).astype(np.int64)
    groups, off = _plan(bp, counts)
    assert 2 <= len(groups) <= 5
    assert groups[0][0] == 0 and groups[-1][1] == len(counts)
    for (a0, a1, alo, ahi), (b0, b1, blo, bhi) in zip(groups, groups[1:]):
        assert a1 == b0 and ahi < blo
    for b0, b1, lo, hi in groups:
        assert (lo, hi) == (off[b0], off[b1] - 1)
    # a permutation within each set (the wrapper's argsort) reads the same rows
    perm = np.concatenate([off[b] + rng.permutation(int(n)) for b, n in enumerate(counts)])
    assert _plan(bp, counts, perm)[0] == groups


def test_one_pass_cases(bp):
    assert _plan(bp, [100] * 16, ubytes=(256 << 20) - 1)[0] == []   # small input
    assert _plan(bp, [100] * 16, nin=2)[0] == []                    # two-part input
    assert _plan(bp, [1600])[0] == []                               # one set
    perm = np.arange(1600)
    perm[[0, 1599]] = perm[[1599, 0]]                               # sets mixed
    assert _plan(bp, [100] * 16, perm)[0] == []
