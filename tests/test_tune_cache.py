"""The autotuners' persistent table (csrc/tune_cache.h) without a GPU:
round trip, replacement of a (device, tuner, class) line, device names with
blanks, and lines the reader must ignore. The GPU side -- a tuned choice
written by one process and used by another -- is in
tests/test_gpu_variants.py."""
import ctypes
import os
import shutil
import subprocess

import pytest

from conftest import REPO


@pytest.fixture(scope="module")
def tc(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    so = str(tmp_path_factory.mktemp("tc") / "libtc.so")
    subprocess.run([cxx, "-O1", "-std=c++17", "-shared", "-fPIC",
                    "-I", os.path.join(REPO, "cc-fjpy_b200", "csrc"),
                    os.path.join(REPO, "tests", "tune_cache_check.cpp"), "-o", so], check=True)
    lib = ctypes.CDLL(so)
    lib.tc_upsert.argtypes = [ctypes.c_char_p] * 3 + [ctypes.c_longlong, ctypes.c_int,
                                                      ctypes.c_float]
    lib.tc_lookup.argtypes = [ctypes.c_char_p] * 3 + [ctypes.c_longlong]
    lib.tc_count.argtypes = [ctypes.c_char_p]
    return lib


def test_round_trip_and_replace(tc, tmp_path):
    p = str(tmp_path / "tune.txt").encode()
    assert tc.tc_count(p) == 0 and tc.tc_lookup(p, b"NVIDIA B200", b"fj", 7) == -1
    assert tc.tc_upsert(p, b"NVIDIA B200", b"fj", 7, 2 + 8 * 3, 1.5) == 0
    assert tc.tc_upsert(p, b"NVIDIA B200", b"batch", 7, 4, 9.0) == 0
    assert tc.tc_upsert(p, b"NVIDIA H100", b"fj", 7, 1 + 8, 2.0) == 0
    assert tc.tc_lookup(p, b"NVIDIA B200", b"fj", 7) == 26
    assert tc.tc_lookup(p, b"NVIDIA B200", b"batch", 7) == 4
    assert tc.tc_lookup(p, b"NVIDIA H100", b"fj", 7) == 9
    assert tc.tc_upsert(p, b"NVIDIA B200", b"fj", 7, 4 + 8, 1.2) == 0   # replaces, not appends
    assert tc.tc_count(p) == 3 and tc.tc_lookup(p, b"NVIDIA B200", b"fj", 7) == 12
    text = open(p.decode()).read()
    assert "ccfj-tune-v1 NVIDIA_B200 fj 7 12 " in text


def test_foreign_lines_are_kept_and_ignored(tc, tmp_path):
    path = tmp_path / "tune.txt"
    path.write_text("# notes\nccfj-tune-v1 X fj 1 2\nccfj-tune-v1 X fj 1 2 3.0 extra\n"
                    "ccfj-tune-v2 X fj 1 2 3.0\n")
    p = str(path).encode()
    assert tc.tc_count(p) == 0
    assert tc.tc_upsert(p, b"X", b"fj", 1, 4, 0.5) == 0
    assert tc.tc_lookup(p, b"X", b"fj", 1) == 4
    assert path.read_text().startswith("# notes\n")
