import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(REPO, "cc-fjpy_b200"), os.path.join(REPO, "oracle"),
          os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(REPO, "tests", "golden", "reference_outputs.npz")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def lib():
    from ccfj import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def probe():
    """The test-only special-function probe library (not the product)."""
    from ccfj import _lib
    return _lib.load_probe()


@pytest.fixture(scope="session")
def emul(tmp_path_factory):
    """The host replay of the cross-correlation kernels (tests/cc_emul.cpp:
    the kernels' plan and per-thread arithmetic in their loop structure),
    compiled with the host C++ compiler."""
    import ctypes
    import shutil
    import subprocess
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    csrc = os.path.join(REPO, "cc-fjpy_b200", "csrc")
    so = str(tmp_path_factory.mktemp("ccemul") / "libccemul.so")
    subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-Wno-unknown-pragmas",
                    "-I", os.path.join(REPO, "include"), "-I", csrc,
                    os.path.join(REPO, "tests", "cc_emul.cpp"), "-o", so], check=True)
    from ccfj import _cc
    lib = ctypes.CDLL(so)
    lib.cc_emul_v1.argtypes = [ctypes.POINTER(_cc.CcArgs)]
    lib.cc_emul_v1.restype = ctypes.c_int
    lib.cc_emul_error.restype = ctypes.c_char_p
    lib.cc_emul_spectra.argtypes = [ctypes.POINTER(_cc.CcArgs), ctypes.c_void_p,
                                    ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_longlong),
                                    ctypes.POINTER(ctypes.c_int)]
    lib.cc_emul_spectra.restype = ctypes.c_int
    lib.cc_emul_shift_range.argtypes = [ctypes.c_longlong] * 5 + \
        [ctypes.POINTER(ctypes.c_longlong)] * 2
    lib.cc_emul_shift_range.restype = None
    lib.cc_emul_fft_plan.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.cc_emul_fft_plan.restype = ctypes.c_int
    return lib
