"""ccfj_fj_noalloc_v1: the transform for callers that cannot allocate device
memory during a call (their own pool allocator holds the free memory, or
they must avoid the device synchronisation cudaMalloc may cause). It takes
its scratch from a fixed array in the library instead of allocating it.

Checked through the C ABI against the allocating entry ccfj_fj_v1 on the
same device inputs, on two calls in a row (the fixed scratch keeps the
previous call's contents), with the parity tolerance of the other tests.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import cases
import fj_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _device_case(torch, mode, itype):
    case = cases.noise_case("noise_small")
    idx = np.argsort(case["r"])
    uf = case["uf"]                      # complex64 [nr, nf]
    nr, nf, nc = len(case["r"]), len(case["f"]), len(case["c"])
    d = {
        "u": torch.from_numpy(np.ascontiguousarray(uf).view(np.float32)).cuda(),
        "perm": torch.from_numpy(idx.astype(np.int64)).cuda(),
        "r": torch.from_numpy(np.ascontiguousarray(case["r"][idx], dtype=np.float32)).cuda(),
        "f": torch.from_numpy(case["f"].astype(np.float32)).cuda(),
        "c": torch.from_numpy(case["c"].astype(np.float32)).cuda(),
    }
    from ccfj import _lib
    a = _lib.FjArgs()
    a.struct_size = ctypes.sizeof(a)
    a.nr, a.nf, a.nc = nr, nf, nc
    a.itype, a.mode, a.precision, a.normalize, a.device_ptrs = itype, mode, 0, 1, 1
    a.u[0] = d["u"].data_ptr()                                     # real parts
    a.u[1] = d["u"].data_ptr() + 4 if mode != _lib.MODE_J else None  # imaginary parts
    a.u_ld, a.u_rows, a.u_es, a.u_ncols, a.fstride = 2 * nf, nr, 2, nf, 1
    a.perm = d["perm"].data_ptr()
    a.r, a.f, a.c = d["r"].data_ptr(), d["f"].data_ptr(), d["c"].data_ptr()
    return a, d, (nc, nf)


@pytest.mark.parametrize("mode,itype", [(0, 1), (3, 0), (4, 1)])
def test_no_alloc_entry_matches_allocating_entry(lib, mode, itype):
    import torch
    from ccfj import _lib
    a, keep, shape = _device_case(torch, mode, itype)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ref = torch.empty(shape, dtype=torch.float32, device="cuda")
    a.out = ref.data_ptr()
    _lib.check(lib.ccfj_fj_v1(ctypes.byref(a), stream))
    outs = []
    for _ in range(2):
        y = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
        a.out = y.data_ptr()
        st = lib.ccfj_fj_noalloc_v1(ctypes.byref(a), stream)
        assert st == 0, lib.ccfj_last_error()
        outs.append(y)
    torch.cuda.synchronize()
    r = ref.cpu().numpy()
    for y in outs:
        assert O.rel_error(y.cpu().numpy(), r) <= TOL


def test_no_alloc_entry_rejects_oversize_problem(lib):
    import torch
    a, keep, shape = _device_case(torch, 0, 1)
    a.nr, a.nf, a.u_ncols, a.u_rows = 4096, 4096, 4096, 4096  # 128 MiB of scratch
    a.u_ld = 2 * 4096
    a.out = keep["u"].data_ptr()
    st = lib.ccfj_fj_noalloc_v1(ctypes.byref(a), None)
    assert st == 1  # CCFJ_ERR_INVALID, before any device work
    assert "fixed scratch holds" in lib.ccfj_last_error().decode()
