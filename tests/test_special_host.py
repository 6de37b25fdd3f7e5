"""The special-function approximations of the kernels (host-compiled copy of
the same source, from the test library libccfj_b200_probe.so) against mpmath: J0, J1, Y0, Y1 and B = int_0^x Z0."""
import ctypes

import mpmath as mp
import numpy as np
import pytest

mp.mp.dps = 30


def _mp_values(x):
    xm = mp.mpf(x)
    j0, j1, y0, y1 = mp.besselj(0, xm), mp.besselj(1, xm), mp.bessely(0, xm), mp.bessely(1, xm)
    h0, h1 = mp.struveh(0, xm), mp.struveh(1, xm)
    bj = xm * j0 + mp.pi * xm / 2 * (j1 * h0 - j0 * h1)
    by = xm * y0 + mp.pi * xm / 2 * (y1 * h0 - y0 * h1)
    return [float(v) for v in (j0, j1, bj, y0, y1, by)]


XS = np.concatenate([np.linspace(0.02, 12, 240), np.geomspace(12, 2e4, 160),
                     [1.999999, 2.0, 4.9999, 5.0, 7.99999, 8.0, 8.00001]])
REF = np.array([_mp_values(x) for x in XS])


def _eval(lib, prec):
    out = np.zeros((len(XS), 6))
    st = lib.ccfj_special_host(prec, len(XS), XS.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert st == 0
    return out


def _amplitude(x):
    # the oscillation amplitude sqrt(2/(pi x)) for x > 1, 1 below
    return np.minimum(1.0, np.sqrt(2 / (np.pi * np.maximum(x, 1e-30))))


def test_fp32_functions(probe):
    got = _eval(probe, 0)
    amp = _amplitude(XS)
    for j, name in enumerate(("J0", "J1", "BJ", "Y0", "Y1", "BY")):
        scale = amp if name[0] != "B" else np.maximum(amp, np.abs(REF[:, j]))
        if name in ("Y0", "Y1", "BY"):
            scale = np.maximum(scale, np.abs(REF[:, j]))
        err = np.abs(got[:, j] - REF[:, j]) / scale
        assert err.max() < 1.5e-6, (name, err.max(), XS[err.argmax()])


def test_fp64_functions(probe):
    got = _eval(probe, 1)
    amp = _amplitude(XS)
    for j, name in enumerate(("J0", "J1", "BJ", "Y0", "Y1", "BY")):
        scale = np.maximum(amp, np.abs(REF[:, j]))
        # the host harness forms the phase as x / (2 pi) in double, which is
        # already off by about x * 1e-16 rad (the kernels form it from f r / c)
        err = np.abs(got[:, j] - REF[:, j]) / scale / (1e-13 + 3e-16 * XS)
        assert err.max() < 1.0, (name, err.max(), XS[err.argmax()])


def test_bad_precision(probe):
    x = np.ones(1)
    out = np.zeros(6)
    assert probe.ccfj_special_host(2, 1, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(0, 1.5e-6), (1, None)])
def test_device_functions(probe, prec, tol):
    """The kernels' own code on the GPU (fast SFU sine/cosine in FP32)."""
    import torch
    x = torch.from_numpy(XS).cuda()
    out = torch.zeros((len(XS), 6), dtype=torch.float64, device="cuda")
    st = probe.ccfj_special_device(prec, len(XS), ctypes.c_void_p(x.data_ptr()),
                                 ctypes.c_void_p(out.data_ptr()), None)
    assert st == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    amp = _amplitude(XS)
    for j, name in enumerate(("J0", "J1", "BJ", "Y0", "Y1", "BY")):
        scale = np.maximum(amp, np.abs(REF[:, j]))
        if tol is None:
            err = np.abs(got[:, j] - REF[:, j]) / scale / (1e-13 + 3e-16 * XS)
            assert err.max() < 1.0, (name, err.max(), XS[err.argmax()])
        else:
            err = np.abs(got[:, j] - REF[:, j]) / scale
            assert err.max() < tol, (name, err.max(), XS[err.argmax()])


@pytest.mark.gpu
def test_paired_station_values_equal_scalar(probe):
    """The paired (two cells per FFMA2 / FMUL2 / FADD2) x >= 8 evaluation of
    the transform kernels against their scalar one: the same values, cell by
    cell, over the frequencies, velocities and distances of the benchmark
    workloads."""
    import torch
    rng = np.random.default_rng(3)
    n = 200000
    f = rng.uniform(0.005, 2.0, n)
    c0 = rng.uniform(500.0, 5000.0, n)
    c1 = c0 + rng.choice([4.5, 1.75, 224.0], n)
    r = rng.uniform(1e3, 1.5e6, n)
    x = 2 * np.pi * f * r / np.maximum(c0, c1)
    keep = x >= 8.5
    inp = np.stack([f, c0, c1, r], axis=1)[keep].astype(np.float32)
    d_in = torch.from_numpy(np.ascontiguousarray(inp)).cuda()
    d_out = torch.zeros((len(inp), 8), dtype=torch.float32, device="cuda")
    st = probe.ccfj_paired_probe(len(inp), ctypes.c_void_p(d_in.data_ptr()),
                                 ctypes.c_void_p(d_out.data_ptr()), None)
    assert st == 0
    o = d_out.cpu().numpy()
    scalar, paired = o[:, :4], o[:, 4:]
    diff = np.abs(scalar - paired)
    assert diff.max() <= 2e-6, (diff.max(), inp[diff.max(axis=1).argmax()])
