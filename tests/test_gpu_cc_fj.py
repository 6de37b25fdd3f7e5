"""Records to dispersion spectrum in one call (ccfj.cc_fj_noise over
ccfj_cc_fj_noise_v1): the cross-spectra stay on the device between the
cross-correlation and the transform. Checked against the reference's
two-step pipeline on the host (ccfj.CC, then ccfj.fj_noise on its output):
the same kernels on the same values, so the results are equal bit for bit;
against the FP64 oracles (CC, then fj_noise) within 1e-4; and the pinned
`.npz` loader's round trip into fj_noise."""
import numpy as np
import pytest

import cc_oracle as C
import fj_oracle as O

pytestmark = pytest.mark.gpu


def _case(seed=7, nsta=12, npts=6000, fftlen=600, nf=150, fstride=2):
    rng = np.random.default_rng(seed)
    data = rng.standard_normal(nsta * npts).astype(np.float32)
    # a common arrival so that the spectra carry a coherent part
    data[: nsta * npts] += np.tile(np.sin(np.arange(npts) * 0.05).astype(np.float32), nsta)
    se = np.tile([0, npts], nsta).astype(np.int32)
    se[2:4] = [400, npts - 300]                 # a ragged record
    import ccfj
    pairs = ccfj.GetStationPairs(nsta)
    xy = rng.uniform(0, 5e4, (nsta, 2))
    p2 = pairs.reshape(-1, 2)
    r = np.hypot(*(xy[p2[:, 0]] - xy[p2[:, 1]]).T)
    f = np.arange(nf) * fstride * 4.0 / fftlen + 0.01
    c = np.linspace(1500.0, 4500.0, 90)
    return dict(npts=npts, nsta=nsta, nf=nf, fftlen=fftlen, pairs=pairs, se=se, data=data,
                r=r, f=f, c=c, fstride=fstride)


@pytest.mark.parametrize("func,itype,onebit", [(0, 1, 0), (1, 1, 0), (0, 0, 1)])
def test_one_call_equals_two_step_pipeline(func, itype, onebit):
    import ccfj
    k = _case()
    # one-bit records make exactly vanishing spectral values likely, where
    # whitening turns FP32 rounding into an arbitrary unit phase (no FP32
    # implementation can match FP64 there): the one-bit case is not whitened
    kw = dict(overlaprate=0.5, fstride=k["fstride"], ifonebit=onebit,
              ifspecwhittenning=0 if onebit else 1)
    d1 = k["data"].copy()
    got = ccfj.cc_fj_noise(k["npts"], k["nsta"], k["nf"], k["fftlen"], k["pairs"], k["se"], d1,
                           k["r"], k["c"], k["f"], itype=itype, func=func, **kw)
    assert np.array_equal(d1, k["data"])          # one-bit is applied on load only
    d2 = k["data"].copy()
    ncfs = ccfj.CC(k["npts"], k["nsta"], k["nf"], k["fftlen"], k["pairs"], k["se"], d2, **kw)
    two = ccfj.fj_noise(ncfs, k["r"], k["c"], k["f"], itype=itype, func=func)
    assert got.shape == (len(k["c"]), k["nf"]) and got.dtype == np.float32
    assert np.array_equal(got, two, equal_nan=True)
    # the FP64 oracles chained the same way
    ncfs64 = C.CC(k["npts"], k["nsta"], k["nf"], k["fftlen"], k["pairs"], k["se"],
                  k["data"].copy(), **kw)
    y64 = O.fj_noise(ncfs64, k["r"], k["c"], k["f"], itype=itype, func=func)
    assert O.rel_error(got, y64) <= 1e-4


def test_pinned_npz_round_trip(tmp_path):
    import ccfj
    k = _case(seed=8)
    ncfs = ccfj.CC(k["npts"], k["nsta"], k["nf"], k["fftlen"], k["pairs"], k["se"],
                   k["data"].copy(), overlaprate=0.5, fstride=k["fstride"])
    p = tmp_path / "summed.npz"
    np.savez(p, ncfs=ncfs, r=k["r"] / 1e3, f=k["f"])   # r in km, as the reference's example
    z = ccfj.load_ncfs(p)
    ref = np.load(p)
    assert all(np.array_equal(z[key], ref[key]) for key in ("ncfs", "r", "f"))
    a = ccfj.fj_noise(np.real(z["ncfs"]), z["r"] * 1e3, k["c"], z["f"])
    b = ccfj.fj_noise(np.real(ref["ncfs"]), ref["r"] * 1e3, k["c"], ref["f"])
    assert np.array_equal(a, b, equal_nan=True)
