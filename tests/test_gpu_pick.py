"""Dispersion-curve picking (ccfj.pick_curve over ccfj_pick_v1) against a
numpy restatement of the same rule: the first largest value in the band,
then the parabola vertex through it and its neighbours. No reference
counterpart (the reference's users pick from the plotted spectrum)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pick_np(spec, c, lo, hi):
    nc, nf = spec.shape
    cp = np.full(nf, np.nan, np.float32)
    amp = np.full(nf, np.nan, np.float32)
    for i in range(nf):
        band = np.flatnonzero((c >= lo[i]) & (c <= hi[i]))
        if len(band) == 0 or np.isnan(spec[band, i]).any():
            continue
        b = band[np.argmax(spec[band, i])]
        y0 = np.float32(spec[b, i])
        cpi, ai = np.float32(c[b]), y0
        if b - 1 in band and b + 1 in band:
            ym, yp = np.float32(spec[b - 1, i]), np.float32(spec[b + 1, i])
            den = np.float32(ym - np.float32(2) * y0 + yp)
            if den < 0:
                d = np.float32(min(0.5, max(-0.5, np.float32(0.5) * (ym - yp) / den)))
                step = c[b + 1] - c[b] if d >= 0 else c[b] - c[b - 1]
                cpi = np.float32(c[b] + d * step)
                ai = np.float32(y0 - np.float32(0.25) * (ym - yp) * d)
        cp[i], amp[i] = cpi, ai
    return cp, amp


def test_pick_matches_numpy_rule():
    import ccfj
    import cases
    case = cases.noise_case("noise_small")
    spec = ccfj.fj_noise(case["uf"], case["r"], case["c"], case["f"])
    c = case["c"].astype(np.float32)
    lo = np.full(len(case["f"]), 1500.0, np.float32)
    hi = np.linspace(4000.0, 4800.0, len(case["f"])).astype(np.float32)
    cp, amp = ccfj.pick_curve(spec, c, lo, hi)
    ecp, eamp = _pick_np(spec, c, lo, hi)
    assert np.array_equal(np.isnan(cp), np.isnan(ecp))
    ok = ~np.isnan(ecp)
    assert np.allclose(cp[ok], ecp[ok], rtol=1e-6, atol=1e-3)
    assert np.allclose(amp[ok], eamp[ok], rtol=1e-6, atol=1e-6)
    assert np.all((cp[ok] >= lo[ok] - 1e-3) & (cp[ok] <= hi[ok] + 1e-3))


def test_pick_edges():
    import ccfj
    c = np.linspace(1000.0, 2000.0, 11).astype(np.float32)
    spec = np.zeros((11, 4), np.float32)
    spec[:, 0] = np.exp(-((c - 1530.0) / 200.0) ** 2)   # interior peak: refined
    spec[:, 1] = np.linspace(0, 1, 11)                   # at the band edge: not refined
    spec[3, 2] = np.nan                                  # NaN in the band
    spec[:, 3] = 1.0                                      # ties: the first
    cp, amp = ccfj.pick_curve(spec, c)
    assert 1500.0 < cp[0] < 1600.0 and abs(cp[0] - 1530.0) < 15.0
    assert cp[1] == 2000.0 and amp[1] == 1.0
    assert np.isnan(cp[2]) and np.isnan(amp[2])
    assert cp[3] == 1000.0
    cp, _ = ccfj.pick_curve(spec, c, cmin=1210.0, cmax=1250.0)   # no velocity in the band
    assert np.all(np.isnan(cp))
