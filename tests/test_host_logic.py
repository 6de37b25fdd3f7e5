"""Host-side logic that needs no GPU: the taper window and the station-pair
list against the reference's own compiled module (oracle/_ref, built from
src/ccfj.pyx), the integer window parameters that the device FFT front end
turns into its per-sample taper, and argument errors that fj_noise raises
before any device work."""
import os
import sys
import warnings

import numpy as np
import pytest

import cases

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def ref():
    d = os.path.join(REPO, "oracle", "_ref")
    if d not in sys.path:
        sys.path.insert(0, d)
    return pytest.importorskip("ccfj_ref", reason="reference build (make -C oracle) absent")


def _windows():
    rng = np.random.default_rng(5)
    out = []
    for _ in range(40):
        npts = int(rng.integers(64, 4096))
        Fs = float(rng.choice([1.0, 10.0, 20.0, 12.5]))
        T1 = float(rng.uniform(-5.0, npts / Fs))
        T2 = float(rng.uniform(0.0, 1.2 * npts / Fs))
        out.append((npts, Fs, T1, T2, float(rng.uniform(-1.0, 1.5))))
    # edges: no taper, full taper, overlapping ramps, no ramps, window past
    # the end, empty window
    out += [(512, 10.0, 3.0, 40.0, 0.0), (512, 10.0, 3.0, 40.0, 1.0),
            (512, 10.0, 3.0, 40.0, -0.5), (512, 10.0, 3.0, 40.0, 1.5),
            (300, 20.0, 2.0, 99.0, 0.8), (300, 20.0, 9.0, 4.0, 0.8)]
    return out


def _call(fn, *a):
    try:
        return fn(*a), None
    except IndexError as e:
        return None, str(e)


def test_win_matches_reference(ref):
    """Values, and the IndexError `win` raises for windows whose ramps
    leave the array."""
    import ccfj
    for w in _windows():
        (a, ea), (b, eb) = _call(ccfj.win, *w), _call(ref.win, *w)
        assert ea == eb, w
        if ea is None:
            assert np.array_equal(a, b), w


def test_station_pairs_match_reference(ref):
    import ccfj
    for n in (2, 3, 17, 200):
        assert np.array_equal(ccfj.GetStationPairs(n), np.asarray(ref.GetStationPairs(n)))


def _device_rule(npts, n1, n2, dl):
    """The per-sample taper of the device FFT front end (taper_value in
    fj_fft.cu), restated: the last write of win's ramp loop to sample t --
    the largest of t - n1, n2 - 1 - t and n2 - 1 - t + npts (a negative index
    counts from the end) that lies in [0, delta) -- else the zero-filled head
    [0, n1) and tail (from n2, or npts + n2 when n2 < 0), else 1."""
    w = np.ones(npts)
    tail = n2 if n2 >= 0 else max(npts + n2, 0)
    for t in range(npts):
        cands = [i for i in (t - n1, n2 - 1 - t, n2 - 1 - t + npts) if 0 <= i < dl]
        if cands:
            w[t] = np.sin(np.pi / 2 * max(cands) / dl)
        elif t < n1 or t >= tail:
            w[t] = 0.0
    return w


def test_device_taper_rule_reproduces_win(ref):
    """The window parameters the device receives (_win_params) and its
    per-sample rule reproduce the reference's `win` exactly, degenerate
    windows included (ends before starts, tapers outside [0, 1], windows
    before 0 s or past the end); where `win` raises IndexError,
    _win_params raises the same."""
    from ccfj import _eq
    rng = np.random.default_rng(9)
    wins = _windows() + [(int(rng.integers(4, 200)), float(rng.choice([1.0, 2.0, 0.5])),
                          float(rng.uniform(-50, 300)), float(rng.uniform(-300, 300)),
                          float(rng.uniform(-3, 3))) for _ in range(600)]
    for npts, Fs, T1, T2, taper in wins:
        expect, err = _call(ref.win, npts, Fs, T1, T2, taper)
        params, perr = _call(_eq._win_params, npts, Fs, [T1], [T2], taper)
        assert perr == err, (npts, Fs, T1, T2, taper)
        if err is None:
            n1, n2, dl = (int(v[0]) for v in params)
            assert np.array_equal(_device_rule(npts, n1, n2, dl), expect), (npts, Fs, T1, T2,
                                                                             taper)


def test_fj_noise_argument_errors_before_device_work(capsys):
    import ccfj
    case = cases.noise_case("noise_small")
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        # an unknown func prints the reference's message and returns 0
        assert ccfj.fj_noise(case["uf"], case["r"], case["c"], case["f"], func=3) == 0
        assert "set func as 0" in capsys.readouterr().out
        # the reference's reshape error for a spectrum that does not hold nf columns
        with pytest.raises(ValueError, match="cannot reshape"):
            ccfj.fj_noise(case["uf"][:, :-1], case["r"], case["c"], case["f"])
        with pytest.raises(ValueError):
            ccfj.fj_noise(case["uf"], case["r"], case["c"], case["f"], fstride=0)


def _device_support(npts, n1, n2, dl):
    """taper_support in fj_fft.cu, restated: the hull of the ramps and the
    plateau, clipped to [0, npts)."""
    tail = n2 if n2 >= 0 else max(npts + n2, 0)
    lo, hi = npts, 0
    for s, e in ((n1, n1 + dl), (n2 - dl, n2), (n2 + npts - dl, n2 + npts), (n1, tail)):
        a, b = max(s, 0), min(e, npts)
        if a < b:
            lo, hi = min(lo, a), max(hi, b)
    return lo, hi


def test_device_taper_support_holds_every_nonzero_sample():
    """The FFT front end loads no sample outside taper_support's range; the
    taper is zero there for every window the device can receive (the same
    600+ windows, plus the configuration-4 window shapes)."""
    from ccfj import _eq
    rng = np.random.default_rng(19)
    wins = _windows() + [(int(rng.integers(4, 200)), float(rng.choice([1.0, 2.0, 0.5])),
                          float(rng.uniform(-50, 300)), float(rng.uniform(-300, 300)),
                          float(rng.uniform(-3, 3))) for _ in range(600)]
    L = rng.integers(200, 2001, size=50)
    start = rng.integers(0, 16384 - L)
    wins += [(16384, 10.0, s / 10.0, (s + n) / 10.0, 0.9) for s, n in zip(start, L)]
    checked = 0
    for npts, Fs, T1, T2, taper in wins:
        params, perr = _call(_eq._win_params, npts, Fs, [T1], [T2], taper)
        if perr is not None:
            continue
        n1, n2, dl = (int(v[0]) for v in params)
        w = _device_rule(npts, n1, n2, dl)
        lo, hi = _device_support(npts, n1, n2, dl)
        outside = np.ones(npts, dtype=bool)
        outside[lo:hi] = False
        assert not np.any(w[outside] != 0), (npts, Fs, T1, T2, taper, lo, hi)
        checked += 1
    assert checked > 500
