"""Argument checks of dispersion-curve picking that run before any device
work (no GPU needed): the Python wrapper's shape and band checks, and the
C entry's rejection of empty sizes and NULL arrays."""
import ctypes

import numpy as np
import pytest


def test_spec_must_be_two_dimensional():
    import ccfj
    with pytest.raises(ValueError, match=r"\[nc, nf\]"):
        ccfj.pick_curve(np.zeros(5, np.float32), np.arange(5.0))


def test_velocities_must_match_rows():
    import ccfj
    with pytest.raises(ValueError, match="velocities"):
        ccfj.pick_curve(np.zeros((4, 3), np.float32), np.arange(5.0))


@pytest.mark.parametrize("which", ["cmin", "cmax"])
def test_band_without_nan(which):
    import ccfj
    band = np.array([1.0, np.nan, 2.0])
    kw = {which: band}
    with pytest.raises(ValueError, match=which):
        ccfj.pick_curve(np.zeros((4, 3), np.float32), np.arange(4.0), **kw)


def test_band_broadcasts_per_frequency():
    """A scalar band is one value per frequency; a band of the wrong length
    is a broadcasting error, raised before the library is called."""
    import ccfj
    with pytest.raises(ValueError):
        ccfj.pick_curve(np.zeros((4, 3), np.float32), np.arange(4.0), cmin=np.ones(2))


def test_c_entry_rejects_empty_sizes_and_null_arrays(lib):
    from ccfj import _pick  # noqa: F401  (registers the signature)
    from ccfj import _lib
    lib = _lib.load()
    spec = np.zeros((2, 3), np.float32)
    c = np.zeros(2, np.float32)
    out = np.zeros(3, np.float32)
    assert lib.ccfj_pick_v1(spec.ctypes.data, 0, 3, c.ctypes.data, None, None, out.ctypes.data,
                            None, 0, None) == 1
    assert "must be >= 1" in lib.ccfj_last_error().decode()
    assert lib.ccfj_pick_v1(None, 2, 3, c.ctypes.data, None, None, out.ctypes.data, None, 0,
                            None) == 1
    assert "NULL" in lib.ccfj_last_error().decode()
