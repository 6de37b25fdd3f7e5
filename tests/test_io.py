"""The `.npz` hand-off between CC and fj_noise (ccfj.load_ncfs), without a
GPU: the member-by-member reader against np.load on stored, compressed and
Fortran-ordered archives written as the reference's workflow writes them
(np.savez(name, ncfs=..., r=..., f=...)). Page-locked allocation itself
needs the CUDA runtime and is exercised by tests/test_gpu_cc_fj.py."""
import numpy as np
import pytest


@pytest.fixture
def plain_memory(monkeypatch):
    from ccfj import _io
    monkeypatch.setattr(_io, "pinned_empty", lambda shape, dtype: np.empty(shape, dtype))


@pytest.mark.parametrize("writer", [np.savez, np.savez_compressed])
@pytest.mark.parametrize("fortran", [False, True])
def test_load_ncfs_matches_np_load(tmp_path, plain_memory, writer, fortran):
    import ccfj
    rng = np.random.default_rng(4)
    ncfs = (rng.standard_normal((70, 41)) + 1j * rng.standard_normal((70, 41))).astype(
        np.complex64)
    if fortran:
        ncfs = np.asfortranarray(ncfs)
    r, f = rng.uniform(1, 300, 70), np.linspace(0.0, 1.0, 41)
    p = tmp_path / "summed.npz"
    writer(p, ncfs=ncfs, r=r, f=f, StationPairs=np.arange(140, dtype=np.int32))
    got = ccfj.load_ncfs(p)
    ref = np.load(p)
    assert set(got) == {"ncfs", "r", "f"}
    for k in got:
        assert got[k].dtype == ref[k].dtype and np.array_equal(got[k], ref[k]), k


def test_load_ncfs_missing_key(tmp_path, plain_memory):
    import ccfj
    p = tmp_path / "x.npz"
    np.savez(p, ncfs=np.zeros((2, 3), np.complex64), f=np.zeros(3))
    with pytest.raises(KeyError):
        ccfj.load_ncfs(p)
