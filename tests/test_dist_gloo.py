"""The multi-process (frequency-sharded) path on CPU: world_size 2 over gloo,
with the FP64 oracle standing in for the CUDA transform of each shard. The
gathered result must equal the unsharded transform exactly."""
import os
import socket

import numpy as np
import pytest

import cases


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_cols(uf, r, c, f, fstride, itype, func, cols):
    import fj_oracle as O
    a, b = cols
    uf = np.asarray(uf)
    if func == 0:
        return O.fj_noise(uf[:, a * fstride:b * fstride], r, c, np.asarray(f)[a:b], fstride, itype, 0)
    # the Hilbert transform runs along the full row, then the shard's columns
    indx = np.argsort(r)
    rs = np.asarray(r)[indx]
    U, r32, f32, c32 = O._prep(uf[indx], rs, c, f, fstride)
    H = O._prep(O.hilbert_rows(uf[indx]), rs, c, f, fstride)[0]
    out = (O.fj_transform(U[:, a:b], r32, f32[a:b], c32, itype, "J")
           - O.fj_transform(H[:, a:b], r32, f32[a:b], c32, itype, "Y"))
    return O._normalize(out)


def _worker(rank, world, port, func, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys
        here = os.path.dirname(os.path.abspath(__file__))
        for p in (os.path.join(os.path.dirname(here), "cc-fjpy_b200"),
                  os.path.join(os.path.dirname(here), "oracle"), here):
            sys.path.insert(0, p)
        from ccfj import dist as cdist
        case = cases.noise_case("noise_small")
        y = cdist.fj_noise_sharded(case["uf"], case["r"], case["c"], case["f"], itype=1,
                                   func=func, transform=_oracle_cols)
        q.put((rank, y))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("func", [0, 1])
def test_frequency_sharding_world2_gloo(func):
    import torch.multiprocessing as mp
    import fj_oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, 2, port, func, q)) for k in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    case = cases.noise_case("noise_small")
    full = O.fj_noise(case["uf"], case["r"], case["c"], case["f"], itype=1, func=func)
    for k in range(2):
        assert res[k].shape == full.shape
        np.testing.assert_allclose(res[k], full.astype(np.float32), rtol=0, atol=1e-6)
    assert np.array_equal(res[0], res[1])


@pytest.mark.parametrize("n,world", [(10, 3), (2048, 8), (5, 8), (1, 1)])
def test_shard_ranges_cover_exactly(n, world):
    from ccfj.dist import shard_range
    spans = [shard_range(n, k, world) for k in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    for (a0, b0), (a1, b1) in zip(spans, spans[1:]):
        assert b0 == a1
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1
