"""Frequency-sharded F-J transforms across processes (one GPU each).

The transform of every frequency column, its normalisation included, is
independent of the others (src/ccfj-gpu.pyx:266-267 normalises column by
column), so N ranks can split the frequencies and exchange nothing but the
finished columns. `fj_noise_sharded` computes this rank's block of
frequencies with the CUDA library and all-gathers the blocks through
torch.distributed (NCCL on GPUs; gloo works for CPU-side tests with a
substitute transform). The result equals single-process `fj_noise`.
"""
import numpy as np


def shard_range(n, rank, world):
    """Contiguous block [start, stop) of n items for `rank` of `world`; the
    first n % world ranks get one extra item."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %r outside a world of %r" % (rank, world))
    base, rem = divmod(n, world)
    start = rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


def gather_frequency_blocks(block, nf, group=None):
    """All-gathers per-rank [nc, nf_rank] float32 blocks (in rank order) into
    the full [nc, nf] array on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nc = block.shape[0]
    widths = [shard_range(nf, q, world) for q in range(world)]
    wmax = max(b - a for a, b in widths)
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else "cpu"
    pad = np.zeros((nc, wmax), dtype=np.float32)
    pad[:, :block.shape[1]] = block
    mine = torch.from_numpy(pad).to(device)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    out = np.empty((nc, nf), dtype=np.float32)
    for q, (a, b) in enumerate(widths):
        out[:, a:b] = parts[q].cpu().numpy()[:, :b - a]
    assert widths[rank][1] - widths[rank][0] == block.shape[1]
    return out


def fj_noise_sharded(uf, r, c, f, fstride=1, itype=1, func=0, group=None, transform=None):
    """fj_noise with the frequencies split over the ranks of `group`.

    Every rank passes the same arguments; each computes frequencies
    shard_range(len(f), rank, world) and receives the full float32 [nc, nf]
    result. `transform(uf, r, c, f, fstride, itype, func, cols)` computes the
    columns cols = (a, b) of the normalised transform; it defaults to this
    package's CUDA implementation."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    a, b = shard_range(len(f), rank, world)
    if transform is None:
        transform = _cuda_columns
    block = np.asarray(transform(uf, r, c, f, fstride, itype, func, (a, b)), dtype=np.float32)
    return gather_frequency_blocks(block, len(f), group)


def _cuda_columns(uf, r, c, f, fstride, itype, func, cols):
    import warnings

    from . import _lib, _transform
    if func not in (0, 1) or itype not in (0, 1):
        raise ValueError("func and itype must be 0 or 1")
    r = np.asarray(r)
    indx = np.argsort(r)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        if func == 0:
            return _transform([uf], r[indx], c, f, fstride, itype, _lib.MODE_J, perm=indx,
                              normalize=True, cols=cols)
        return _transform([uf], r[indx], c, f, fstride, itype, _lib.MODE_J_MINUS_Y, perm=indx,
                          hilbert=True, normalize=True, cols=cols)
