"""Multi-GPU sharding of sample passes (one process per GPU).

Paths are independent, so a render shards by sample pass with no exchange in
the data path: rank r renders its own contiguous run of whole spectral blocks
(each with its own random streams, since the pass index keys Philox) into its
own film.  The one exchange is at the end: the FP64 block statistics of all
ranks are summed (``torch.distributed.all_reduce``, NCCL over NVLink on GPUs,
gloo on CPUs) into the film of the whole render.
"""
import torch


def block_range(total_blocks, rank, world):
    """Contiguous share [first, last) of ``total_blocks`` spectral blocks for ``rank``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(int(total_blocks), world)
    first = rank * base + min(rank, extra)
    return first, first + base + (1 if rank < extra else 0)


def pass_indices(total_blocks, bands, rank, world):
    """(pass_idx, band) of every pass rank ``rank`` renders, in order."""
    first, last = block_range(total_blocks, rank, world)
    return [(b * bands + k, k) for b in range(first, last) for k in range(bands)]


def reduce_film(mean, m2, num_blocks, group=None):
    """Combine per-rank films: mean over all blocks, summed squares, total count.

    mean/m2: float64 tensors of identical shape on every rank; the result
    replaces them in place on every rank."""
    import torch.distributed as dist
    if mean.dtype != torch.float64 or m2.dtype != torch.float64:
        raise TypeError("film statistics must be float64")
    n = torch.tensor([float(num_blocks)], dtype=torch.float64, device=mean.device)
    dist.all_reduce(n, group=group)
    total = float(n.item())
    mean.mul_(float(num_blocks))
    dist.all_reduce(mean, group=group)
    if total > 0:
        mean.div_(total)
    dist.all_reduce(m2, group=group)
    return mean, m2, int(round(total))


def adjoint_range(total_passes, rank, world):
    """Contiguous share [first, last) of ``total_passes`` adjoint passes for ``rank``
    (the adjoint has no film planes, so passes need not come in whole blocks)."""
    return block_range(total_passes, rank, world)


def reduce_gradient(grad, group=None):
    """Sum the per-rank FP64 parameter gradients (each rank replayed its own passes)
    in place on every rank: the one exchange of a multi-GPU adjoint."""
    import torch.distributed as dist
    if grad.dtype != torch.float64:
        raise TypeError("gradients are reduced in float64")
    dist.all_reduce(grad, group=group)
    return grad


def scene_shard(costs, rank, world):
    """Scenes of a multi-scene batch for ``rank``: scenes are independent, so a
    batch shards by scene with no exchange in the data path.  Greedy longest-
    processing-time assignment on estimated costs (e.g. pixels x depth x the
    blocks a scene needs): scenes by decreasing cost (ties by index), each to
    the least-loaded rank (ties to the lowest rank).  Every rank computes the
    same assignment; returns this rank's scene indices in increasing order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    costs = [float(c) for c in costs]
    if any(c < 0 for c in costs):
        raise ValueError("negative scene cost")
    load = [0.0] * world
    mine = []
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += costs[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


def gather_scene_blocks(blocks, indices, num_scenes, group=None):
    """Every rank's per-scene block counts (``blocks[j]`` for scene
    ``indices[j]``) combined into one int64 vector of ``num_scenes`` entries on
    every rank (one all-reduce; each scene belongs to exactly one rank)."""
    import torch.distributed as dist
    out = torch.zeros(int(num_scenes), dtype=torch.int64)
    for j, i in enumerate(indices):
        out[int(i)] = int(blocks[j])
    dist.all_reduce(out, group=group)
    return out
