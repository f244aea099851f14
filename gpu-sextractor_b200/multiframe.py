"""Frame sharding across processes (one process per GPU).

Frames are independent units of the extraction path, so a multi-GPU run
shards frames across ranks with no collective on the data path; the only
communication is the barrier around the timed region and the max-over-ranks
reduction of the elapsed time (torch.distributed, NCCL on GPUs, gloo on CPU).
"""


def shard(nframes, rank, world, sizes=None):
    """Frames of this rank.  With sizes (work per frame), longest-processing-
    time-first greedy assignment; otherwise round robin."""
    if sizes is None:
        return list(range(rank, nframes, world))
    order = sorted(range(nframes), key=lambda i: (-sizes[i], i))
    load = [0] * world
    owner = [0] * nframes
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += sizes[i]
    return [i for i in range(nframes) if owner[i] == rank]


def max_over_ranks(values, dist=None, device=None):
    """Element-wise max of a list of floats over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(values)
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]
