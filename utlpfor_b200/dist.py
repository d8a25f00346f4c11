"""Batches of streams over several GPUs, one process per GPU.

Streams are independent, so a batch shards by streams with no exchange on
the data path: each rank packs, unpacks or queries its own contiguous range
of streams.  When the ranks' packed shards form one stream (rank after rank,
as repeated PackUint32(flag|Append, ...) calls would lay it out), the only
exchange is an exclusive scan of the ranks' packed byte counts: one
all-gather of 8 bytes per rank.  Timing across ranks is the maximum.
"""
import numpy as np


def _dist():
    import torch.distributed as dist
    return dist


def shard_streams(val_off, rank, world):
    """The contiguous range [s0, s1) of streams rank `rank` of `world` owns:
    cut at the stream boundaries nearest to equal shares of the values."""
    vo = np.ascontiguousarray(val_off, dtype=np.uint64)
    ns = len(vo) - 1
    total = int(vo[-1] - vo[0])
    cuts = [0]
    for r in range(1, world):
        target = int(vo[0]) + total * r // world
        cuts.append(max(cuts[-1], int(np.searchsorted(vo[:-1], target, side="left"))))
    cuts.append(ns)
    return cuts[rank], cuts[rank + 1]


def _device_for(group):
    dist = _dist()
    import torch
    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def exclusive_offsets(local_bytes, group=None):
    """(this rank's byte offset in the joint stream, the joint length): an
    exclusive scan of every rank's packed byte count (one all-gather)."""
    import torch
    dist = _dist()
    dev = _device_for(group)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = torch.tensor([int(local_bytes)], dtype=torch.int64, device=dev)
    allv = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(allv, mine, group=group)
    sizes = [int(t.item()) for t in allv]
    return sum(sizes[:rank]), sum(sizes)


def max_over_ranks(values, group=None):
    """Element-wise maximum of a list of floats over the ranks."""
    import torch
    dist = _dist()
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=_device_for(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [float(x) for x in t.tolist()]


def global_block_offsets(local_block_off, byte_offset):
    """A rank's block offsets moved to their place in the joint stream."""
    return np.asarray(local_block_off, dtype=np.uint64) + np.uint64(byte_offset)
