"""A batch of independent transforms split over GPUs, one process per GPU:
rank r of `world` takes the contiguous slice batch_slice(batch, r, world) of
the batch (slices differ in size by at most one transform).  No collective
is on the data path: each rank transforms its slice on its own GPU and its
output stays there.  gather() assembles the slices on one rank, for callers
that want the whole result in one place.
"""
from __future__ import annotations


def batch_slice(batch, rank, world):
    """[start, stop) of rank's contiguous share of `batch` transforms."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    per, extra = divmod(int(batch), int(world))
    start = rank * per + min(rank, extra)
    return start, start + per + (1 if rank < extra else 0)


def local_part(a, rank, world):
    """Rank's slice of `a` along its first (batch) axis."""
    s, e = batch_slice(a.shape[0], rank, world)
    return a[s:e]


def gather(part, batch, rank, world, dist, dst=0):
    """The whole batch on rank `dst` (None elsewhere) from every rank's slice
    `part` (a torch tensor, batch axis first).  Every rank calls it."""
    import torch
    per = -(-batch // world)
    pad = torch.zeros((per,) + tuple(part.shape[1:]), dtype=part.dtype, device=part.device)
    pad[:part.shape[0]] = part
    bufs = [torch.empty_like(pad) for _ in range(world)] if rank == dst else None
    dist.gather(pad, bufs, dst=dst)
    if rank != dst:
        return None
    pieces = []
    for r in range(world):
        s, e = batch_slice(batch, r, world)
        pieces.append(bufs[r][:e - s])
    return torch.cat(pieces, 0)
