"""Multi-GPU search by stream sharding (one process per GPU).

Windows are independent, so a search over one long stream splits into
contiguous window ranges, one per rank; rank r needs the samples of its
windows plus the M-1 that follow (the halo).  Each rank runs the pruned search
on its shard and the ranks exchange one 8-byte key: (distance bits << 32 |
window), reduced with MIN, which gives the global best match with the lowest
window on ties — the same result as one search over the whole stream.

``sharded_search`` takes the per-shard search as a callable, so the same
exchange runs with the GPU search (``gpu_search``) under NCCL and with any
stand-in under gloo.
"""
from __future__ import annotations

import struct
from typing import Callable

import numpy as np


def shard_windows(N: int, M: int, rank: int, world: int) -> tuple[int, int]:
    """Window range [w0, w1) of ``rank``: an even split of the N-M+1 windows."""
    nw = N - M + 1
    if nw <= 0:
        raise ValueError("subject shorter than the query")
    return rank * nw // world, (rank + 1) * nw // world


def shard_samples(N: int, M: int, rank: int, world: int) -> tuple[int, int]:
    """Sample range [s0, s1) rank needs: its windows plus the M-1 halo."""
    w0, w1 = shard_windows(N, M, rank, world)
    return w0, (w1 + M - 1) if w1 > w0 else w0


def pack_key(distance: float, window: int) -> int:
    """(float32 bits of a non-negative distance) << 32 | window, as int64:
    ordered by distance, then by window."""
    bits = struct.unpack("<I", struct.pack("<f", float(distance)))[0]
    return (bits << 32) | (int(window) & 0xFFFFFFFF)


def unpack_key(key: int) -> tuple[float, int]:
    bits = (int(key) >> 32) & 0xFFFFFFFF
    return struct.unpack("<f", struct.pack("<I", bits))[0], int(key) & 0xFFFFFFFF


NO_MATCH = (0x7F800000 << 32) | 0xFFFFFFFF  # +inf, no window


def sharded_search(search: Callable[[int, int], tuple[int, float]], N: int, M: int,
                   group=None, device=None) -> tuple[int, float]:
    """Global best (window, distance) of a search split over the ranks of
    ``group``.  ``search(s0, s1)`` searches the samples [s0, s1) of the
    stream and returns (window relative to s0, distance) or (-1, inf)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    s0, s1 = shard_samples(N, M, rank, world)
    key = NO_MATCH
    if s1 - s0 >= M:
        loc, d = search(s0, s1)
        if loc >= 0 and np.isfinite(d):
            key = pack_key(d, s0 + loc)
    t = torch.tensor([key], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    k = int(t.item())
    if k == NO_MATCH:
        return -1, float("inf")
    d, w = unpack_key(k)
    return w, d


def gpu_search(handle, subject, query, W: int, metric=0):
    """The per-shard search on this rank's GPU: ``subject`` is the full
    stream as a CUDA tensor (each rank reads only its shard), the query a host
    array.  Returns the ``search`` callable for ``sharded_search``."""
    def search(s0: int, s1: int):
        x = subject[s0:s1]
        avg, std = handle.avg_std(x, len(query))
        handle.set_query(query, W)
        loc, d = handle.prune_cdtw(x, avg, std, metric=metric)
        return int(loc), float(d)
    return search
