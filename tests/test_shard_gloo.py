"""Sharded search over 2 ranks (gloo, CPU): the window split with its halo
covers every window exactly once, and the one MIN exchange of packed
(distance, window) keys returns the whole-stream best match with the lowest
window on ties.  The per-shard search is the FP64 oracle here (the GPU search
is the same callable shape, see cudadtw_b200.shard.gpu_search)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from cudadtw_b200 import shard, synth


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, x, q, W, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        def search(s0, s1):
            d = oracle.cdtw_all(q, x[s0:s1], W)
            i = int(np.argmin(d))
            return i, float(np.float32(d[i]))
        out[rank] = shard.sharded_search(search, x.size, q.size)
    finally:
        dist.destroy_process_group()


def test_shard_ranges_cover_all_windows():
    for N, M, world in ((1000, 10, 2), (1000, 10, 3), (64, 64, 4), (100, 7, 8)):
        seen = []
        for r in range(world):
            w0, w1 = shard.shard_windows(N, M, r, world)
            s0, s1 = shard.shard_samples(N, M, r, world)
            seen.extend(range(w0, w1))
            if w1 > w0:
                assert s0 == w0 and s1 == w1 + M - 1 and s1 <= N
        assert seen == list(range(N - M + 1))


def test_key_order():
    assert shard.pack_key(1.0, 5) < shard.pack_key(1.0, 6) < shard.pack_key(1.5, 0)
    assert shard.unpack_key(shard.pack_key(2.5, 77)) == (2.5, 77)
    assert shard.pack_key(float("inf"), 0xFFFFFFFF) == shard.NO_MATCH


@pytest.mark.parametrize("world", [2])
def test_sharded_search_equals_whole_stream(world):
    x = synth.ecg_like(20000, seed=3)
    q, off = synth.cut_query(x, 64, seed=4, noise=0.05)
    W = 6
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), x, q, W, out), nprocs=world, join=True)
    d = oracle.cdtw_all(q, x, W)
    best = int(np.argmin(d))
    for r in range(world):
        loc, dist = out[r]
        assert loc == best
        assert dist == pytest.approx(d[best], rel=1e-6)
