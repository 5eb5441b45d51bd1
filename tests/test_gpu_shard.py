"""The sharded search's per-shard GPU search (cudadtw_b200.shard.gpu_search)
on one GPU: the shards of a 2- and 3-way split, searched one after the other
and combined by their packed keys, give the whole-stream search result."""
import numpy as np
import pytest
import torch

from cudadtw_b200 import shard, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_shards_combine_to_whole_search(world):
    from cudadtw_b200 import Handle
    x = synth.metal_like(1 << 20, seed=5)
    q, _ = synth.cut_query(x, 128, seed=6, noise=0.1)
    W = 12
    with Handle(0) as h:
        dx = torch.from_numpy(x).cuda()
        avg, std = h.avg_std(dx, q.size)
        h.set_query(q, W)
        whole = h.prune_cdtw(dx, avg, std)
        search = shard.gpu_search(h, dx, q, W)
        keys = []
        for r in range(world):
            s0, s1 = shard.shard_samples(x.size, q.size, r, world)
            loc, d = search(s0, s1)
            keys.append(shard.pack_key(d, s0 + loc))
        d, w = shard.unpack_key(min(keys))
        assert w == whole[0]
        assert d == pytest.approx(whole[1], rel=1e-6)
