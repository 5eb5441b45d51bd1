"""The autotuner on the GPU: it tunes a small batched workload, every shape it
returns is accepted by the C ABI, and the batched search with the tuned shapes
finds the same matches as with the built-in rule."""
import numpy as np
import pytest
import torch

from cudadtw_b200 import autotune as at
from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu


def test_tuned_shapes_give_same_matches(tmp_path):
    from cudadtw_b200 import Handle
    x = synth.ecg_like(1 << 18, seed=4)
    batch = synth.batch_queries(x, 12, seed=5, m_lo=64, m_hi=400)
    qs = [b[0] for b in batch]
    ws = [b[1] for b in batch]
    with Handle(0) as h:
        dx = torch.from_numpy(x).cuda()
        table = at.tune_batched(qs, ws, at.gpu_batched_measure(h, dx, qs, ws), per_bucket=3)
        rows, tiles = at.shapes_for(qs, ws, table)
        assert rows is not None
        l0, d0 = h.search_batched(dx, qs, ws)
        l1, d1 = h.search_batched(dx, qs, ws, rows=rows, tiles=tiles)
        np.testing.assert_array_equal(l0, l1)
        np.testing.assert_allclose(d0, d1, rtol=1e-5)
        variants = at.tune_variants(sorted(set(ws)), at.gpu_variant_measure(h, dx, qs[0]))
        at.apply_variants(h, variants)
        at.save(torch.cuda.get_device_name(0), {"batched": table, "variants": variants},
                str(tmp_path / "c.json"))
        assert at.load(torch.cuda.get_device_name(0), str(tmp_path / "c.json"))["variants"]
