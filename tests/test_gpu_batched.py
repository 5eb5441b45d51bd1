"""GPU parity of the batched search: every query's best match equals the
single-query pruned search (and so the unpruned argmin) -- bit for bit in the
concurrent-pipelines mode, to the tile statistics' rounding in the
persistent-tile mode -- across mixed lengths, bands, both cell costs and
every strip-row choice, and the FP64 oracle's argmin; repeated calls replay
the cached graph with new query values."""
import numpy as np
import pytest
import torch

from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    from cudadtw_b200 import Handle
    with Handle(0) as h:
        yield h


def _single(h, dx, q, w, metric=0):
    avg, std = h.avg_std(dx, q.size)
    h.set_query(q, w)
    return h.prune_cdtw(dx, avg, std, metric=metric)


def _check(h, dx, qs, ws, locs, dists, metric=0):
    for q, w, loc, dist in zip(qs, ws, locs, dists):
        l1, d1 = _single(h, dx, q, w, metric)
        # the batch computes window statistics per tile (different FP64
        # summation order): equal location unless two windows tie at 1e-5
        assert abs(dist - d1) <= 1e-5 * d1 + 1e-6
        if loc != l1:
            allw = h.gpu_cdtw(dx, *h.avg_std(dx, q.size), metric=metric).cpu().numpy()
            v = np.sqrt(allw) if metric == 0 else allw
            assert abs(v[loc] - v[l1]) <= 1e-5 * v[l1]


def test_batched_equals_single_query_search(handle):
    x = synth.ecg_like(300_000, seed=31)
    batch = synth.batch_queries(x, 24, seed=5, m_lo=64, m_hi=700)
    qs = [b[0] for b in batch]
    ws = [b[1] for b in batch]
    dx = torch.from_numpy(x).cuda()
    locs, dists = handle.search_batched(dx, qs, ws)
    _check(handle, dx, qs, ws, locs, dists)
    # replay with new query values (same shapes): the cached graph
    qs2 = [q[::-1].copy() for q in qs]
    locs2, dists2 = handle.search_batched(dx, qs2, ws)
    _check(handle, dx, qs2, ws, locs2, dists2)


@pytest.mark.parametrize("metric", [0, 1])
def test_batched_pipelines_bit_identical_to_single_search(handle, metric):
    """Without tile shapes every query runs the single-query pipeline in one
    of the concurrent lanes of the batch graph: locations and distances equal
    prune_cdtw's exactly, on the first (eager) call, on replays with new
    query values, and after switching to the tile mode and back.  The batch
    mixes register-band, lane-group and strip bands and repeated lengths
    (shared statistics)."""
    x = synth.ecg_like(200_000, seed=51)
    batch = synth.batch_queries(x, 40, seed=9, m_lo=64, m_hi=1500)
    qs = [b[0] for b in batch]
    ws = [b[1] for b in batch]
    qs += [qs[3].copy(), synth.random_walk(1600, 5)]
    ws += [max(1, ws[3] // 2), 800]  # a repeated length; a band above the lane kernels
    dx = torch.from_numpy(x).cuda()

    def check(qv):
        locs, dists = handle.search_batched(dx, qv, ws, metric=metric)
        for q, w, loc, dist in zip(qv, ws, locs, dists):
            assert (loc, dist) == _single(handle, dx, q, w, metric)

    check(qs)
    check([q[::-1].copy() for q in qs])  # replay of the captured graph
    handle.search_batched(dx, qs[:3], ws[:3], metric=metric, rows=[16] * 3)
    check(qs)


@pytest.mark.parametrize("metric", [0, 1])
def test_batched_matches_fp64_oracle(handle, metric):
    """Anchor independent of the plain CUDA path: every query's location is
    the FP64 oracle's argmin over all windows (or ties with it at 1e-5
    relative), its distance within 1e-4 of the oracle at that window."""
    import oracle
    x = synth.ecg_like(40_000, seed=41)
    batch = synth.batch_queries(x, 12, seed=8, m_lo=64, m_hi=200)
    qs = [b[0] for b in batch]
    ws = [b[1] for b in batch]
    dx = torch.from_numpy(x).cuda()
    locs, dists = handle.search_batched(dx, qs, ws, metric=metric)
    eu = metric == 0
    for q, w, loc, dist in zip(qs, ws, locs, dists):
        ref = oracle.cdtw_all(q, x, w, euclid=eu)
        v = np.sqrt(ref) if eu else ref
        best, _ = oracle.argmin(ref)
        assert abs(v[loc] - v[best]) <= 1e-5 * v[best]
        assert abs(dist - v[loc]) <= 1e-4 * v[loc]


@pytest.mark.parametrize("rows", [0, 1, 2, 4, 8, 16])
def test_batched_every_strip_height(handle, rows):
    """rows = 0: register-band main pass; 1..16: strips of that height."""
    x = synth.metal_like(120_000, seed=rows)
    qs, ws = [], []
    for k, m in enumerate((100, 257, 401)):
        q, _ = synth.cut_query(x, m, seed=k + rows, noise=0.1)
        qs.append(q)
        ws.append(max(rows - 1, synth.band_from_percent(m, 10)))
    dx = torch.from_numpy(x).cuda()
    for metric in (0, 1):
        locs, dists = handle.search_batched(dx, qs, ws, metric=metric, rows=[rows] * 3,
                                            tiles=[512, 1024, 2048])
        _check(handle, dx, qs, ws, locs, dists, metric)


def test_batched_rejects_bad_shapes(handle):
    from cudadtw_b200 import CudaDTWError
    dx = torch.zeros(10000, device="cuda")
    with pytest.raises(CudaDTWError):
        handle.search_batched(dx, [np.zeros(8, np.float32)], [2])  # M < 11
    with pytest.raises(CudaDTWError):
        handle.search_batched(dx, [np.arange(100, dtype=np.float32)], [10], tiles=[100])
