"""Top-k non-overlapping matches (cdtw_topk) through the C ABI.

The pruned top-k must equal the greedy non-overlapping selection, in
(distance, window) order, over the unpruned all-windows cDTW of the same
query (cdtw_gpu_cdtw, the same cDTW arithmetic, so the comparison is exact):
no window the selection needs may be pruned by the threshold.  Distances are
also checked against the FP64 oracle at the 1e-4 relative tolerance."""
import numpy as np
import pytest
import torch

import oracle
from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu


def greedy(d, k, M):
    order = np.lexsort((np.arange(d.size), d))
    taken = []
    for w in order:
        if len(taken) == k or not np.isfinite(d[w]):
            break
        if all(abs(int(w) - t) >= M for t in taken):
            taken.append(int(w))
    return np.array(taken, np.int64)


@pytest.fixture(scope="module")
def handle():
    from cudadtw_b200 import Handle
    with Handle(0) as h:
        yield h


@pytest.mark.parametrize("kind,n,M,P,k,metric", [
    ("ecg", 1 << 16, 64, 10, 20, 0),
    ("ecg", 1 << 16, 128, 20, 50, 0),
    ("metal", 1 << 16, 96, 5, 30, 0),
    ("ecg", 1 << 15, 64, 10, 25, 1),
    ("ecg", 4000, 64, 10, 1000, 0),   # fewer non-overlapping windows than k
])
def test_topk_equals_greedy_over_all_windows(handle, kind, n, M, P, k, metric):
    x = synth.ecg_like(n, seed=7) if kind == "ecg" else synth.metal_like(n, seed=8)
    q, _ = synth.cut_query(x, M, seed=9, noise=0.05)
    W = synth.band_from_percent(M, P)
    dx = torch.from_numpy(x).cuda()
    avg, std = handle.avg_std(dx, M)
    handle.set_query(q, W)
    locs, dists = handle.topk(dx, avg, std, k, metric=metric)
    full = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
    want = greedy(full, k, M)
    np.testing.assert_array_equal(locs, want)
    printed = np.sqrt(full[want]) if metric == 0 else full[want]
    np.testing.assert_allclose(dists, printed, rtol=1e-6)
    ref = oracle.cdtw_all(q, x, W, euclid=(metric == 0))
    np.testing.assert_allclose(full[want], ref[want], rtol=1e-4, atol=1e-5)
    if k < 1000:
        assert locs.size == k
    assert np.all(np.diff(np.sort(locs)) >= M)


@pytest.mark.parametrize("kind,n,M,P,k,metric", [
    ("ecg", 1 << 16, 64, 10, 20, 0),
    ("ecg", 1 << 16, 128, 20, 50, 1),
    ("metal", 1 << 17, 96, 5, 200, 0),
    ("walk", 1 << 16, 200, 10, 40, 0),    # random walk: dense candidate valleys
    ("ecg", 1 << 18, 64, 10, 1000, 0),    # several ordered key blocks in the greedy
    ("ecg", 4000, 64, 10, 1000, 0),       # fewer non-overlapping windows than k
])
def test_topk_device_equals_host_topk(handle, kind, n, M, P, k, metric):
    """cdtw_topk_device (threshold, collection and greedy selection on the
    device) returns exactly cdtw_topk's picks and distances."""
    x = {"ecg": lambda: synth.ecg_like(n, seed=7), "metal": lambda: synth.metal_like(n, seed=8),
         "walk": lambda: synth.random_walk(n, 9)}[kind]()
    q, _ = synth.cut_query(x, M, seed=9, noise=0.05)
    W = synth.band_from_percent(M, P)
    dx = torch.from_numpy(x).cuda()
    avg, std = handle.avg_std(dx, M)
    handle.set_query(q, W)
    hl, hd = handle.topk(dx, avg, std, k, metric=metric)
    dl, dd = handle.topk_device(dx, avg, std, k, metric=metric)
    np.testing.assert_array_equal(dl, hl)
    np.testing.assert_array_equal(dd, hd)
    if n > 4000:
        full = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
        np.testing.assert_array_equal(dl, greedy(full, k, M))


@pytest.mark.parametrize("variant", ["lane", "strip16", "auto"])
def test_topk_device_wide_band_variants(handle, variant):
    """Wide bands (W = 102): the candidates under the threshold are collected
    by the lane-group or strip search kernels' hit list; the picks equal
    cdtw_topk's and the greedy over the unpruned all-windows cDTW."""
    x = synth.metal_like(1 << 17, seed=12)
    M, W, k = 512, 102, 30
    q, _ = synth.cut_query(x, M, seed=13, noise=0.2)
    dx = torch.from_numpy(x).cuda()
    avg, std = handle.avg_std(dx, M)
    handle.set_query(q, W)
    handle.set_band_variant(W, W, variant)
    try:
        for metric in (0, 1):
            hl, hd = handle.topk(dx, avg, std, k, metric=metric)
            dl, dd = handle.topk_device(dx, avg, std, k, metric=metric)
            np.testing.assert_array_equal(dl, hl)
            np.testing.assert_array_equal(dd, hd)
            full = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
            np.testing.assert_array_equal(dl, greedy(full, k, M))
    finally:
        handle.set_band_variant(W, W, "auto")


def test_topk_errors(handle):
    from cudadtw_b200 import CudaDTWError
    x = torch.from_numpy(synth.ecg_like(5000, seed=1)).cuda()
    handle.set_query(np.random.default_rng(0).standard_normal(8).astype(np.float32), 2)
    avg, std = handle.avg_std(x, 8)
    with pytest.raises(CudaDTWError):
        handle.topk(x, avg, std, 5)
