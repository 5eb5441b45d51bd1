"""GPU parity of the lower bounds and the pruned search.

Bounds: against the FP64 oracle at 1e-4 relative, and the reference's own
property test (tests/test_dtwbounds.cu:129-149: no bound above cDTW).
Search: the location equals the UCR Suite's on every golden case and equals
the argmin of the unpruned all-windows cDTW (pruning changes nothing), the
distance is within 1e-4 relative of UCR / the FP64 oracle."""
import numpy as np
import pytest
import torch

import oracle
from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-4, 1e-5


@pytest.fixture(scope="module")
def handle():
    from cudadtw_b200 import Handle
    with Handle(0) as h:
        yield h


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _prep(h, q, x, w):
    dx = _dev(x)
    avg, std = h.avg_std(dx, q.size)
    h.set_query(q, w)
    return dx, avg, std


@pytest.mark.parametrize("m,w", [(128, 12), (64, 3), (200, 40), (256, 51)])
def test_bounds_match_oracle_and_stay_below_cdtw(handle, m, w):
    x = synth.ecg_like(8000, seed=m + w)
    q, _ = synth.cut_query(x, m, seed=w, noise=0.2)
    for metric, eu in ((0, True), (1, False)):
        dx, avg, std = _prep(handle, q, x, w)
        kim = handle.lb_kim(dx, avg, std, metric=metric).cpu().numpy()
        fwd, rev = handle.lb_keogh(dx, avg, std, metric=metric)
        fwd, rev = fwd.cpu().numpy(), rev.cpu().numpy()
        d = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
        np.testing.assert_allclose(kim, oracle.lb_kim(q, x, eu), rtol=RTOL, atol=ATOL)
        np.testing.assert_allclose(fwd, oracle.lb_keogh(q, x, w, eu), rtol=RTOL, atol=ATOL)
        np.testing.assert_allclose(rev, oracle.lb_keogh_rev(q, x, w, eu), rtol=RTOL, atol=ATOL)
        for lb in (kim, fwd, rev):
            assert np.all(lb <= d * (1 + 1e-5) + 1e-4)


def test_bounds_index_list(handle):
    x = synth.metal_like(30000, seed=3)
    q, _ = synth.cut_query(x, 300, seed=3, noise=0.1)
    dx, avg, std = _prep(handle, q, x, 30)
    idx = np.random.default_rng(2).permutation(x.size - 299)[:777].astype(np.int32)
    kim_all = handle.lb_kim(dx, avg, std).cpu().numpy()
    kim = handle.lb_kim(dx, avg, std, indices=_dev(idx)).cpu().numpy()
    np.testing.assert_array_equal(kim, kim_all[idx])
    f_all, r_all = handle.lb_keogh(dx, avg, std)
    f, r = handle.lb_keogh(dx, avg, std, indices=_dev(idx))
    np.testing.assert_array_equal(f.cpu().numpy(), f_all.cpu().numpy()[idx])
    np.testing.assert_array_equal(r.cpu().numpy(), r_all.cpu().numpy()[idx])


def test_lb_kim_needs_11_samples(handle):
    from cudadtw_b200 import CudaDTWError
    x = synth.ecg_like(2000, seed=1)
    q = x[100:110].copy()
    dx, avg, std = _prep(handle, q, x, 2)
    with pytest.raises(CudaDTWError):
        handle.lb_kim(dx, avg, std)


def test_search_matches_ucr_golden(handle, golden):
    meta, load = golden
    for c in meta["cases"]:
        x, q = load(c["name"])
        dx, avg, std = _prep(handle, q, x, c["W"])
        loc, dist = handle.prune_cdtw(dx, avg, std)
        assert loc == c["ucr_location"], c["name"]
        assert abs(dist - c["ucr_distance"]) <= 1e-4 * c["ucr_distance"], c["name"]
        allw = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
        assert loc == int(np.argmin(allw))
        assert dist == np.float32(np.sqrt(allw.min()))


@pytest.mark.parametrize("kind,m,p", [("ecg", 128, 10), ("ecg", 128, 20), ("metal", 128, 5),
                                      ("metal", 256, 10), ("metal", 512, 20), ("ecg", 1024, 10),
                                      ("walk", 333, 20), ("ecg", 64, 5)])
def test_search_equals_unpruned_argmin(handle, kind, m, p):
    n = 60000 if m < 1024 else 20000
    x = {"ecg": synth.ecg_like, "metal": synth.metal_like,
         "walk": lambda n, seed: synth.random_walk(n, seed)}[kind](n, seed=m + p)
    q, _ = synth.cut_query(x, m, seed=p, noise=0.1)
    w = synth.band_from_percent(m, p)
    for metric in (0, 1):
        dx, avg, std = _prep(handle, q, x, w)
        loc, dist = handle.prune_cdtw(dx, avg, std, metric=metric)
        allw = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
        assert loc == int(np.argmin(allw))
        best = allw.min()
        assert dist == np.float32(np.sqrt(best) if metric == 0 else best)
        nw, nkim, ndtw = handle.search_counts()
        assert nw == x.size - m + 1 and 0 < ndtw <= nkim <= nw
        # the reference's termination flag (cdtw.cuh:585): best < largest LB_Kim
        kim = handle.lb_kim(dx, avg, std, metric=metric).cpu().numpy()
        assert handle.search_flag() == int(np.float32(best) < kim.max())
        ref = oracle.cdtw_list(q, x, w, np.array([loc]), euclid=(metric == 0))[0]
        ref = np.sqrt(ref) if metric == 0 else ref
        assert abs(dist - ref) <= 1e-4 * ref


@pytest.mark.parametrize("kind,m,p,noise", [("metal", 1024, 20, 1.0), ("walk", 800, 20, 1.0)])
def test_search_wavefront_survivor_range(handle, kind, m, p, noise):
    """Cases whose bound survivors (about 1.1-1.4 thousand by the FP64
    oracle's bounds against the best distance) fall in the range that runs as
    pairwise wavefronts (more than 512, at most 8192, with at least 4e4 band
    cells per window): location and distance equal the unpruned argmin's."""
    x = {"metal": synth.metal_like,
         "walk": lambda n, seed: synth.random_walk(n, seed)}[kind](60000, seed=m + p)
    q, _ = synth.cut_query(x, m, seed=p, noise=noise)
    w = synth.band_from_percent(m, p)
    assert m * (2 * w + 1) - w * (w + 1) >= 4e4
    for metric in (0, 1):
        dx, avg, std = _prep(handle, q, x, w)
        loc, dist = handle.prune_cdtw(dx, avg, std, metric=metric)
        allw = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
        assert loc == int(np.argmin(allw))
        best = allw.min()
        assert dist == np.float32(np.sqrt(best) if metric == 0 else best)
        if metric == 0:
            _, _, ndtw = handle.search_counts()
            assert 512 < ndtw <= 8192, ndtw


@pytest.mark.parametrize("m,p", [(700, 20), (1024, 10), (300, 50)])
def test_search_variants_agree(handle, m, p):
    """ECG-like streams with a noisy query: tens of thousands of windows
    survive the bounds, so the survivors run on the early-abandoning kernels
    (lane groups, or the strips): every variant gives the unpruned argmin."""
    x = synth.ecg_like(40000, seed=m + p)
    q, _ = synth.cut_query(x, m, seed=p, noise=0.3)
    w = synth.band_from_percent(m, p)
    dx, avg, std = _prep(handle, q, x, w)
    for metric in (0, 1):
        allw = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
        best = allw.min()
        want = (int(np.argmin(allw)), np.float32(np.sqrt(best) if metric == 0 else best))
        for v in ("lane", "strip16", "strip32"):
            handle.set_band_variant(w, w, v)
            loc, dist = handle.prune_cdtw(dx, avg, std, metric=metric)
            assert (loc, dist) == want, v
        handle.set_band_variant(w, w, "auto")
        _, _, ndtw = handle.search_counts()
        assert ndtw > 8192


def test_search_host_path_and_ties(handle):
    x = synth.ecg_like(40000, seed=9)
    q, off = synth.cut_query(x, 128, seed=9, noise=0.0)
    # plant an exact copy of the window later: equal distances -> lowest index
    x[30000:30128] = x[off:off + 128]
    loc, dist = handle.search_host(q, x, 12)
    assert loc in (off, 30000) and dist < 1e-2
    dx, avg, std = _prep(handle, q, x, 12)
    assert handle.prune_cdtw(dx, avg, std) == (loc, dist)
    allw = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
    assert loc == int(np.argmin(allw))  # lowest index among equal distances


@pytest.mark.parametrize("m,w", [(128, 12), (300, 60), (512, 102), (96, 0)])
def test_search_exact_match_beats_seed_bound(handle, m, w):
    """A query equal to one of the windows (distance about 0).  The seeds'
    pairwise cDTW gives the search only an upper bound (raised a little, with
    no window); the exact window must replace it, for both metrics and for
    register-band and strip bands."""
    x = synth.metal_like(50000, seed=m + w)
    q, off = synth.cut_query(x, m, seed=w + 3, noise=0.0)
    for metric in (0, 1):
        dx, avg, std = _prep(handle, q, x, w)
        loc, dist = handle.prune_cdtw(dx, avg, std, metric=metric)
        allw = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
        best = allw.min()
        assert loc == int(np.argmin(allw)) and best < 1e-3
        assert dist == np.float32(np.sqrt(best) if metric == 0 else best)


def test_search_with_constant_windows(handle):
    x = synth.ecg_like(20000, seed=4)
    x[5000:7000] = 2.0  # zero-variance windows: sigma = 1 (stats.cuh:50)
    q, off = synth.cut_query(x, 128, seed=4, noise=0.05)
    dx, avg, std = _prep(handle, q, x, 12)
    loc, dist = handle.prune_cdtw(dx, avg, std)
    allw = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
    assert loc == int(np.argmin(allw))


def test_search_config0_full_size_equals_unpruned(handle):
    """The 2^20-sample ECG-like configuration: pruned search == argmin of the
    unpruned all-windows cDTW, for W=12 (10%) and W=13."""
    x = synth.ecg_like(1 << 20, seed=0)
    q, _ = synth.cut_query(x, 128, seed=12810, noise=0.05)
    for w in (12, 13):
        dx, avg, std = _prep(handle, q, x, w)
        loc, dist = handle.prune_cdtw(dx, avg, std)
        allw = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
        assert loc == int(np.argmin(allw)) and dist == np.float32(np.sqrt(allw.min()))
