"""Full-size searches pinned to the reference's own CPU search, UCR_DTW_BIN
(built from the reference sources into oracle/_ref), on identical inputs.

* The 2^20-sample ECG-like stream with a length-128 query (band 10 %: W=12,
  and the absolute band W=13): UCR runs on the whole stream (about 2 s).
* The 2^25-sample metal-like stream (level shifts of N(0, 20): the case where
  the reference GPU path's FP32 variance loses the window statistics):
  M in {128, 256} at P in {5, 10, 20}, M=512 at P in {5, 10} and M=1024 at
  P=5, with UCR run as concurrent shard processes over the windows (each
  shard with the M-1 samples that follow), combined by the FP64 oracle.

Each case asserts the same location as UCR, and the distance within 1e-4
relative of UCR's printed value and of the FP64 oracle at that window.  The
remaining 2^25 cases (M=512 at P=20, M=1024 at P=10 and 20, each a minute or
more of UCR on every core) assert the pruned search against the argmin of the
unpruned all-windows cDTW over every window, and the FP64 oracle at the
reported window.  The queries are the benchmark's (bench.py sub-results)."""
import numpy as np
import pytest
import torch

import oracle
from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu

RTOL = 1e-4


@pytest.fixture(scope="module")
def handle():
    from cudadtw_b200 import Handle
    with Handle(0) as h:
        yield h


def _search(h, dx, q, w, metric=0):
    avg, std = h.avg_std(dx, q.size)
    h.set_query(q, w)
    loc, dist = h.prune_cdtw(dx, avg, std, metric=metric)
    return int(loc), float(dist), (avg, std)


def _fp64_dist(q, x, w, loc):
    return float(np.sqrt(oracle.cdtw_list(q, x, w, np.array([loc]))[0]))


@pytest.mark.parametrize("w", [12, 13])
def test_config0_full_size_matches_ucr(handle, w):
    x = synth.ecg_like(1 << 20, seed=0)
    q, _ = synth.cut_query(x, 128, seed=100 + 128 + 10, noise=0.05)
    dx = torch.from_numpy(x).cuda()
    loc, dist, _ = _search(handle, dx, q, w)
    uloc, udist, _, _ = oracle.ucr_dtw(x, q, oracle.ucr_band_arg(w, 128))
    assert loc == uloc
    assert abs(dist - udist) <= RTOL * udist
    ref = _fp64_dist(q, x, w, loc)
    assert abs(dist - ref) <= RTOL * ref


@pytest.fixture(scope="module")
def metal():
    x = synth.metal_like(1 << 25, seed=1)
    with oracle.UcrShards(x, max_m=1024) as ucr:
        yield x, torch.from_numpy(x).cuda(), ucr


@pytest.mark.parametrize("m,p", [(128, 5), (128, 10), (128, 20), (256, 5), (256, 10),
                                 (256, 20), (512, 5), (512, 10), (1024, 5)])
def test_config1_full_size_matches_ucr(handle, metal, m, p):
    x, dx, ucr = metal
    q, _ = synth.cut_query(x, m, seed=100 + m + p, noise=0.1)
    w = synth.band_from_percent(m, p)
    loc, dist, _ = _search(handle, dx, q, w)
    uloc, udist, _, _ = ucr.search(q, w)
    assert loc == uloc, (m, p)
    assert abs(dist - udist) <= RTOL * udist
    ref = _fp64_dist(q, x, w, loc)
    assert abs(dist - ref) <= RTOL * ref


@pytest.mark.parametrize("m,p", [(512, 20), (1024, 10), (1024, 20)])
def test_config1_wide_bands_equal_unpruned_argmin(handle, metal, m, p):
    x, dx, _ = metal
    q, _ = synth.cut_query(x, m, seed=100 + m + p, noise=0.1)
    w = synth.band_from_percent(m, p)
    loc, dist, (avg, std) = _search(handle, dx, q, w)
    allw = handle.gpu_cdtw(dx, avg, std)
    best = int(torch.argmin(allw).item())
    assert loc == best
    assert dist == np.float32(np.sqrt(allw[best].item()))
    ref = _fp64_dist(q, x, w, loc)
    assert abs(dist - ref) <= RTOL * ref
