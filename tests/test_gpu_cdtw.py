"""GPU parity: windowed statistics and unpruned all-windows cDTW through the C
ABI against the FP64 oracle, and the all-windows argmin against the UCR Suite
golden results.  Tolerance: the north-star 1e-4 relative distance error
(plus 1e-5 absolute for distances near zero), stated per case below."""
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


def _all_windows(h, q, x, w, metric=0):
    dx = _dev(x)
    avg, std = h.avg_std(dx, q.size)
    h.set_query(q, w)
    out = h.gpu_cdtw(dx, avg, std, metric=metric)
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.float64)


def test_avg_std_matches_oracle_on_level_shifted_stream(handle):
    x = synth.metal_like(400_000, seed=7)  # values in the thousands
    for m in (64, 128, 1000):
        avg, std = handle.avg_std(_dev(x), m)
        mu, sd = oracle.window_stats(x, m)
        got_mu, got_sd = avg.cpu().numpy(), std.cpu().numpy().astype(np.float64)
        # mean to ~1e-12 relative of the level; sigma to FP32 rounding
        assert np.max(np.abs(got_mu - mu) / np.maximum(np.abs(mu), 1.0)) < 1e-11
        assert np.max(np.abs(got_sd - sd) / sd) < 2e-7


def test_avg_std_constant_window_sigma_one(handle):
    x = np.ones(5000, np.float32) * 3.5
    x[2500:] = np.arange(2500, dtype=np.float32)
    avg, std = handle.avg_std(_dev(x), 100)
    s = std.cpu().numpy()
    assert np.all(s[:2401] == 1.0)  # variance 0 -> sigma 1 (stats.cuh:50)
    assert np.all(s[2500:] > 1.0)


def test_all_windows_matches_oracle_golden(handle, golden):
    meta, load = golden
    for c in meta["cases"]:
        x, q = load(c["name"])
        got = _all_windows(handle, q, x, c["W"])
        ref = oracle.cdtw_all(q, x, c["W"])
        np.testing.assert_allclose(got, ref, rtol=RTOL, atol=ATOL, err_msg=c["name"])
        loc = int(np.argmin(got))
        assert loc == c["ucr_location"], c["name"]
        assert abs(np.sqrt(got[loc]) - c["ucr_distance"]) <= 1e-4 * c["ucr_distance"]


@pytest.mark.parametrize("w", [0, 1, 2, 3, 5, 8, 13, 17, 24, 31, 40])
def test_all_windows_every_band(handle, w):
    x = synth.ecg_like(6000, seed=w + 1)
    m = 96
    q, _ = synth.cut_query(x, m, seed=w, noise=0.1)
    got = _all_windows(handle, q, x, w)
    np.testing.assert_allclose(got, oracle.cdtw_all(q, x, w), rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("m", [11, 13, 64, 127, 130, 255, 301])
def test_all_windows_ragged_lengths(handle, m):
    x = synth.metal_like(9000, seed=m)
    q, _ = synth.cut_query(x, m, seed=m, noise=0.2)
    w = synth.band_from_percent(m, 10)
    got = _all_windows(handle, q, x, w)
    np.testing.assert_allclose(got, oracle.cdtw_all(q, x, w), rtol=RTOL, atol=ATOL)


def test_manhattan_metric(handle):
    x = synth.ecg_like(5000, seed=3)
    q, _ = synth.cut_query(x, 128, seed=4, noise=0.1)
    got = _all_windows(handle, q, x, 12, metric=1)
    np.testing.assert_allclose(got, oracle.cdtw_all(q, x, 12, euclid=False), rtol=RTOL, atol=ATOL)


def test_index_list_and_host_path(handle):
    x = synth.ecg_like(20000, seed=8)
    q, _ = synth.cut_query(x, 128, seed=8, noise=0.05)
    dx = _dev(x)
    avg, std = handle.avg_std(dx, 128)
    handle.set_query(q, 12)
    rng = np.random.default_rng(0)
    idx = rng.permutation(x.size - 127)[:3000].astype(np.int32)
    got = handle.gpu_cdtw(dx, avg, std, indices=_dev(idx)).cpu().numpy()
    full = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
    np.testing.assert_array_equal(got, full[idx])
    host = handle.all_windows_host(q, x, 12)
    np.testing.assert_array_equal(host, full)


def test_query_on_device_equals_host(handle):
    x = synth.ecg_like(8000, seed=2)
    q, _ = synth.cut_query(x, 100, seed=2, noise=0.05)
    dx = _dev(x)
    avg, std = handle.avg_std(dx, 100)
    handle.set_query(q, 10)
    a = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
    handle.set_query(_dev(q), 10)
    b = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
    np.testing.assert_array_equal(a, b)


def test_errors_are_status_codes(handle):
    from cudadtw_b200 import CudaDTWError
    x = _dev(np.zeros(100, np.float32))
    with pytest.raises(CudaDTWError) as e:
        handle.avg_std(x, 200)  # M > N
    assert e.value.status == 1
    with pytest.raises(CudaDTWError):
        handle.set_query(np.zeros(0, np.float32), 3)


@pytest.mark.parametrize("m,w,nwin", [(128, 41, 3000), (256, 51, 3000), (300, 62, 2000),
                                      (300, 63, 2000), (512, 102, 1500), (1024, 204, 600),
                                      (2048, 409, 200), (777, 300, 300)])
def test_all_windows_wide_bands(handle, m, w, nwin):
    """Bands above the register-band limit: the lane-group kernel (the
    strip kernel where no lane shape fits)."""
    x = synth.metal_like(m + nwin - 1, seed=w)
    q, _ = synth.cut_query(x, m, seed=w, noise=0.2)
    got = _all_windows(handle, q, x, w)
    np.testing.assert_allclose(got, oracle.cdtw_all(q, x, w), rtol=RTOL, atol=ATOL)
    got1 = _all_windows(handle, q, x, w, metric=1)
    np.testing.assert_allclose(got1, oracle.cdtw_all(q, x, w, euclid=False), rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("m,w", [(200, 27), (300, 60), (400, 96), (260, 97), (700, 150),
                                 (1024, 204), (1100, 383), (1500, 384), (2048, 409),
                                 (1600, 767)])
def test_all_windows_variants_bit_identical(handle, m, w):
    """The lane-group kernel (band over a group of lanes, two windows per
    group), the strip kernels and the register band compute every cell with
    the same operations: their all-windows outputs are bit-identical, for
    both costs, across lane shapes (4 to 32 lanes of 18 to 48 cells) and at
    the bands no lane shape fits (384), and stay within 1e-4 of the oracle."""
    from cudadtw_b200 import autotune as at
    nwin = 700
    x = synth.metal_like(m + nwin - 1, seed=m + w)
    q, _ = synth.cut_query(x, m, seed=w, noise=0.2)
    dx = _dev(x)
    avg, std = handle.avg_std(dx, m)
    handle.set_query(q, w)
    variants = ["strip16"] + (["register"] if w <= 96 else []) + \
        (["lane"] if at.lane_shape(w) else [])
    for metric in (0, 1):
        outs = {}
        for v in variants:
            handle.set_band_variant(w, w, v)
            outs[v] = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
        handle.set_band_variant(w, w, "auto")
        auto = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
        for v in variants:
            np.testing.assert_array_equal(outs[v], auto, err_msg=v)
        ref = oracle.cdtw_all(q, x, w, euclid=(metric == 0))
        np.testing.assert_allclose(auto.astype(np.float64), ref, rtol=RTOL, atol=ATOL)


def test_lane_kernel_index_list(handle):
    x = synth.ecg_like(20000, seed=15)
    q, _ = synth.cut_query(x, 512, seed=15, noise=0.05)
    dx = _dev(x)
    avg, std = handle.avg_std(dx, 512)
    handle.set_query(q, 150)
    idx = np.random.default_rng(3).permutation(x.size - 511)[:501].astype(np.int32)
    idx[8] = -3  # outside the subject: NaN, no access
    got = handle.gpu_cdtw(dx, avg, std, indices=_dev(idx)).cpu().numpy()
    full = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
    assert np.isnan(got[8])
    keep = np.arange(idx.size) != 8
    np.testing.assert_array_equal(got[keep], full[idx[keep]])


def test_strip_kernel_index_list(handle):
    x = synth.ecg_like(20000, seed=5)
    q, _ = synth.cut_query(x, 512, seed=5, noise=0.05)
    dx = _dev(x)
    avg, std = handle.avg_std(dx, 512)
    handle.set_query(q, 102)
    handle.set_band_variant(102, 102, "strip16")
    idx = np.random.default_rng(1).permutation(x.size - 511)[:500].astype(np.int32)
    idx[7] = x.size  # outside the subject: NaN, no access
    got = handle.gpu_cdtw(dx, avg, std, indices=_dev(idx)).cpu().numpy()
    full = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
    handle.set_band_variant(102, 102, "auto")
    assert np.isnan(got[7])
    keep = np.arange(idx.size) != 7
    np.testing.assert_array_equal(got[keep], full[idx[keep]])


@pytest.mark.parametrize("W", [12, 60, 120])
def test_host_call_pipelined_chunks_equal_device_path(handle, W):
    """cdtw_all_windows_host pipelines copies and compute over window chunks;
    with chunk starts on the statistics kernel's 2048-window runs its results
    are bit-identical to the device-buffer path (several chunks, ragged tail,
    the two-window, one-window and strip kernels)."""
    x = synth.metal_like((1 << 21) + 777, seed=9)
    q, _ = synth.cut_query(x, 160, seed=10, noise=0.1)
    dx = _dev(x)
    avg, std = handle.avg_std(dx, q.size)
    handle.set_query(q, W)
    full = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
    host = handle.all_windows_host(q, x, W)
    np.testing.assert_array_equal(host, full)
