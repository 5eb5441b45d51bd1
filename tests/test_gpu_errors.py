"""Error paths of the C ABI, made on the host: every failure comes back as a
status (never a process exit, as the reference's CUERR does,
include/cuda_def.cuh:6-8) and leaves the handle usable.

* a negative band, a too-short query, a bad metric: CDTW_EINVAL (1);
* an allocation refused by the handle's memory limit (cdtw_set_memory_limit):
  CDTW_ENOMEM (2), then the same call succeeds once the limit is lifted;
* NaN / Inf samples: windows holding them have no finite distance and never
  win; a stream whose every window is non-finite is CDTW_EINVAL."""
import numpy as np
import pytest
import torch

from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture()
def handle():
    from cudadtw_b200 import Handle
    with Handle(0) as h:
        yield h


def _status(fn):
    from cudadtw_b200 import CudaDTWError
    try:
        fn()
    except CudaDTWError as e:
        return e.status
    return 0


def test_bad_arguments_are_einval(handle):
    x = synth.ecg_like(5000, seed=1)
    q, _ = synth.cut_query(x, 128, seed=1, noise=0.1)
    assert _status(lambda: handle.set_query(q, -1)) == 1
    assert _status(lambda: handle.search_host(q[:8], x, 2)) == 1
    dx = torch.from_numpy(x).cuda()
    avg, std = handle.avg_std(dx, 128)
    handle.set_query(q, 12)
    import ctypes
    loc, dist = ctypes.c_int64(), ctypes.c_float()
    st = handle._lib.cdtw_prune_cdtw(handle._h, ctypes.c_void_p(dx.data_ptr()), dx.numel(),
                                     ctypes.c_void_p(avg.data_ptr()),
                                     ctypes.c_void_p(std.data_ptr()), 7, ctypes.byref(loc),
                                     ctypes.byref(dist))
    assert st == 1 and b"metric" in handle._lib.cdtw_last_error(handle._h)
    # the handle still works
    loc, dist = handle.prune_cdtw(dx, avg, std)
    assert 0 <= loc < x.size - 127 and np.isfinite(dist)


def test_memory_limit_gives_enomem_and_recovers(handle):
    x = synth.metal_like(200_000, seed=2)
    q, off = synth.cut_query(x, 256, seed=2, noise=0.1)
    handle.set_memory_limit(1 << 20)  # 1 MiB: below what the search needs
    assert _status(lambda: handle.search_host(q, x, 25)) == 2
    handle.set_memory_limit(0)
    loc, dist = handle.search_host(q, x, 25)
    assert abs(loc - off) <= 2 and np.isfinite(dist)
    # a limit above what the handle holds lets the same call run again
    handle.set_memory_limit(1 << 34)
    assert handle.search_host(q, x, 25) == (loc, dist)


def test_nan_and_inf_windows_never_win(handle):
    x = synth.ecg_like(30_000, seed=3)
    q, off = synth.cut_query(x, 128, seed=3, noise=0.05)
    x[off + 10] = np.nan       # the planted window and its neighbours go non-finite
    x[20_000] = np.inf
    dx = torch.from_numpy(x).cuda()
    avg, std = handle.avg_std(dx, 128)
    handle.set_query(q, 12)
    loc, dist = handle.prune_cdtw(dx, avg, std)
    allw = handle.gpu_cdtw(dx, avg, std).cpu().numpy()
    finite = np.where(np.isfinite(allw), allw, np.inf)
    assert loc == int(np.argmin(finite)) and np.isfinite(dist)
    assert not (off - 127 <= loc <= off + 10) and not (20_000 - 127 <= loc <= 20_000)


def test_all_windows_non_finite_is_einval(handle):
    x = np.full(2000, np.nan, dtype=np.float32)
    q = synth.ecg_like(128, seed=4)
    assert _status(lambda: handle.search_host(q, x, 12)) == 1
    qn = q.copy()
    qn[5] = np.inf
    y = synth.ecg_like(4000, seed=5)
    assert _status(lambda: handle.search_host(qn, y, 12)) == 1
    # the handle still works
    loc, _ = handle.search_host(q, y, 12)
    assert 0 <= loc < y.size - 127
