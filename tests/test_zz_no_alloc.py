"""GPU test of cdtw_all_windows_noalloc, the all-windows cDTW entry point that
allocates nothing (for callers that cannot let the library allocate device
memory: hosts that own the device memory budget, or pipelines that cannot
absorb cudaMalloc's device-wide synchronisation).  Its working memory is one
fixed device array shared by all calls, so two calls in a row are checked
against the handle path: a stale query pack or statistics left by the first
call would show up in the second.  The file name makes pytest collect it
last; it also runs alone in a fresh process (the first call does the per-device
address lookup)."""
import ctypes

import numpy as np
import pytest
import torch

from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-4, 1e-5  # the tolerance of the other cDTW parity tests


def _noalloc(lib, dq, M, dx, W, metric, out):
    err = ctypes.create_string_buffer(256)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib.cdtw_all_windows_noalloc(ctypes.c_void_p(dq.data_ptr()), M,
                                      ctypes.c_void_p(dx.data_ptr()), dx.numel(), W, metric,
                                      ctypes.c_void_p(out.data_ptr()), stream, err, 256)
    return st, err.value.decode()


def test_noalloc_matches_handle_path_on_two_calls():
    from cudadtw_b200 import Handle
    from cudadtw_b200._lib import load
    lib = load()
    cases = [  # (stream, M, W, metric): two different calls in a row
        (synth.ecg_like(30000, seed=21), 128, 12, 0),
        (synth.metal_like(60000, seed=22), 300, 30, 1),
    ]
    with Handle(0) as h:
        for x, m, w, metric in cases:
            q, _ = synth.cut_query(x, m, seed=m, noise=0.1)
            dx = torch.from_numpy(x).cuda()
            dq = torch.from_numpy(q).cuda()
            avg, std = h.avg_std(dx, m)
            h.set_query(dq, w)
            ref = h.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
            out = torch.full((x.size - m + 1,), float("nan"), device="cuda")
            st, msg = _noalloc(lib, dq, m, dx, w, metric, out)
            assert st == 0, msg
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            np.testing.assert_allclose(got, ref, rtol=RTOL, atol=ATOL)


def test_noalloc_rejects_sizes_beyond_its_limits():
    from cudadtw_b200._lib import load
    lib = load()
    x = torch.zeros(1 << 21, device="cuda")
    q = torch.arange(128, dtype=torch.float32, device="cuda")
    out = torch.empty(x.numel(), device="cuda")
    st, msg = _noalloc(lib, q, 128, x, 12, 0, out)  # 2^21-127 windows > 2^20
    assert st == 5 and "windows exceed" in msg
    q5 = torch.arange(5000, dtype=torch.float32, device="cuda")
    st, msg = _noalloc(lib, q5, 5000, x, 12, 0, out)
    assert st == 5 and "query length" in msg
