"""GPU tests of cdtw_all_windows_noalloc, the all-windows cDTW entry point that
allocates nothing.

It serves callers that cannot let the library allocate device memory: a host
that owns the device memory budget and lends the library only the buffers of
one call, or a pipeline whose other streams cannot absorb the device-wide
synchronisation of cudaMalloc/cudaFree.  Its working memory is one fixed
device array shared by all calls, so successive calls are checked against the
handle path (set_query + avg_std + gpu_cdtw), in both orders of size, where a
stale query pack or statistics left by an earlier call would show up; the
device's free memory is checked to stay the same across the calls.  The two
paths run the same kernels on the same inputs, so the results must be
bit-identical.  The file name makes pytest collect it last; one test also runs
the calls in a fresh child process, where the entry point's first call on the
device comes before anything else touches the GPU."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _noalloc(lib, dq, M, dx, W, metric, out):
    err = ctypes.create_string_buffer(256)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib.cdtw_all_windows_noalloc(ctypes.c_void_p(dq.data_ptr()), M,
                                      ctypes.c_void_p(dx.data_ptr()), dx.numel(), W, metric,
                                      ctypes.c_void_p(out.data_ptr()), stream, err, 256)
    return st, err.value.decode()


def _cases():
    """(stream, query, M, W, metric): a small and a large call."""
    out = []
    for x, m, w, metric in ((synth.ecg_like(30000, seed=21), 128, 12, 0),
                            (synth.metal_like(60000, seed=22), 300, 30, 1)):
        q, _ = synth.cut_query(x, m, seed=m, noise=0.1)
        out.append((x, q, m, w, metric))
    return out


def _check_noalloc_against_handle(order):
    """Runs the handle path for every case, then the no-alloc call for the
    cases in `order` (twice through); returns (results equal, free-memory
    deltas after the first pass)."""
    from cudadtw_b200 import Handle
    from cudadtw_b200._lib import load
    lib = load()
    cases = _cases()
    dev = [(torch.from_numpy(x).cuda(), torch.from_numpy(q).cuda()) for x, q, _, _, _ in cases]
    outs = [torch.full((x.size - m + 1,), float("nan"), device="cuda")
            for x, _, m, _, _ in cases]
    torch.cuda.synchronize()
    # no-alloc calls first (in a fresh process this is the first GPU work of
    # the library), then the handle path as the check
    got = {}
    free = []
    for rep in range(2):
        for i in order:
            _, _, m, w, metric = cases[i]
            dx, dq = dev[i]
            outs[i].fill_(float("nan"))
            st, msg = _noalloc(lib, dq, m, dx, w, metric, outs[i])
            assert st == 0, msg
            torch.cuda.synchronize()
            got[(rep, i)] = outs[i].cpu().numpy().copy()
        free.append(torch.cuda.mem_get_info()[0])
    with Handle(0) as h:
        for i, (x, q, m, w, metric) in enumerate(cases):
            dx, dq = dev[i]
            avg, std = h.avg_std(dx, m)
            h.set_query(dq, w)
            ref = h.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
            for rep in range(2):
                g = got[(rep, i)]
                assert np.all(np.isfinite(g))
                np.testing.assert_array_equal(g, ref)
    return free


def test_noalloc_matches_handle_path_small_then_large():
    free = _check_noalloc_against_handle([0, 1])
    # the second pass through the same calls takes no device memory
    assert free[0] == free[1]


def test_noalloc_matches_handle_path_large_then_small():
    free = _check_noalloc_against_handle([1, 0])
    assert free[0] == free[1]


def test_noalloc_first_call_in_fresh_process():
    code = ("import sys; sys.path.insert(0, %r); sys.path.insert(0, %r); "
            "import test_zz_no_alloc as t; t._check_noalloc_against_handle([1, 0]); print('ok')"
            % (ROOT, os.path.join(ROOT, "tests")))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


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
    st, msg = _noalloc(lib, q, 128, x[:4096], 60, 0, out)
    assert st == 5 and "band" in msg
