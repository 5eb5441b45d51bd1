"""GPU-LDTW in the reference's own FP32 arithmetic against the reference's own
code: the host templates z_serial_ldtw / serial_ldtw of include/ldtw.cuh,
built from the reference sources into oracle/_ref/ref_ldtw and fed the
inputs its GPU-ldtw.cu makes (FP32 query z-normalisation, avg_std window
statistics).

Per window the device and the reference code do the same float operations;
the only difference is the window sums (direct FP64 sums here, differences
of FP64 prefix sums there), equal to a few FP64 ulps, which moves a window's
float mean or E[x^2] by one ulp in a few windows per million.  So the test
asserts the per-window costs equal at 1e-6 relative for all but 1e-4 of the
windows, the index of the first strict minimum equal, and the same through
the GPU-LDTW driver's stdout."""
import os
import re
import subprocess

import numpy as np
import pytest
import torch

import oracle
from cudadtw_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVERS = os.path.join(ROOT, "cudadtw_b200", "drivers")

CASES = [("ecg", 30000, 128, 10, 0.05), ("ecg", 20000, 64, 5, 0.1), ("metal", 40000, 256, 10, 0.1),
         ("walk", 25000, 200, 20, 0.5), ("metal", 30000, 100, 0, 0.2)]


def _stream(kind, n, seed):
    if kind == "ecg":
        return synth.ecg_like(n, seed=seed)
    if kind == "metal":
        return synth.metal_like(n, seed=seed)
    return synth.random_walk(n, seed)


@pytest.fixture(scope="module")
def handle():
    from cudadtw_b200 import Handle
    with Handle(0) as h:
        yield h


@pytest.mark.parametrize("kind,n,m,p,noise", CASES)
@pytest.mark.parametrize("znorm", [True, False])
def test_ldtw_reference_arithmetic_matches_reference_code(handle, kind, n, m, p, noise, znorm):
    x = _stream(kind, n, seed=n + m)
    q, _ = synth.cut_query(x, m, seed=m + p, noise=noise)
    w = synth.band_from_percent(m, p)
    if not znorm:  # the tsh2 line of GPU-ldtw.cu: the driver-normalised query, raw windows
        q = ((q - q.mean()) / q.std()).astype(np.float32)
    ref, ref_loc = oracle.ref_ldtw(q, x, w, znorm=znorm)
    dx = torch.from_numpy(x).cuda()
    handle.set_query(q, w)
    got = handle.ldtw_ref_all_windows(dx, znorm=znorm).cpu().numpy()
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-30)
    assert np.mean(rel > 1e-6) <= 1e-4, (np.mean(rel > 1e-6), rel.max())
    loc = int(np.argmin(got))
    assert loc == ref_loc or got[loc] == ref[ref_loc]
    hloc, hdist = handle.ldtw_ref_search_host(q, x, w, znorm=znorm)
    assert hloc == loc and hdist == np.float32(np.sqrt(got[loc]))


def test_gpu_ldtw_driver_reports_the_reference_index(tmp_path):
    for kind, n, m, p, noise in CASES[:3]:
        x = _stream(kind, n, seed=n + m)
        q, _ = synth.cut_query(x, m, seed=m + p, noise=noise)
        w = synth.band_from_percent(m, p)
        _, ref_loc = oracle.ref_ldtw(q, x, w)
        qf, xf = tmp_path / "q.bin", tmp_path / "s.bin"
        q.astype(np.float32).tofile(qf)
        x.astype(np.float32).tofile(xf)
        r = subprocess.run([os.path.join(DRIVERS, "GPU-LDTW"), str(qf), str(xf), str(m), str(n),
                            str(p)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        loc = int(re.search(r"found at index (\d+)", r.stdout).group(1))
        assert loc == ref_loc, (kind, m, p)
