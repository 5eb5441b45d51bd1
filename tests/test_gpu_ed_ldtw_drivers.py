"""GPU parity of the GPU-ED and GPU-LDTW paths, and of the three drop-in
drivers end to end (argv, binary files and stdout lines of the reference's
GPU-DTW / GPU-ED / GPU-LDTW), against the UCR Suite golden results and the
FP64 oracle.  ED is FP64 end to end: 1e-9 relative; LDTW is FP64: 1e-9
relative (its greedy branch decisions are exact comparisons)."""
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


@pytest.fixture(scope="module")
def handle():
    from cudadtw_b200 import Handle
    with Handle(0) as h:
        yield h


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("kind,m", [("ecg", 128), ("metal", 256), ("walk", 1000), ("ecg", 8192)])
def test_ed_all_windows_matches_oracle(handle, kind, m):
    n = max(4 * m, 20000)
    x = {"ecg": synth.ecg_like, "metal": synth.metal_like,
         "walk": lambda n, seed: synth.random_walk(n, seed)}[kind](n, seed=m)
    q, _ = synth.cut_query(x, m, seed=m, noise=0.1)
    x64, q64 = x.astype(np.float64), q.astype(np.float64)
    got = handle.ed_all_windows(_dev(q64), _dev(x64)).cpu().numpy()
    ref = oracle.ed_all(q64, x64)
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9 * m)


def test_ed_search_matches_ucr_golden(handle, golden):
    meta, load = golden
    for c in meta["ed_cases"]:
        x, q = load(c["name"])
        loc, dist = handle.ed_search_host(q.astype(np.float64), x.astype(np.float64))
        assert loc == c["ucr_location"], c["name"]
        assert abs(dist - c["ucr_distance"]) <= 6e-6 * c["ucr_distance"]


@pytest.mark.parametrize("m,w", [(128, 12), (64, 0), (100, 25), (300, 60)])
def test_ldtw_matches_oracle(handle, m, w):
    x = synth.ecg_like(12000, seed=m + w)
    q, _ = synth.cut_query(x, m, seed=w, noise=0.1)
    handle.set_query(q, w)
    for metric, eu in ((0, True), (1, False)):
        got = handle.ldtw_all_windows(_dev(x), metric=metric).cpu().numpy()
        np.testing.assert_allclose(got, oracle.ldtw_all(q, x, w, eu), rtol=1e-9, atol=1e-9)
    loc, dist = handle.ldtw_search_host(q, x, w)
    ref = oracle.ldtw_all(q, x, w)
    i, v = oracle.argmin(ref)
    assert loc == i and abs(dist - np.sqrt(v)) <= 1e-9 * np.sqrt(v)


def _run(args):
    return subprocess.run(args, capture_output=True, text=True, timeout=300)


def test_gpu_dtw_driver_matches_ucr(tmp_path, golden):
    meta, load = golden
    for c in meta["cases"]:
        if c["band"][0] != "P":
            continue  # the driver takes a band percentage, as the reference's
        x, q = load(c["name"])
        qf, xf = tmp_path / "q.bin", tmp_path / "s.bin"
        q.astype(np.float32).tofile(qf)
        x.astype(np.float32).tofile(xf)
        r = _run([os.path.join(DRIVERS, "GPU-DTW"), str(qf), str(xf), str(q.size), str(x.size),
                  str(c["band"][1])])
        assert r.returncode == 0, r.stderr
        assert f"window = {c['W']}" in r.stdout
        loc = int(re.search(r"Location: (\d+)", r.stdout).group(1))
        dist = float(re.search(r"Distance: ([0-9.eE+-]+)", r.stdout).group(1))
        assert "best match:" in r.stdout  # the line results/benchCDTW.py parses
        assert loc == c["ucr_location"], c["name"]
        # the termination flag printed after the distance (cdtw.cuh:585):
        # squared best < largest LB_Kim (FP64 oracle)
        flag = int(re.search(r"Distance: [^\n]*\n(\d)\n", r.stdout).group(1))
        assert flag == int(dist * dist < oracle.lb_kim(q, x).max())
        assert abs(dist - c["ucr_distance"]) <= 1e-4 * c["ucr_distance"]


def test_gpu_ed_driver_matches_ucr(tmp_path, golden):
    meta, load = golden
    for c in meta["ed_cases"]:
        x, q = load(c["name"])
        qf, xf = tmp_path / "q.bin", tmp_path / "s.bin"
        q.astype(np.float64).tofile(qf)
        x.astype(np.float64).tofile(xf)
        r = _run([os.path.join(DRIVERS, "GPU-ED"), str(qf), str(xf), str(q.size), str(x.size)])
        assert r.returncode == 0, r.stderr
        loc = int(re.search(r"location: (\d+)", r.stdout).group(1))
        dist = float(re.search(r"distance: ([0-9.eE+-]+)", r.stdout).group(1))
        assert loc == c["ucr_location"] and abs(dist - c["ucr_distance"]) <= 1e-5 * dist


def test_gpu_ldtw_driver_matches_oracle(tmp_path):
    x = synth.ecg_like(30000, seed=77)
    q, _ = synth.cut_query(x, 128, seed=77, noise=0.05)
    qf, xf = tmp_path / "q.bin", tmp_path / "s.bin"
    q.tofile(qf)
    x.tofile(xf)
    r = _run([os.path.join(DRIVERS, "GPU-LDTW"), str(qf), str(xf), "128", str(x.size), "10"])
    assert r.returncode == 0, r.stderr
    m = re.search(r"best alignment found at index (\d+) with distance ([0-9.eE+-]+)", r.stdout)
    i, v = oracle.argmin(oracle.ldtw_all(q, x, 12))
    assert int(m.group(1)) == i and abs(float(m.group(2)) - np.sqrt(v)) <= 1e-5 * np.sqrt(v)


def test_drivers_reject_short_files(tmp_path):
    q = np.zeros(64, np.float32)
    qf, xf = tmp_path / "q.bin", tmp_path / "s.bin"
    q.tofile(qf)
    np.zeros(100, np.float32).tofile(xf)
    r = _run([os.path.join(DRIVERS, "GPU-DTW"), str(qf), str(xf), "64", "1000", "10"])
    assert r.returncode == 1 and "could not read" in r.stderr
