"""GPU tests of the search over a stream pushed in pieces (cdtw_stream_begin /
push / end) and of the UCR-DTW / UCR-DTW-BIN drivers built on it.

* Pieces of random sizes, chunks much smaller than the stream (many halos
  and carried bounds): the location equals the whole-stream search's and the
  unpruned argmin's, for both costs, and the distance to float rounding (the
  chunks' FP64 window sums start from other points).
* A planted exact copy of the best window in a later chunk: the earliest
  window wins, as UCR's first strict minimum.
* The 2^25-sample metal-like stream in the default chunks (four of them):
  the same window as the in-memory search.
* The drivers against the reference's UCR_DTW (text) and UCR_DTW_BIN
  (binary), built from the reference sources, on the same files."""
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


def _stream_search(h, q, x, w, metric=0, chunk=0, seed=0):
    h.stream_begin(q, w, metric=metric, chunk=chunk)
    rng = np.random.default_rng(seed)
    at = 0
    while at < x.size:
        n = int(rng.integers(1, 50_000))
        h.stream_push(x[at:at + n])
        at += n
    return h.stream_end()


@pytest.mark.parametrize("m,p,metric", [(128, 10, 0), (300, 20, 1), (700, 15, 0)])
def test_stream_equals_whole_search(handle, m, p, metric):
    x = synth.ecg_like(400_000, seed=m)
    q, _ = synth.cut_query(x, m, seed=p, noise=0.1)
    w = synth.band_from_percent(m, p)
    loc, dist, n = _stream_search(handle, q, x, w, metric, chunk=65_536, seed=m)
    assert n == x.size
    nw, nkim, ndtw = handle.search_counts()  # summed over the chunks
    assert nw == x.size - m + 1 and 0 < ndtw <= nkim <= nw
    # the chunks' window statistics are summed from other starting points
    # than the whole stream's (FP64, equal to a few ulps): equal location,
    # distance equal to float rounding
    hloc, hdist = handle.search_host(q, x, w, metric=metric)
    assert loc == hloc and abs(dist - hdist) <= 1e-5 * hdist
    dx = torch.from_numpy(x).cuda()
    avg, std = handle.avg_std(dx, m)
    handle.set_query(q, w)
    allw = handle.gpu_cdtw(dx, avg, std, metric=metric).cpu().numpy()
    assert loc == int(np.argmin(allw))


def test_stream_tie_keeps_the_earliest_window(handle):
    x = synth.ecg_like(300_000, seed=3)
    q, off = synth.cut_query(x, 128, seed=3, noise=0.0)
    x[250_000:250_128] = x[off:off + 128]  # an exact copy in a later chunk
    loc, dist, _ = _stream_search(handle, q, x, 12, chunk=40_000, seed=1)
    assert loc == min(off, 250_000) and dist < 1e-2


def test_stream_full_size_metal(handle):
    x = synth.metal_like(1 << 25, seed=1)
    q, off = synth.cut_query(x, 256, seed=100 + 256 + 10, noise=0.1)
    w = synth.band_from_percent(256, 10)
    handle.stream_begin(q, w)
    for a in range(0, x.size, 3_000_000):
        handle.stream_push(x[a:a + 3_000_000])
    loc, dist, n = handle.stream_end()
    assert n == x.size
    dx = torch.from_numpy(x).cuda()
    avg, std = handle.avg_std(dx, 256)
    handle.set_query(q, w)
    ploc, pdist = handle.prune_cdtw(dx, avg, std)
    assert loc == ploc and abs(dist - pdist) <= 1e-5 * pdist


def test_stream_from_page_locked_memory(handle):
    """Pushes from page-locked memory are copied straight into the device
    chunk (no staging): same result as pushing the same samples from pageable
    memory, and the caller's buffer may be overwritten as soon as a push
    returns."""
    x = synth.ecg_like(500_000, seed=17)
    q, _ = synth.cut_query(x, 200, seed=4, noise=0.1)
    ref = _stream_search(handle, q, x, 20, chunk=100_000, seed=2)
    buf = torch.empty(37_000, dtype=torch.float32).pin_memory().numpy()
    handle.stream_begin(q, 20, chunk=100_000)
    for a in range(0, x.size, buf.size):
        piece = x[a:a + buf.size]
        buf[:piece.size] = piece
        handle.stream_push(buf[:piece.size])
        buf[:] = np.nan  # reused at once: the push has finished with it
    assert handle.stream_end() == ref


def test_stream_buffers_reused_across_streams(handle):
    """Streams back to back on one handle reuse the buffers of the earlier
    ones (growing them for a larger chunk or query); a stream begun again
    before its end drops the unfinished one.  Every result equals the
    stream's own fresh-handle search, and repeating a stream of the same
    shape takes no device memory."""
    from cudadtw_b200 import Handle
    x = synth.ecg_like(300_000, seed=12)
    cases = [(128, 12, 0, 65_536), (300, 30, 1, 50_000), (128, 12, 0, 65_536),
             (700, 70, 0, 131_072)]
    want = []
    with Handle(0) as fresh:
        for m, w, metric, chunk in cases:
            q, _ = synth.cut_query(x, m, seed=m + w, noise=0.1)
            want.append(_stream_search(fresh, q, x, w, metric, chunk=chunk, seed=m))
    q0, _ = synth.cut_query(x, 128, seed=140, noise=0.1)
    handle.stream_begin(q0, 12, chunk=65_536)
    handle.stream_push(x[:200_000])  # never ended
    free = []
    for (m, w, metric, chunk), ref in zip(cases, want):
        q, _ = synth.cut_query(x, m, seed=m + w, noise=0.1)
        assert _stream_search(handle, q, x, w, metric, chunk=chunk, seed=m) == ref
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    assert free[2] == free[1]


def test_stream_errors(handle):
    from cudadtw_b200 import CudaDTWError
    q = synth.ecg_like(128, seed=1)
    handle.stream_begin(q, 12)
    handle.stream_push(np.zeros(100, np.float32))
    with pytest.raises(CudaDTWError) as e:
        handle.stream_end()  # 100 samples: shorter than the query
    assert e.value.status == 1
    with pytest.raises(CudaDTWError):
        handle.stream_push(np.zeros(10, np.float32))  # no stream begun
    with pytest.raises(CudaDTWError):
        handle.stream_begin(q, 12, chunk=64)  # chunk shorter than the query


def _parse(out):
    loc = int(re.search(r"Location\s*:\s*(\d+)", out).group(1))
    dist = float(re.search(r"Distance\s*:\s*([0-9.eE+-]+)", out).group(1))
    return loc, dist


@pytest.mark.parametrize("kind,m,r_arg", [("ecg", 128, "0.1"), ("metal", 256, "25"),
                                          ("ecg", 200, "0.05")])
def test_ucr_drivers_match_reference_ucr(tmp_path, kind, m, r_arg):
    x = synth.ecg_like(200_000, seed=7) if kind == "ecg" else synth.metal_like(200_000, seed=8)
    q, _ = synth.cut_query(x, m, seed=m, noise=0.1)
    dt, qt = str(tmp_path / "data.txt"), str(tmp_path / "query.txt")
    oracle.write_text(dt, x)
    oracle.write_text(qt, q)
    ref = oracle.ucr_dtw_text(dt, qt, m, r_arg)
    r = subprocess.run([os.path.join(DRIVERS, "UCR-DTW"), dt, qt, str(m), r_arg],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    loc, dist = _parse(r.stdout)
    assert loc == ref[0] and abs(dist - ref[1]) <= 1e-4 * ref[1]
    assert f"Data Scanned : {x.size}" in r.stdout
    db, qb = str(tmp_path / "data.bin"), str(tmp_path / "query.bin")
    x.astype(np.float64).tofile(db)
    q.astype(np.float64).tofile(qb)
    r = subprocess.run([os.path.join(DRIVERS, "UCR-DTW-BIN"), db, qb, str(m), r_arg,
                        str(x.size)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert _parse(r.stdout)[0] == ref[0]
    ub = oracle.ucr_dtw(x, q, r_arg)
    assert ub[0] == ref[0]
