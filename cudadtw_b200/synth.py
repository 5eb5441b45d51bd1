"""Seeded synthetic streams and queries for the subsequence cDTW search.

The reference's benchmarks ran on ECG and metal recordings that are not
available (data/.MISSING_LARGE_BLOBS); these generators stand in for them with
signals of the same shape and value range.  Every generator works in FP64 and
rounds once to float32; ``widen`` gives the exact FP64 twin that the UCR Suite
binaries read, so both tools see identical numbers (the reference's own
data/metal/extract.py:40-54 writes single_* and double_* twins the same way).
"""
from __future__ import annotations

import numpy as np


def ecg_like(n: int, seed: int = 0) -> np.ndarray:
    """ECG-like stream: a train of Gaussian pulses (amplitude 1.0+-0.1, width
    8+-2 samples) with period 250+-15 samples (uniform jitter), on a random-walk
    baseline wander (increment std 0.005), plus i.i.d. N(0, 0.05) noise."""
    rng = np.random.default_rng(seed)
    t_last = n + 64
    gaps = rng.uniform(235.0, 265.0, size=int(t_last / 235.0) + 2)
    centers = rng.uniform(0.0, 250.0) + np.concatenate([[0.0], np.cumsum(gaps)])
    centers = centers[centers < t_last]
    amp = rng.uniform(0.9, 1.1, size=centers.size)
    width = rng.uniform(6.0, 10.0, size=centers.size)
    x = np.zeros(n, dtype=np.float64)
    offs = np.arange(-48, 49, dtype=np.int64)
    base = np.floor(centers).astype(np.int64)
    pos = base[:, None] + offs[None, :]
    val = amp[:, None] * np.exp(-0.5 * ((pos - centers[:, None]) / width[:, None]) ** 2)
    ok = (pos >= 0) & (pos < n)
    np.add.at(x, pos[ok], val[ok])
    x += np.cumsum(rng.normal(0.0, 0.005, size=n))
    x += rng.normal(0.0, 0.05, size=n)
    return x.astype(np.float32)


def metal_like(n: int, seed: int = 1) -> np.ndarray:
    """Metal-like stream: cumulative sum of N(0,1) increments with a level
    shift of N(0,20) inserted every 1e5+-2e4 samples.  Magnitudes reach the
    thousands, the regime where a single-precision variance fails."""
    rng = np.random.default_rng(seed)
    inc = rng.normal(0.0, 1.0, size=n)
    p = 0
    while True:
        p += int(rng.integers(80_000, 120_001))
        if p >= n:
            break
        inc[p] += rng.normal(0.0, 20.0)
    return np.cumsum(inc).astype(np.float32)


def random_walk(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.normal(0.0, 1.0, size=n)).astype(np.float32)


def cut_query(stream: np.ndarray, m: int, seed: int, noise: float) -> tuple[np.ndarray, int]:
    """A length-m query cut from ``stream`` at a seeded offset, plus N(0, noise)."""
    rng = np.random.default_rng(seed)
    off = int(rng.integers(0, stream.size - m + 1))
    q = stream[off:off + m].astype(np.float64) + rng.normal(0.0, noise, size=m)
    return q.astype(np.float32), off


def band_from_percent(m: int, p: int) -> int:
    """W = M*(P*0.01) truncated, the reference driver's formula (GPU-dtw.cu:27)."""
    return int(m * (p * 0.01))


def widen(x: np.ndarray) -> np.ndarray:
    """Exact FP64 twin of a float32 array (for the FP64 UCR Suite tools)."""
    return x.astype(np.float64)


def batch_queries(stream: np.ndarray, n: int = 512, seed: int = 2, m_lo: int = 64,
                  m_hi: int = 1024, pcts=(5, 10, 20), noise: float = 0.05):
    """The batched-search workload: n queries with lengths uniform in
    [m_lo, m_hi] and band ratios drawn from ``pcts``; the first half cut from
    ``stream`` at seeded offsets (+ N(0, noise)), the second half independent
    random walks.  Returns a list of (query float32, W, P, cut offset or -1)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        m = int(rng.integers(m_lo, m_hi + 1))
        p = int(pcts[int(rng.integers(0, len(pcts)))])
        w = band_from_percent(m, p)
        if k < n // 2:
            q, off = cut_query(stream, m, seed=int(rng.integers(1 << 30)), noise=noise)
        else:
            q, off = random_walk(m, seed=int(rng.integers(1 << 30))), -1
        out.append((q, w, p, off))
    return out
