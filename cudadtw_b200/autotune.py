"""Autotuner of the kernel shapes, per (query length, band) bucket.

Two knobs of the library depend on the bucket and on the GPU:

* the batched search's main pass (``cdtw_search_batched``): ``rows`` (0 = the
  register-band kernel, W <= 96; 1/2/4/8/16 = strips of that many rows,
  W >= rows-1) and ``tiles`` (windows per work item);
* the plain search's cDTW variant per band (``cdtw_set_band_variant``):
  register band, 16-row or 32-row strips.

``tune_batched`` times every candidate on a sample of the bucket's queries and
keeps the fastest; ``tune_variants`` does the same for the all-windows cDTW of
one query per band.  Results are cached as JSON keyed by the device name
(``$CUDADTW_AUTOTUNE_CACHE``, default ``~/.cache/cudadtw_b200/autotune.json``),
so a process reuses them with ``load`` + ``shapes_for`` / ``apply_variants``.
Timing goes through an injectable ``measure`` callable (the default ones time
the library on the GPU), which keeps the selection logic testable without one.
"""
from __future__ import annotations

import json
import os
import time
from typing import Callable, Iterable

import numpy as np

MAX_REGISTER_BAND = 96
STRIP_ROWS = (1, 2, 4, 8, 16)
TILE_CHOICES = (512, 1024, 2048)
DEFAULT_ROWS_TILES = None  # the library's built-in rule when a bucket is untuned


def cache_path() -> str:
    return os.environ.get("CUDADTW_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "cudadtw_b200",
                                       "autotune.json"))


def bucket(M: int, W: int) -> str:
    """Bucket key: the query length rounded up to a power of two (>= 64) and the
    band rounded up to a multiple of 8 (register-band kernels are per W, strips
    depend on W only through the strip count)."""
    m = 64
    while m < M:
        m *= 2
    w = ((max(W, 0) + 7) // 8) * 8
    return f"M{m}_W{w}"


def batched_candidates(W: int) -> list[tuple[int, int]]:
    """(rows, tiles) pairs the batched search accepts for band W."""
    rows = ([0] if W <= MAX_REGISTER_BAND else []) + [r for r in STRIP_ROWS if W >= r - 1]
    return [(r, t) for r in rows for t in TILE_CHOICES]


def variant_candidates(W: int) -> list[str]:
    """Plain-search cDTW variants that can run band W."""
    out = []
    if W <= MAX_REGISTER_BAND:
        out.append("register")
    if W >= 15:
        out.append("strip16")
    if W >= 31:
        out.append("strip32")
    if lane_shape(W) is not None:
        out.append("lane")
    return out


def lane_shape(W: int):
    """(lanes per window group, cells per lane) of the lane-group kernels for
    band W, or None when they cannot run it: the rule of lane_shape in
    csrc/cdtw_lane.cu (G in {4, 8, 16, 32}, 18 <= B <= 48, G*B >= 2W+1,
    (G-1)*B <= 2W, least 3GB + 10G)."""
    best = None
    for g in (4, 8, 16, 32):
        for b in range(18, 49):
            if g * b < 2 * W + 1 or (g - 1) * b > 2 * W:
                continue
            cost = 3 * g * b + 10 * g
            if best is None or cost < best[0]:
                best = (cost, g, b)
    return None if best is None else best[1:]


def tune_batched(queries: list, bands: Iterable[int],
                 measure: Callable[[list[int], int, int], float],
                 per_bucket: int = 8) -> dict:
    """Best (rows, tiles) per bucket.  ``measure(query_indices, rows, tiles)``
    returns the seconds the batched search of those queries takes with that
    shape; each bucket is timed on up to ``per_bucket`` of its queries."""
    bands = list(bands)
    groups: dict[str, list[int]] = {}
    for i, (q, w) in enumerate(zip(queries, bands)):
        groups.setdefault(bucket(len(q), w), []).append(i)
    table = {}
    for key, idx in sorted(groups.items()):
        sample = idx[:per_bucket]
        wmin = min(bands[i] for i in sample)
        wmax = max(bands[i] for i in sample)
        # candidates valid for every query of the sample
        cands = [c for c in batched_candidates(wmin) if c in batched_candidates(wmax)]
        timed = [(measure(sample, r, t), r, t) for r, t in cands]
        best = min(timed)
        table[key] = {"rows": best[1], "tiles": best[2], "seconds": best[0],
                      "tried": [[r, t, s] for s, r, t in timed]}
    return table


def shapes_for(queries: list, bands: Iterable[int], table: dict):
    """Per-query (rows, tiles) arrays for ``search_batched`` from a tuned table;
    None when no query's bucket is in the table (built-in rule)."""
    bands = list(bands)
    rows = np.zeros(len(bands), np.int32)
    tiles = np.zeros(len(bands), np.int32)
    hit = False
    for i, (q, w) in enumerate(zip(queries, bands)):
        e = table.get(bucket(len(q), w))
        if e is not None and (e["rows"], e["tiles"]) in batched_candidates(w):
            rows[i], tiles[i] = e["rows"], e["tiles"]
            hit = True
        else:  # the built-in rule for this query
            rows[i] = 0 if w <= MAX_REGISTER_BAND else 16
            tiles[i] = 1024
    return (rows, tiles) if hit else (None, None)


def tune_variants(bands: Iterable[int], measure: Callable[[int, str], float]) -> dict:
    """Fastest plain-search variant per band: ``measure(W, variant)`` returns
    seconds for the all-windows cDTW at band W with that variant."""
    out = {}
    for w in sorted(set(bands)):
        timed = [(measure(w, v), v) for v in variant_candidates(w)]
        out[str(w)] = min(timed)[1]
    return out


def apply_variants(handle, variants: dict) -> None:
    """Set the tuned variant of every band on a Handle."""
    for w, v in variants.items():
        handle.set_band_variant(int(w), int(w), v)


# -- persistence ----------------------------------------------------------------

def load(device_name: str, path: str | None = None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            return json.load(f).get(device_name, {})
    except (OSError, ValueError):
        return {}


def save(device_name: str, entry: dict, path: str | None = None) -> None:
    path = path or cache_path()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    try:
        with open(path) as f:
            allv = json.load(f)
    except (OSError, ValueError):
        allv = {}
    allv.setdefault(device_name, {}).update(entry)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(allv, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


# -- GPU measurements ---------------------------------------------------------

def gpu_batched_measure(handle, subject, queries: list, bands: list, metric: int = 0):
    """A ``measure`` for tune_batched that runs the library on the GPU: one
    untimed call (plan + graph build), then one timed replay."""
    import torch

    def measure(idx, rows, tiles):
        qs = [queries[i] for i in idx]
        ws = [bands[i] for i in idx]
        r = [rows] * len(idx)
        t = [tiles] * len(idx)
        handle.search_batched(subject, qs, ws, metric, rows=r, tiles=t)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        handle.search_batched(subject, qs, ws, metric, rows=r, tiles=t)
        torch.cuda.synchronize()
        return time.perf_counter() - t0
    return measure


def gpu_variant_measure(handle, subject, query, metric: int = 0, reps: int = 3):
    """A ``measure`` for tune_variants: all-windows cDTW of ``query`` over
    ``subject`` (torch CUDA tensor) per band and variant, CUDA-event timed."""
    import torch
    avg, std = handle.avg_std(subject, len(query))

    def measure(w, variant):
        handle.set_band_variant(w, w, variant)
        handle.set_query(query, w)
        out = handle.gpu_cdtw(subject, avg, std, metric=metric)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            handle.gpu_cdtw(subject, avg, std, metric=metric, out=out)
        e1.record()
        torch.cuda.synchronize()
        handle.set_band_variant(w, w, "auto")
        return e0.elapsed_time(e1) / 1e3 / reps
    return measure
