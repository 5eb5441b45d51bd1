"""Host-side mirror of the reference's search interface over the C ABI.

The reference exposes header templates taking device pointers
(avg_std<prefx_t>(Series, AvgS, StdS, M, N, stream), include/stats.cuh:115;
gpu_cdtw<euclidean>(Subject, AvgS, StdS, Cdtw, M, Indices, L, W, ...),
include/cdtw.cuh:450; prune_cdtw<euclidean>(Subject, AvgS, StdS, M, N, W),
cdtw.cuh:510) with the query in __constant__ memory.  ``Handle`` keeps the
same names and argument meaning with torch CUDA tensors as device buffers and
the query as per-handle state.  Errors raise ``CudaDTWError`` carrying the C
status; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import CudaDTWError, load

EUCLIDEAN, MANHATTAN = 0, 1
HOST, DEVICE = 0, 1


def _metric(m) -> int:
    """0 / "euclidean" -> squared cost, 1 / "manhattan" -> absolute cost."""
    if isinstance(m, str):
        m = {"euclidean": EUCLIDEAN, "manhattan": MANHATTAN}.get(m.lower(), -1)
    if isinstance(m, bool) or m not in (EUCLIDEAN, MANHATTAN):
        raise ValueError(f"unknown metric {m!r}")
    return int(m)


def band_from_percent(m: int, p: int) -> int:
    """W = M*(P*0.01) truncated (GPU-dtw.cu:27)."""
    return load().cdtw_band_from_percent(m, p)


def _ptr(t) -> ctypes.c_void_p:
    if t is None:
        return ctypes.c_void_p(0)
    if isinstance(t, np.ndarray):
        return ctypes.c_void_p(t.ctypes.data)
    return ctypes.c_void_p(t.data_ptr())


def _dev(t: torch.Tensor, dtype: torch.dtype, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype or not t.is_contiguous():
        raise TypeError(f"{name} must be a contiguous {dtype} tensor")
    return t


class Handle:
    """One cudadtw handle: device, stream, query state and work buffers."""

    def __init__(self, device: int = 0):
        self._lib = load()
        h = ctypes.c_void_p()
        st = self._lib.cdtw_create(ctypes.byref(h), device)
        if st != 0:
            raise CudaDTWError(st, f"cdtw_create(device={device}) failed: "
                                   f"{self._lib.cdtw_status_string(st).decode()}")
        self._h = h
        self.device = device
        self.M = None
        self.W = None
        # Work on torch's current stream so torch-made inputs are ordered
        # before the kernels and torch consumers after them.
        self.use_torch_stream()

    # -- plumbing ----------------------------------------------------------
    def _check(self, st: int) -> None:
        if st != 0:
            raise CudaDTWError(st, self._lib.cdtw_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.cdtw_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def use_torch_stream(self, stream: torch.cuda.Stream | None = None) -> None:
        """Run on a torch stream (default: torch's current stream)."""
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        self._check(self._lib.cdtw_set_stream(self._h, ctypes.c_void_p(s.cuda_stream)))

    # -- reference-named operations -----------------------------------------
    def avg_std(self, series: torch.Tensor, M: int):
        """Windowed mean (FP64) and std (FP32) of every length-M window
        (avg_std, include/stats.cuh:115-142)."""
        _dev(series, torch.float32, "series")
        nw = series.numel() - M + 1
        avg = torch.empty(max(nw, 0), dtype=torch.float64, device=series.device)
        std = torch.empty(max(nw, 0), dtype=torch.float32, device=series.device)
        self._check(self._lib.cdtw_avg_std(self._h, _ptr(series), series.numel(), M, _ptr(avg),
                                           _ptr(std)))
        return avg, std

    def set_query(self, query, W: int) -> None:
        """z-normalise the query and build its envelope (znormalize + envelope +
        cudaMemcpyToSymbol of GPU-dtw.cu:67-68, :82-84)."""
        if isinstance(query, torch.Tensor) and query.is_cuda:
            keep, loc, n = _dev(query, torch.float32, "query"), DEVICE, query.numel()
        else:
            keep = np.ascontiguousarray(np.asarray(query, dtype=np.float32))
            loc, n = HOST, keep.size
        self._check(self._lib.cdtw_set_query(self._h, _ptr(keep), n, W, loc))
        self.M = n
        self.W = min(W, self.M - 1)

    def gpu_cdtw(self, subject: torch.Tensor, avg: torch.Tensor, std: torch.Tensor,
                 indices: torch.Tensor | None = None, metric=EUCLIDEAN,
                 out: torch.Tensor | None = None) -> torch.Tensor:
        """cDTW of the query against listed windows, all windows if ``indices``
        is None (gpu_cdtw, include/cdtw.cuh:450-487).  Squared distances for
        the Euclidean cost, as the reference's Cdtw array."""
        _dev(subject, torch.float32, "subject")
        _dev(avg, torch.float64, "avg")
        _dev(std, torch.float32, "std")
        if indices is not None:
            _dev(indices, torch.int32, "indices")
            n = indices.numel()
        else:
            n = subject.numel() - self.M + 1
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device=subject.device)
        self._check(self._lib.cdtw_gpu_cdtw(self._h, _ptr(subject), subject.numel(), _ptr(avg),
                                            _ptr(std), _ptr(indices), n, _metric(metric),
                                            _ptr(out)))
        return out

    def all_windows_host(self, query: np.ndarray, subject: np.ndarray, W: int,
                         metric=EUCLIDEAN, out: np.ndarray | None = None) -> np.ndarray:
        """Unpruned all-windows cDTW from host arrays (copies inside the call)."""
        q = np.ascontiguousarray(query, dtype=np.float32)
        s = subject if (isinstance(subject, np.ndarray) and subject.dtype == np.float32
                        and subject.flags.c_contiguous) else np.ascontiguousarray(subject, np.float32)
        nw = s.size - q.size + 1
        if out is None:
            out = np.empty(nw, np.float32)
        self._check(self._lib.cdtw_all_windows_host(self._h, _ptr(q), q.size, _ptr(s), s.size, W,
                                                    _metric(metric), _ptr(out)))
        return out

    # -- lower bounds and search ---------------------------------------------
    def lb_kim(self, subject, avg, std, indices=None, metric=EUCLIDEAN):
        """LB_Kim (5x5 front/back, include/bounds.cuh:413-441) per window."""
        n = indices.numel() if indices is not None else subject.numel() - self.M + 1
        out = torch.empty(n, dtype=torch.float32, device=subject.device)
        self._check(self._lib.cdtw_lb_kim(self._h, _ptr(subject), subject.numel(), _ptr(avg),
                                          _ptr(std), _ptr(indices), n, _metric(metric),
                                          _ptr(out)))
        return out

    def lb_keogh(self, subject, avg, std, indices=None, metric=EUCLIDEAN, reverse=True):
        """(forward LB_Keogh, reverse LB_Keogh) per window (bounds.cuh:443-465;
        UCR_DTW_BIN.cpp:262-282)."""
        n = indices.numel() if indices is not None else subject.numel() - self.M + 1
        fwd = torch.empty(n, dtype=torch.float32, device=subject.device)
        rev = torch.empty(n, dtype=torch.float32, device=subject.device) if reverse else None
        self._check(self._lib.cdtw_lb_keogh(self._h, _ptr(subject), subject.numel(), _ptr(avg),
                                            _ptr(std), _ptr(indices), n, _metric(metric),
                                            _ptr(fwd), _ptr(rev)))
        return fwd, rev

    def prune_cdtw(self, subject, avg, std, metric=EUCLIDEAN):
        """Best match (location, distance) of the query (prune_cdtw,
        include/cdtw.cuh:510-592); distance as the reference prints it."""
        loc = ctypes.c_int64()
        dist = ctypes.c_float()
        self._check(self._lib.cdtw_prune_cdtw(self._h, _ptr(subject), subject.numel(), _ptr(avg),
                                              _ptr(std), _metric(metric), ctypes.byref(loc),
                                              ctypes.byref(dist)))
        return loc.value, dist.value

    def search_host(self, query, subject, W, metric=EUCLIDEAN):
        """The whole GPU-DTW search from host arrays (GPU-dtw.cu:59-90)."""
        q = np.ascontiguousarray(query, dtype=np.float32)
        s = subject if (isinstance(subject, np.ndarray) and subject.dtype == np.float32
                        and subject.flags.c_contiguous) else np.ascontiguousarray(subject, np.float32)
        loc = ctypes.c_int64()
        dist = ctypes.c_float()
        self._check(self._lib.cdtw_search_host(self._h, _ptr(q), q.size, _ptr(s), s.size, W,
                                               _metric(metric), ctypes.byref(loc),
                                               ctypes.byref(dist)))
        self.M, self.W = q.size, min(W, q.size - 1)
        return loc.value, dist.value

    def topk(self, subject, avg, std, k: int, metric=EUCLIDEAN):
        """The k best non-overlapping windows of the query: (locations,
        distances) best first, distances as the search prints them."""
        locs = np.empty(k, np.int64)
        dists = np.empty(k, np.float32)
        found = ctypes.c_int()
        self._check(self._lib.cdtw_topk(self._h, _ptr(subject), subject.numel(), _ptr(avg),
                                        _ptr(std), _metric(metric), int(k), _ptr(locs),
                                        _ptr(dists), ctypes.byref(found)))
        return locs[:found.value], dists[:found.value]

    def topk_device(self, subject, avg, std, k: int, metric=EUCLIDEAN):
        """topk with every step on the device (cdtw_topk_device): the same
        picks, no host round trip before the end."""
        locs = np.empty(k, np.int64)
        dists = np.empty(k, np.float32)
        found = ctypes.c_int()
        self._check(self._lib.cdtw_topk_device(self._h, _ptr(subject), subject.numel(),
                                               _ptr(avg), _ptr(std), _metric(metric), int(k),
                                               _ptr(locs), _ptr(dists), ctypes.byref(found)))
        return locs[:found.value], dists[:found.value]

    # -- search over a stream pushed in pieces ------------------------------
    def stream_begin(self, query, W: int, metric=EUCLIDEAN, chunk: int = 0) -> None:
        """Start a search whose subject arrives by stream_push (chunked copies
        overlapping the search of the previous chunk; UCR's EPOCH loop)."""
        q = np.ascontiguousarray(query, dtype=np.float32)
        self._check(self._lib.cdtw_stream_begin(self._h, _ptr(q), q.size, W, _metric(metric),
                                                int(chunk)))
        self.M, self.W = q.size, min(W, q.size - 1)

    def stream_push(self, samples) -> None:
        s = np.ascontiguousarray(samples, dtype=np.float32)
        self._check(self._lib.cdtw_stream_push(self._h, _ptr(s), s.size))

    def stream_end(self):
        """(location, distance, samples scanned) of the whole stream."""
        loc, dist, n = ctypes.c_int64(), ctypes.c_float(), ctypes.c_int64()
        self._check(self._lib.cdtw_stream_end(self._h, ctypes.byref(loc), ctypes.byref(dist),
                                              ctypes.byref(n)))
        return loc.value, dist.value, n.value

    def set_memory_limit(self, nbytes: int) -> None:
        """Cap the device memory the handle holds (0: no cap); calls that
        would need more raise CudaDTWError with status CDTW_ENOMEM (2)."""
        self._check(self._lib.cdtw_set_memory_limit(self._h, int(nbytes)))

    def search_flag(self) -> int:
        """The reference's termination flag of the last search (the line
        GPU-DTW prints after "Distance:"): best distance < largest LB_Kim."""
        f = ctypes.c_int()
        self._check(self._lib.cdtw_search_flag(self._h, ctypes.byref(f)))
        return f.value

    def search_counts(self):
        """(windows, below bsf after LB_Kim, reaching cDTW) of the last search."""
        c = (ctypes.c_int64 * 3)()
        self._check(self._lib.cdtw_search_counts(self._h, c))
        return tuple(c)

    # -- GPU-ED and GPU-LDTW ----------------------------------------------------
    def ed_all_windows(self, query64, subject64):
        """Squared z-normalised Euclidean distance per window, FP64
        (calculate_ed, include/ed.cuh:71-153)."""
        _dev(query64, torch.float64, "query")
        _dev(subject64, torch.float64, "subject")
        out = torch.empty(subject64.numel() - query64.numel() + 1, dtype=torch.float64,
                          device=subject64.device)
        self._check(self._lib.ed_all_windows(self._h, _ptr(query64), query64.numel(),
                                             _ptr(subject64), subject64.numel(), _ptr(out)))
        return out

    def ed_search_host(self, query, subject):
        q = np.ascontiguousarray(query, dtype=np.float64)
        s = np.ascontiguousarray(subject, dtype=np.float64)
        loc, dist = ctypes.c_int64(), ctypes.c_double()
        self._check(self._lib.ed_search_host(self._h, _ptr(q), q.size, _ptr(s), s.size,
                                             ctypes.byref(loc), ctypes.byref(dist)))
        return loc.value, dist.value

    def ldtw_all_windows(self, subject, metric=EUCLIDEAN):
        """Greedy LDTW path cost of the query vs every window, FP64
        (ztsh2_ldtw, include/ldtw.cuh:294-391)."""
        _dev(subject, torch.float32, "subject")
        out = torch.empty(subject.numel() - self.M + 1, dtype=torch.float64, device=subject.device)
        self._check(self._lib.ldtw_all_windows(self._h, _ptr(subject), subject.numel(),
                                               _metric(metric), _ptr(out)))
        return out

    def ldtw_search_host(self, query, subject, W, metric=EUCLIDEAN):
        q = np.ascontiguousarray(query, dtype=np.float32)
        s = np.ascontiguousarray(subject, dtype=np.float32)
        loc, dist = ctypes.c_int64(), ctypes.c_double()
        self._check(self._lib.ldtw_search_host(self._h, _ptr(q), q.size, _ptr(s), s.size, W,
                                               _metric(metric), ctypes.byref(loc),
                                               ctypes.byref(dist)))
        self.M, self.W = q.size, min(W, q.size - 1)
        return loc.value, dist.value

    def ldtw_ref_all_windows(self, subject, metric=EUCLIDEAN, znorm: bool = True):
        """Greedy LDTW path cost per window in the reference's own FP32
        arithmetic (ztsh2_ldtw, or tsh2_ldtw with znorm=False), float32."""
        _dev(subject, torch.float32, "subject")
        out = torch.empty(subject.numel() - self.M + 1, dtype=torch.float32, device=subject.device)
        self._check(self._lib.ldtw_ref_all_windows(self._h, _ptr(subject), subject.numel(),
                                                   _metric(metric), int(bool(znorm)), _ptr(out)))
        return out

    def ldtw_ref_search_host(self, query, subject, W, metric=EUCLIDEAN, znorm: bool = True):
        """GPU-LDTW as the reference computes it (FP32): (location, distance)."""
        q = np.ascontiguousarray(query, dtype=np.float32)
        s = np.ascontiguousarray(subject, dtype=np.float32)
        loc, dist = ctypes.c_int64(), ctypes.c_float()
        self._check(self._lib.ldtw_ref_search_host(self._h, _ptr(q), q.size, _ptr(s), s.size, W,
                                                   _metric(metric), int(bool(znorm)),
                                                   ctypes.byref(loc), ctypes.byref(dist)))
        self.M, self.W = q.size, min(W, q.size - 1)
        return loc.value, dist.value

    # -- kernel selection -----------------------------------------------------
    VARIANTS = {"auto": 0, "register": 1, "strip16": 2, "strip32": 3, "lane": 4}

    def set_band_variant(self, w_lo: int, w_hi: int, variant) -> None:
        """cDTW kernel variant for bands w_lo..w_hi (the autotuner's knob)."""
        v = self.VARIANTS[variant] if isinstance(variant, str) else int(variant)
        self._check(self._lib.cdtw_set_band_variant(self._h, w_lo, w_hi, v))

    # -- batched search ---------------------------------------------------------
    def search_batched(self, subject: torch.Tensor, queries, bands, metric=EUCLIDEAN,
                       rows=None, tiles=None):
        """Best match (locations, distances) of every query in one graph
        launch.  ``queries``: list of 1-D arrays, ``bands``: W per query.
        Without ``rows`` / ``tiles``: concurrent single-query pipelines
        (results bit-identical to prune_cdtw); with them (the autotuner fills
        them per bucket): the persistent (query, stream-tile) kernels."""
        _dev(subject, torch.float32, "subject")
        qs = [np.ascontiguousarray(q, dtype=np.float32) for q in queries]
        nq = len(qs)
        flat = np.concatenate(qs) if nq else np.zeros(0, np.float32)
        ms = np.array([q.size for q in qs], dtype=np.int32)
        ws = np.ascontiguousarray(bands, dtype=np.int32)
        r = None if rows is None else np.ascontiguousarray(rows, dtype=np.int32)
        t = None if tiles is None else np.ascontiguousarray(tiles, dtype=np.int32)
        locs = np.empty(nq, np.int64)
        dists = np.empty(nq, np.float32)
        self._check(self._lib.cdtw_search_batched(
            self._h, _ptr(subject), subject.numel(), _ptr(flat), _ptr(ms), _ptr(ws), nq,
            _metric(metric), _ptr(r), _ptr(t), _ptr(locs), _ptr(dists)))
        return locs, dists

    # -- differentiable pairwise cDTW -------------------------------------------
    PAIR_ZNORM = 1

    def pair_path_bytes(self, n: int, L: int) -> int:
        """Bytes of the path record cdtw_pair_fwd writes for n pairs of length L."""
        return int(self._lib.cdtw_pair_path_bytes(n, L))

    PAIR_MODES = {None: 0, "auto": 0, "store": 2, "recompute": 4}

    def pair_workspace_bytes(self, n: int, L: int, W: int, znorm: bool = True,
                             with_path: bool = True, mode=None) -> int:
        """Device work memory pair_fwd takes from the handle's workspace."""
        flags = (self.PAIR_ZNORM if znorm else 0) | self.PAIR_MODES[mode]
        return int(self._lib.cdtw_pair_workspace_bytes(n, L, W, flags, int(with_path)))

    def pair_last_mode(self) -> str:
        """"recompute" or "store": how the last pair_fwd with a path recorded it."""
        r = ctypes.c_int()
        self._check(self._lib.cdtw_pair_last_mode(self._h, ctypes.byref(r)))
        return "recompute" if r.value else "store"

    def pair_fwd(self, q: torch.Tensor, s: torch.Tensor, W: int, metric=EUCLIDEAN,
                 znorm: bool = True, path: torch.Tensor | None = None,
                 out: torch.Tensor | None = None, mode=None) -> torch.Tensor:
        """Banded cDTW of every pair (q[p], s[p]) (device (n, L) float32).  With
        ``path`` (a uint8 device buffer of pair_path_bytes) the optimal path is
        recorded for pair_bwd; ``mode`` "store" (2-bit directions) or
        "recompute" (checkpoints, segments recomputed during the walk), None
        for the library's choice by memory."""
        _dev(q, torch.float32, "q")
        _dev(s, torch.float32, "s")
        if q.shape != s.shape or q.dim() != 2:
            raise ValueError("q and s must both be (n, L)")
        n, L = q.shape
        D = out if out is not None else torch.empty(n, dtype=torch.float32, device=q.device)
        flags = (self.PAIR_ZNORM if znorm else 0) | self.PAIR_MODES[mode]
        self._check(self._lib.cdtw_pair_fwd(self._h, _ptr(q), _ptr(s), n, L, int(W),
                                            _metric(metric), flags, _ptr(D), _ptr(path)))
        return D

    def pair_bwd(self, q: torch.Tensor, s: torch.Tensor, path: torch.Tensor, dD=None,
                 metric=EUCLIDEAN, znorm: bool = True, need_q: bool = True,
                 need_s: bool = True, dq: torch.Tensor | None = None,
                 ds: torch.Tensor | None = None):
        """Gradients (dq, ds) of sum_p dD[p] * D[p] along the recorded paths."""
        n, L = q.shape
        if need_q and dq is None:
            dq = torch.empty_like(q)
        if need_s and ds is None:
            ds = torch.empty_like(s)
        self._check(self._lib.cdtw_pair_bwd(
            self._h, _ptr(q), _ptr(s), n, L, _metric(metric), self.PAIR_ZNORM if znorm else 0,
            _ptr(path), _ptr(dD), _ptr(dq if need_q else None), _ptr(ds if need_s else None)))
        return (dq if need_q else None), (ds if need_s else None)

    # -- template refinement ----------------------------------------------------
    def refine_templates(self, subject: torch.Tensor, templates, bands, locations, steps: int,
                         lr: float = 1e-2, metric=EUCLIDEAN):
        """Adam refinement of templates against their matched windows
        (cdtw_refine_templates).  ``templates``: list of 1-D arrays; ``bands``:
        W per template; ``locations``: (nt, k) window starts.  Returns the
        refined templates (list of float32 arrays) and the (steps+1, nt) losses."""
        _dev(subject, torch.float32, "subject")
        ts = [np.ascontiguousarray(t, dtype=np.float32) for t in templates]
        nt = len(ts)
        flat = torch.from_numpy(np.concatenate(ts)).to(subject.device)
        ms = np.array([t.size for t in ts], dtype=np.int32)
        ws = np.ascontiguousarray(bands, dtype=np.int32)
        loc = np.ascontiguousarray(locations, dtype=np.int64)
        if loc.ndim != 2 or loc.shape[0] != nt:
            raise ValueError("locations must be (n_templates, k)")
        losses = np.empty((steps + 1, nt), np.float32)
        self._check(self._lib.cdtw_refine_templates(
            self._h, _ptr(subject), subject.numel(), _ptr(flat), _ptr(ms), _ptr(ws), nt,
            _ptr(loc), loc.shape[1], int(steps), float(lr), _metric(metric), _ptr(losses)))
        out = flat.cpu().numpy()
        res, o = [], 0
        for m in ms:
            res.append(out[o:o + m].copy())
            o += m
        return res, losses

    def refine_templates_search(self, subject: torch.Tensor, templates, bands, k: int,
                                steps: int, lr: float = 1e-2, metric=EUCLIDEAN):
        """Adam refinement with the top-k matches searched again at every step
        (cdtw_refine_templates_search, one CUDA graph).  Returns the refined
        templates, the (steps+1, nt) mean distances to each step's matches,
        and the (nt, k) matches of the last step."""
        _dev(subject, torch.float32, "subject")
        ts = [np.ascontiguousarray(t, dtype=np.float32) for t in templates]
        nt = len(ts)
        flat = torch.from_numpy(np.concatenate(ts)).to(subject.device)
        ms = np.array([t.size for t in ts], dtype=np.int32)
        ws = np.ascontiguousarray(bands, dtype=np.int32)
        losses = np.empty((steps + 1, nt), np.float32)
        locs = np.empty((nt, k), np.int64)
        self._check(self._lib.cdtw_refine_templates_search(
            self._h, _ptr(subject), subject.numel(), _ptr(flat), _ptr(ms), _ptr(ws), nt, int(k),
            int(steps), float(lr), _metric(metric), _ptr(losses), _ptr(locs)))
        out = flat.cpu().numpy()
        res, o = [], 0
        for m in ms:
            res.append(out[o:o + m].copy())
            o += m
        return res, losses, locs
