#!/usr/bin/env python
"""Benchmark of the cDTW hot path on B200 (one JSON line on rank 0).

Workload (one "step"): the unpruned raw all-windows cDTW of the full-scale
metal-like configuration -- a 2^22-sample metal-like float32 stream (cumulative
N(0,1) increments plus N(0,20) level shifts every 1e5+-2e4 samples), a
length-128 query cut at a seeded offset with N(0,0.1) noise, band ratios 10%
and 20% (W = 12 and 25 by the reference's W = (int)(M*P*0.01)).  A step runs
the windowed statistics once and the cDTW of every window for both bands.
Metric: cell updates per second (GCUPS), cells(M,W) = M(2W+1) - W(W+1) per
window, N-M+1 windows; stream samples/s is reported beside it.

Timing: W warm-up steps, then K steps each bracketed by CUDA events on the
launching stream, with a 256 MiB write between steps to flush the 126 MB L2
(not timed); the whole timed region is bracketed by a barrier and
torch.cuda.synchronize(); the job time is the max over ranks.  Weak scaling:
each rank searches its own stream, no data-path collective.

`--impl reference` times the reference's own CPU all-windows cDTW
(openmp_cdtw, include/cdtw.cuh:91-157, restated in FP32 in the oracle because
the header does not compile outside nvcc with its vendored CUB) on all host
threads, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_STREAM = 1 << 22
M_QUERY = 128
BAND_PCT = (10, 20)
L2_FLUSH_BYTES = 256 << 20
# config-1 (M, P) cases timed with UCR_DTW_BIN beside the GPU search (the
# others take minutes of UCR on every host core)
UCR_CONFIG1 = {(128, 5), (128, 10), (128, 20), (256, 5), (256, 10), (256, 20), (512, 5),
               (512, 10), (1024, 5)}


def cells(m: int, w: int) -> int:
    w = min(w, m - 1)
    return m * (2 * w + 1) - w * (w + 1)


def workload(rank: int):
    from cudadtw_b200 import synth
    x = synth.metal_like(N_STREAM, seed=1 + rank)
    q, off = synth.cut_query(x, M_QUERY, seed=1000 + rank, noise=0.1)
    bands = [synth.band_from_percent(M_QUERY, p) for p in BAND_PCT]
    return x, q, off, bands


def config(bands, world: int, sample=None) -> dict:
    c = {"workload": "raw all-windows cDTW, metal-like stream (config 1 raw part)",
         "stream_samples": N_STREAM, "query_len": M_QUERY, "band_pct": list(BAND_PCT),
         "bands_W": bands, "windows_per_band": N_STREAM - M_QUERY + 1,
         "metric_cost": "squared euclidean", "parallelism": f"stream-per-rank x{world}",
         "l2": "256 MiB write between timed steps (flush)"}
    if sample:
        c["sample"] = sample
    return c


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.proc = None
        self.path = f"/tmp/cdtw_clocks_{os.getpid()}.csv"
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                   "-lms", "200"]
            if gpu_id:
                cmd += ["-i", gpu_id]
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [v.strip() for v in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def cpu_port_gcups(x, q, bands, seconds: float, seed: int = 0):
    """The reference CPU all-windows cDTW (FP32, OpenMP, all host threads) on a
    random sample of windows sized for about `seconds` of work."""
    import oracle
    zq = oracle.znorm(q).astype(np.float32)
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    # stats only for the sampled windows' neighbourhood: compute on a prefix
    span = min(x.size, 1 << 20)
    xs = np.ascontiguousarray(x[:span])
    mu, sd = oracle.window_stats(xs, q.size)
    mu32, sd32 = mu.astype(np.float32), sd.astype(np.float32)
    nw = span - q.size + 1
    # calibrate with a small sample, then size the real one
    probe = rng.integers(0, nw, size=2000, dtype=np.int64)
    t0 = time.perf_counter()
    for w in bands:
        oracle.cdtw_ref_f32(zq, xs, mu32, sd32, probe, w, threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    n = int(min(nw, max(2000, 2000 * seconds / dt)))
    idx = rng.integers(0, nw, size=n, dtype=np.int64)
    t0 = time.perf_counter()
    for w in bands:
        oracle.cdtw_ref_f32(zq, xs, mu32, sd32, idx, w, threads)
    dt = time.perf_counter() - t0
    tot_cells = sum(n * cells(q.size, w) for w in bands)
    return tot_cells / dt / 1e9, threads, n, dt


def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    x, q, _, bands = workload(0)
    per_step_s = max(2.0, 30.0 / max(1, args.steps + args.warmup))
    vals, info = [], None
    for s in range(args.warmup + args.steps):
        g, thr, n, dt = cpu_port_gcups(x, q, bands, per_step_s, seed=s)
        if s >= args.warmup:
            vals.append(g)
            info = (thr, n, dt)
    v = float(np.median(vals))
    thr, n, dt = info
    sample = f"{n} random windows per band of the 2^22-sample stream (first 2^20 samples), per step"
    line = {"impl": "reference", "metric": "GCUPS & stream samples/s", "value": v,
            "unit": "GCUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config(bands, world, sample),
            "stream_samples_per_s": v * 1e9 * len(bands) / sum(cells(M_QUERY, w) for w in bands),
            "cpu_baseline": {"value": v, "unit": "GCUPS", "cores": thr, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local_rank: int) -> None:
    import torch
    import torch.distributed as dist
    from cudadtw_b200 import Handle
    from cudadtw_b200._lib import load

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    x, q, off, bands = workload(rank)
    nw = x.size - q.size + 1
    cells_step = sum(nw * cells(q.size, w) for w in bands)

    h = Handle(local_rank)
    stream = torch.cuda.current_stream(dev)
    dx = torch.from_numpy(x).to(dev)
    dq = torch.from_numpy(q).to(dev)
    outs = [torch.empty(nw, dtype=torch.float32, device=dev) for _ in bands]
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    kev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in bands]

    def step(record_kernels=False):
        avg, std = h.avg_std(dx, q.size)
        for i, w in enumerate(bands):
            h.set_query(dq, w)
            if record_kernels:
                kev[i][0].record(stream)
            h.gpu_cdtw(dx, avg, std, out=outs[i])
            if record_kernels:
                kev[i][1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # peak cell-update rate (issue-bound microkernel) for the roofline
    peak = None if args.only_kernels else ctypes_peak(load(), h)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    smi_id = None
    try:
        smi_id = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    sampler = ClockSampler(smi_id)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    kernel_ms = [[] for _ in bands]
    for s in range(args.steps):
        flush.fill_(s & 0xff)
        ev[s][0].record(stream)
        step(record_kernels=True)
        ev[s][1].record(stream)
        torch.cuda.synchronize()
        for i in range(len(bands)):
            kernel_ms[i].append(kev[i][0].elapsed_time(kev[i][1]))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    t_s = t_ms / 1e3
    if world > 1:
        tt = torch.tensor([t_s], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_s = float(tt.item())
    value = world * cells_step * args.steps / t_s / 1e9

    # parity spot check of this run against the argmin of its own output
    best = [int(torch.argmin(o).item()) for o in outs]

    if args.only_kernels:
        if rank == 0:
            print(json.dumps({"only_kernels": True, "value": value, "unit": "GCUPS",
                              "kernel_ms": kernel_ms, "argmin": best}), flush=True)
        h.close()
        return

    # end to end through the host-buffer C ABI call (copies inside)
    xp = torch.from_numpy(x).pin_memory()
    qp = q.copy()
    hout = [torch.empty(nw, dtype=torch.float32).pin_memory() for _ in bands]
    for i, w in enumerate(bands):  # warm
        h.all_windows_host(qp, xp.numpy(), w, out=hout[i].numpy())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e_steps = max(1, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e_steps):
        for i, w in enumerate(bands):
            h.all_windows_host(qp, xp.numpy(), w, out=hout[i].numpy())
    e_s = time.perf_counter() - t0
    if world > 1:
        tt = torch.tensor([e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e_s = float(tt.item())
    e2e = world * cells_step * e_steps / e_s / 1e9

    kern_s = [float(np.median(k)) / 1e3 for k in kernel_ms]
    achieved = [nw * cells(q.size, w) / ks / 1e9 for w, ks in zip(bands, kern_s)]
    ach = sum(nw * cells(q.size, w) for w in bands) / sum(kern_s) / 1e9

    if rank == 0:
        line = {"metric": "GCUPS & stream samples/s", "value": value, "unit": "GCUPS",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": t_s * 1e3 / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded metal-like stream, FP64 stats / FP32 DTW)",
                "config": config(bands, world),
                "stream_samples_per_s": world * nw * len(bands) * args.steps / t_s,
                "gpu_launches": args.steps * (1 + 2 * len(bands)),
                "clocks": clocks,
                "e2e": {"value": e2e, "unit": "GCUPS",
                        "h2d_bytes_per_step": len(bands) * (x.nbytes + q.nbytes),
                        "d2h_bytes_per_step": len(bands) * nw * 4},
                "roofline": {"bound": "alu",
                             "kernel": "cdtw_regc_kernel<12,EU,4> (W=12) + "
                                       "cdtw_regc_kernel<25,EU,3> (W=25)",
                             "achieved": ach, "peak": peak / 1e9, "unit": "GCUPS",
                             "frac": ach / (peak / 1e9),
                             # DRAM bytes (read + write) of one launch of this workload
                             # from an ncu capture (70.2 / 70.0 MB for W = 12 / 25:
                             # stream, window statistics, results); not measured here
                             "traffic": 70.1e6, "traffic_unit": "bytes per launch",
                             "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write"
                                               ".sum, profiles/cdtw_regc_kernel_raw_allwindows"
                                               "_m128_n4M.md",
                             "per_band": {str(w): a for w, a in zip(bands, achieved)},
                             "peak_source": "measured: cdtw_calibrate_cell_rate (FADD+FMNMX3+FFMA"
                                            " chains) on this GPU in this run"},
                "argmin": {str(w): b for w, b in zip(bands, best)}, "cut_offset": off}
        if world == 1 and not args.no_sub:
            line["subresults"] = subresults(h, dev, peak)
        if world == 1:
            g, thr, n, dt = cpu_port_gcups(x, q, bands, 10.0)
            line["cpu_baseline"] = {
                "value": g, "unit": "GCUPS", "cores": thr, "kind": "port",
                "sample": f"{n} random windows per band (first 2^20 samples), FP32 OpenMP "
                          f"restatement of openmp_cdtw, {dt:.1f}s"}
        print(json.dumps(line), flush=True)
    h.close()


def subresults(h, dev, peak=None) -> dict:
    """The other scope rows, measured beside the headline (one GPU, rank 0).

    * pruned_search: config 0 (2^20 ECG-like, M=128, W=12) and config 1
      (2^25 metal-like, M in {128,256,512,1024} x P in {5,10,20}): device time
      of a full search, the median of five (statistics excluded; they are
      shared per M), stream
      samples/s, the pruning-inclusive rate windows * cells(M,W) / time, the
      FP64 oracle's distance at the reported window and the relative error,
      and, on the same inputs, the location and wall time of the reference's
      UCR_DTW_BIN on the host cores.
    * batched_search: the 512 queries of config 2 (2^24 ECG-like stream,
      M ~ U{64..1024}, P in {5,10,20}) as one batched graph call, against the
      same queries as 512 plain searches on the same GPU, with the cDTW cells
      the plain path computes per query class and their time floor.
    * pair_fwd_bwd: config 3 (4096 pairs, L=256, W=25, z-normalised random
      walks) and its L=2048/W=409 variant: forward (D only), forward with the
      path record, backward, and their ratio; CUDA-graph replays, device time.
    * wide_band_all_windows: all-windows cDTW of 2^18 windows at M=1024 for
      W = 102, 204, 409 (the lane-group kernel).
    """
    import torch
    from cudadtw_b200 import synth
    out = {}
    stream = torch.cuda.current_stream(dev)

    def dev_time(fn, reps=1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps, r

    def dev_time_median(fn, n=5):
        # n single runs, each bracketed by its own events: a host stall
        # between launches inflates one run, not the median
        ts, r = [], None
        for _ in range(n):
            t, r = dev_time(fn)
            ts.append(t)
        return float(np.median(ts)), r

    # -- pruned search -----------------------------------------------------
    import oracle
    rows = []
    cases = [("config0 ecg 2^20", synth.ecg_like(1 << 20, seed=0), [(128, 10)], 0.05)]
    cases.append(("config1 metal 2^25", synth.metal_like(1 << 25, seed=1),
                  [(m, p) for m in (128, 256, 512, 1024) for p in (5, 10, 20)], 0.1))
    ucr_budget_s = 90.0  # wall seconds of UCR_DTW_BIN runs beside the rows
    for name, x, qs, noise in cases:
        dx = torch.from_numpy(x).to(dev)
        ucr = oracle.UcrShards(x, max_m=1024) if x.size > (1 << 20) else None
        for m, pct in qs:
            q, off = synth.cut_query(x, m, seed=100 + m + pct, noise=noise)
            w = synth.band_from_percent(m, pct)
            avg, std = h.avg_std(dx, m)
            h.set_query(q, w)
            h.prune_cdtw(dx, avg, std)  # warm
            t, (loc, dist) = dev_time_median(lambda: h.prune_cdtw(dx, avg, std))
            nwin = x.size - m + 1
            ref = float(np.sqrt(oracle.cdtw_list(q, x, w, np.array([loc]))[0]))
            row = {"case": name, "M": m, "P": pct, "W": w, "ms": t * 1e3,
                   "samples_per_s": nwin / t,
                   # windows x cells(M, W) / search time: includes what pruning
                   # skipped, so it is not a hardware cell rate
                   "pruning_inclusive_gcups": nwin * cells(m, w) / t / 1e9,
                   "location": int(loc), "planted": int(off),
                   "counts": list(h.search_counts()),
                   "fp64_distance": ref, "rel_err": abs(float(dist) - ref) / ref}
            # the reference's own CPU search on the same inputs (UCR_DTW_BIN
            # built from its sources): whole stream in one process for the
            # 2^20 stream, concurrent shard processes (one per host core) on
            # the 2^25 stream while the time budget lasts
            if ucr_budget_s > 0 and (ucr is None or (m, pct) in UCR_CONFIG1):
                if ucr is None:
                    t0 = time.perf_counter()
                    uloc, udist, cpu, _ = oracle.ucr_dtw(x, q, oracle.ucr_band_arg(w, m))
                    wall, cores, cpus = time.perf_counter() - t0, 1, [cpu]
                else:
                    uloc, udist, wall, cpus = ucr.search(q, w)
                    cores = ucr.shards
                ucr_budget_s -= wall
                row["ucr_location"] = int(uloc)
                row["same_location"] = int(uloc) == int(loc)
                row["ucr_distance"] = udist
                row["cpu_baseline"] = {"value": nwin / wall, "unit": "samples/s", "cores": cores,
                                       "kind": "reference",
                                       "sample": "whole stream; UCR_DTW_BIN wall time" +
                                       (f" over {cores} concurrent shard processes (M-1 halo)"
                                        if cores > 1 else ", one process"),
                                       "ucr_clock_s_total": float(sum(c or 0 for c in cpus))}
                row["gpu_over_ucr_wall"] = wall / t
            rows.append(row)
        if ucr is not None:
            ucr.__exit__(None, None, None)
        del dx
    out["pruned_search"] = rows

    # -- batched vs plain ----------------------------------------------------
    x = synth.ecg_like(1 << 24, seed=0)
    dx = torch.from_numpy(x).to(dev)
    batch = synth.batch_queries(x, 512)  # the 512 queries of the batched configuration
    qs = [b[0] for b in batch]
    ws = [b[1] for b in batch]
    h.search_batched(dx, qs, ws)  # builds and replays the graph once
    tb, (bl, bd) = dev_time(lambda: h.search_batched(dx, qs, ws))

    def plain(counts=None):
        res = []
        for q, w in zip(qs, ws):
            avg, std = h.avg_std(dx, q.size)
            h.set_query(q, w)
            res.append(h.prune_cdtw(dx, avg, std))
            if counts is not None:
                counts.append(h.search_counts())
        return res
    counts = []
    tp, pres = dev_time(lambda: plain(counts))
    same = sum(int(a == r[0]) for a, r in zip(bl, pres))
    # cDTW cells the plain path computes at most (windows reaching the cDTW
    # stage x band cells; early abandoning cuts some), per query class, and
    # the time they need at the headline kernels' cell rate: the floor of any
    # schedule that computes them
    classes = {}
    for q, w, (_, _, ndtw), b in zip(qs, ws, counts, batch):
        key = f"M{64 * ((q.size - 1) // 320)}-{64 * ((q.size - 1) // 320) + 319}_P{b[2]}"
        c = classes.setdefault(key, {"queries": 0, "dtw_windows": 0, "cells": 0.0})
        c["queries"] += 1
        c["dtw_windows"] += int(ndtw)
        c["cells"] += float(ndtw) * cells(q.size, w)
    tot_cells = sum(c["cells"] for c in classes.values())
    out["batched_search"] = {"queries": len(qs), "stream": "ecg 2^24", "batched_s": tb,
                             "plain_s": tp, "speedup": tp / tb, "same_location": same,
                             "plain_cdtw_cells": tot_cells,
                             "cell_floor_s_at_7800_gcups": tot_cells / 7.8e12,
                             "classes": classes,
                             "note": "plain includes the per-length statistics"}
    del dx
    # many short queries on a short stream: the regime where the per-search
    # launches and host round trips of the plain path dominate
    x = synth.ecg_like(1 << 20, seed=1)
    dx = torch.from_numpy(x).to(dev)
    batch = synth.batch_queries(x, 512, seed=3, m_lo=64, m_hi=128)
    qs = [b[0] for b in batch]
    ws = [b[1] for b in batch]
    h.search_batched(dx, qs, ws)
    tb, (bl, bd) = dev_time(lambda: h.search_batched(dx, qs, ws))
    counts = []
    tp, pres = dev_time(lambda: plain(counts))
    same = sum(int(a == r[0]) for a, r in zip(bl, pres))
    short_cells = sum(float(c[2]) * cells(q.size, w) for q, w, c in zip(qs, ws, counts))
    out["batched_search_short"] = {"queries": len(qs), "stream": "ecg 2^20", "M": [64, 128],
                                   "batched_s": tb, "plain_s": tp, "speedup": tp / tb,
                                   "same_location": same,
                                   "plain_cdtw_windows": int(sum(c[2] for c in counts[:len(qs)])),
                                   "plain_cdtw_cells": short_cells,
                                   "cell_floor_s_at_7800_gcups": short_cells / 7.8e12}
    del dx

    # -- search over a stream pushed in pieces (host buffers) ---------------
    x = synth.metal_like(1 << 25, seed=1)
    q, off = synth.cut_query(x, 256, seed=100 + 256 + 10, noise=0.1)
    w = synth.band_from_percent(256, 10)
    xp = torch.from_numpy(x).pin_memory().numpy()

    def streamed():
        h.stream_begin(q, w)
        for a in range(0, x.size, 1 << 22):
            h.stream_push(xp[a:a + (1 << 22)])
        return h.stream_end()
    streamed()
    h.search_host(q, xp, w)
    t0 = time.perf_counter()
    sl, sd, _ = streamed()
    ts = time.perf_counter() - t0
    t0 = time.perf_counter()
    hl, hd = h.search_host(q, xp, w)  # the whole stream in one copy, then the search
    th = time.perf_counter() - t0
    out["stream_search"] = {"stream": "metal 2^25 (host, pinned)", "M": 256, "P": 10, "W": w,
                            "chunk_samples": 1 << 23, "pieces": 8, "streamed_s": ts,
                            "whole_host_search_s": th, "location": int(sl),
                            "same_location": int(sl) == int(hl),
                            "samples_per_s": x.size / ts}
    del xp

    # -- pair forward / backward ------------------------------------------
    pair = {}
    for n, L, W in ((4096, 256, 25), (4096, 2048, 409)):
        rng = np.random.default_rng(3)
        q = torch.from_numpy(np.cumsum(rng.standard_normal((n, L)), 1).astype(np.float32)).to(dev)
        s = torch.from_numpy(np.cumsum(rng.standard_normal((n, L)), 1).astype(np.float32)).to(dev)
        path = torch.empty(h.pair_path_bytes(n, L), dtype=torch.uint8, device=dev)
        D = torch.empty(n, device=dev)
        gq, gs = torch.empty_like(q), torch.empty_like(s)
        fns = {"fwd": lambda: h.pair_fwd(q, s, W, out=D),
               "fwd_path": lambda: h.pair_fwd(q, s, W, path=path, out=D, mode="store"),
               "fwd_path_recompute": lambda: h.pair_fwd(q, s, W, path=path, out=D,
                                                        mode="recompute"),
               "bwd": lambda: h.pair_bwd(q, s, path, dq=gq, ds=gs)}
        fns["fwd_bwd"] = lambda: (fns["fwd_path"](), fns["bwd"]())
        fns["fwd_bwd_recompute"] = lambda: (fns["fwd_path_recompute"](), fns["bwd"]())
        r = {}
        side = torch.cuda.Stream(dev)
        h.use_torch_stream(side)
        with torch.cuda.stream(side):
            for k, f in fns.items():
                for _ in range(3):
                    f()
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=side):
                    for _ in range(10):
                        f()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                g.replay()
                torch.cuda.synchronize()
                e0.record(side)
                g.replay()
                e1.record(side)
                torch.cuda.synchronize()
                r[k + "_ms"] = e0.elapsed_time(e1) / 10
                del g
        h.use_torch_stream(stream)
        c = cells(L, W)
        r["fwd_gcups"] = n * c / (r["fwd_ms"] / 1e3) / 1e9
        r["fwd_bwd_over_fwd"] = r["fwd_bwd_ms"] / r["fwd_ms"]
        r["fwd_bwd_recompute_over_fwd"] = r["fwd_bwd_recompute_ms"] / r["fwd_ms"]
        scratch = h.pair_workspace_bytes(1, L, W, False, True, mode="store")
        r["bytes_per_pair"] = {"path_record": h.pair_path_bytes(1, L),
                               "direction_scratch": scratch,
                               "checkpoint_scratch": h.pair_workspace_bytes(
                                   1, L, W, False, True, mode="recompute"),
                               "full_fp32_band_table": 4 * c}
        r["direction_record_in"] = "shared memory" if scratch == 0 else "device scratch"
        pair[f"{n}x{L}_W{W}"] = r
        del q, s, path, gq, gs
    out["pair_fwd_bwd"] = pair

    # -- wide bands: the lane-group kernel, all windows -----------------------
    x = synth.metal_like((1 << 18) + 1023, seed=1)
    dx = torch.from_numpy(x).to(dev)
    q, _ = synth.cut_query(x, 1024, seed=5, noise=0.1)
    avg, std = h.avg_std(dx, 1024)
    wide = {}
    for W in (102, 204, 409):
        h.set_query(q, W)
        h.gpu_cdtw(dx, avg, std)  # warm-up
        t, _ = dev_time_median(lambda: h.gpu_cdtw(dx, avg, std))
        g = (1 << 18) * cells(1024, W) / t / 1e9
        wide[f"W{W}"] = {"ms": t * 1e3, "gcups": g, "variant": "lane group",
                         "frac_of_measured_cell_rate": g / (peak / 1e9) if peak else None}
    out["wide_band_all_windows"] = {"stream": "metal 2^18 windows", "M": 1024, "bands": wide}
    del dx
    out["refine"] = refine_subresult(h, dev)
    return out


def refine_subresult(h, dev) -> dict:
    """Config 4: 64 templates (M ~ U{128..512}, cut from a 2^24 ECG-like
    stream + N(0, 0.2) noise, band 10%), top-1000 non-overlapping matches
    each, 100 Adam steps (lr 1e-2) in one graph; FP64 recheck of the final
    loss on 4 templates."""
    import torch
    import oracle
    from cudadtw_b200 import synth
    rng = np.random.default_rng(4)
    x = synth.ecg_like(1 << 24, seed=0)
    dx = torch.from_numpy(x).to(dev)
    ms = rng.integers(128, 513, size=64)
    temps, bands, locs = [], [], []
    t0 = time.perf_counter()
    stats = {}
    for i, m in enumerate(ms):
        q, _ = synth.cut_query(x, int(m), seed=700 + i, noise=0.2)
        w = synth.band_from_percent(int(m), 10)
        if m not in stats:
            stats[m] = h.avg_std(dx, int(m))
        h.set_query(q, w)
        l, _ = h.topk(dx, *stats[m], 1000)
        temps.append(q)
        bands.append(w)
        locs.append(l)
    torch.cuda.synchronize()
    t_topk = time.perf_counter() - t0
    k = min(len(l) for l in locs)
    loc = np.stack([l[:k] for l in locs])
    t0 = time.perf_counter()
    new, losses = h.refine_templates(dx, temps, bands, loc, steps=100, lr=1e-2)
    t_ref = time.perf_counter() - t0
    pairs = 64 * k
    cells_step = sum(k * cells(int(m), w) for m, w in zip(ms, bands))
    check = []
    for t in range(4):
        win = np.stack([x[s:s + ms[t]] for s in loc[t]]).astype(np.float32)
        qq = np.repeat(new[t][None, :], k, axis=0)
        d = oracle.pair_fwdbwd(qq, win, bands[t], znorm=True)[0].mean()
        check.append(abs(d - losses[-1, t]) / d)
    fixed = {"templates": 64, "k": int(k), "steps": 100, "topk_s": t_topk,
             "refine_s": t_ref, "ms_per_step": t_ref * 1e3 / 100,
             "pair_steps_per_s": pairs * 100 / t_ref,
             "fwd_gcups_equiv": cells_step * 101 / t_ref / 1e9,
             "loss_first_mean": float(losses[0].mean()),
             "loss_last_mean": float(losses[-1].mean()),
             "templates_improved": int(np.sum(losses[-1] < losses[0])),
             "fp64_recheck_max_rel": float(max(check)),
             "matches": "searched once (cdtw_topk), fixed over the steps"}
    # config 4 as specified: random-walk templates, the top-1000 matches
    # searched again on the device at every step inside the one graph
    temps = [synth.random_walk(int(m), 900 + i) for i, m in enumerate(ms)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    new, losses, fin = h.refine_templates_search(dx, temps, bands, 1000, steps=100, lr=1e-2)
    t_rs = time.perf_counter() - t0
    check, same = [], 0
    for t in range(4):
        win = np.stack([x[s:s + ms[t]] for s in fin[t]]).astype(np.float32)
        qq = np.repeat(new[t][None, :], 1000, axis=0)
        d = oracle.pair_fwdbwd(qq, win, bands[t], znorm=True)[0].mean()
        check.append(abs(d - losses[-1, t]) / d)
        h.set_query(new[t], bands[t])
        same += int(np.array_equal(h.topk(dx, *stats[ms[t]], 1000)[0], fin[t]))
    searched = {"templates": 64, "init": "random walk", "k": 1000, "steps": 100,
                "refine_s": t_rs, "ms_per_step": t_rs * 1e3 / 101,
                "loss_per_step_mean": [float(v) for v in losses.mean(axis=1)[::10]],
                "loss_first_mean": float(losses[0].mean()),
                "loss_last_mean": float(losses[-1].mean()),
                "templates_improved": int(np.sum(losses[-1] < losses[0])),
                "fp64_recheck_max_rel": float(max(check)),
                "plain_topk_recheck_same_matches": f"{same}/4",
                "matches": "top-1000 searched on the device at every step, in the graph"}
    return {"fixed_matches": fixed, "searched_every_step": searched}


def profile_case(name: str) -> None:
    """One small run of a scope row (twice, untimed) for an ncu capture:
    search = config-1 pruned search (2^25 metal-like, M=512, P=10); strip /
    wide = all-windows cDTW of 2^18 windows at M=1024, W=204 (strip kernel /
    lane-group kernel), wide409 the same at W=409 (lane-group kernel);
    batch_short = the batched search of 512 queries (M 64-128) on a 2^20 ECG-like
    stream; topk =
    top-1000 of one M=256 template on a 2^22 ECG-like stream; pair = 256 pairs
    of L=2048, W=409 and 4096 pairs of L=256, W=25 (forward, forward with path,
    backward); refine = 8 templates x 200 matches, 5 Adam steps; refine_search
    = the same with random-walk templates and the matches searched at every
    step."""
    import torch
    from cudadtw_b200 import Handle, synth
    dev = torch.device("cuda", 0)
    with Handle(0) as h:
        for _ in range(2):
            if name in ("search", "search1024"):
                # config-1 pruned search: M=512, P=10 ("search") or M=1024,
                # P=20 ("search1024", the widest band)
                m, p = (512, 10) if name == "search" else (1024, 20)
                x = synth.metal_like(1 << 25, seed=1)
                dx = torch.from_numpy(x).to(dev)
                q, _ = synth.cut_query(x, m, seed=100 + m + p, noise=0.1)
                avg, std = h.avg_std(dx, m)
                h.set_query(q, synth.band_from_percent(m, p))
                h.prune_cdtw(dx, avg, std)
            elif name == "topk":
                x = synth.ecg_like(1 << 22, seed=0)
                dx = torch.from_numpy(x).to(dev)
                q, _ = synth.cut_query(x, 256, seed=5, noise=0.2)
                avg, std = h.avg_std(dx, 256)
                h.set_query(q, 25)
                h.topk(dx, avg, std, 1000)
            elif name == "batch_short":
                x = synth.ecg_like(1 << 20, seed=1)
                dx = torch.from_numpy(x).to(dev)
                batch = synth.batch_queries(x, 512, seed=3, m_lo=64, m_hi=128)
                h.search_batched(dx, [b[0] for b in batch], [b[1] for b in batch])
            elif name in ("strip", "wide", "wide409"):
                # all-windows cDTW of 2^18 windows at M=1024, W=204 (W=409 for
                # "wide409"): the strip kernel ("strip") or the lane-group
                # kernel
                W = 409 if name == "wide409" else 204
                x = synth.metal_like((1 << 18) + 1023, seed=1)
                dx = torch.from_numpy(x).to(dev)
                q, _ = synth.cut_query(x, 1024, seed=5, noise=0.1)
                avg, std = h.avg_std(dx, 1024)
                h.set_query(q, W)
                h.set_band_variant(W, W, "strip16" if name == "strip" else "lane")
                h.gpu_cdtw(dx, avg, std)
            elif name == "pair":
                for n, L, W in ((256, 2048, 409), (4096, 256, 25)):
                    rng = np.random.default_rng(0)
                    q = torch.from_numpy(np.cumsum(rng.standard_normal((n, L)), 1)
                                         .astype(np.float32)).to(dev)
                    s = torch.from_numpy(np.cumsum(rng.standard_normal((n, L)), 1)
                                         .astype(np.float32)).to(dev)
                    path = torch.empty(h.pair_path_bytes(n, L), dtype=torch.uint8, device=dev)
                    h.pair_fwd(q, s, W)
                    h.pair_fwd(q, s, W, path=path, mode="store")
                    h.pair_fwd(q, s, W, path=path, mode="recompute")
                    h.pair_bwd(q, s, path)
            elif name == "refine":
                x = synth.ecg_like(1 << 20, seed=0)
                dx = torch.from_numpy(x).to(dev)
                temps, bands, locs = [], [], []
                for i in range(8):
                    m = 128 + 32 * i
                    q, _ = synth.cut_query(x, m, seed=40 + i, noise=0.2)
                    avg, std = h.avg_std(dx, m)
                    h.set_query(q, m // 10)
                    locs.append(h.topk(dx, avg, std, 200)[0][:200])
                    temps.append(q)
                    bands.append(m // 10)
                h.refine_templates(dx, temps, bands, np.stack(locs), steps=5)
            elif name == "refine_search":
                x = synth.ecg_like(1 << 20, seed=0)
                dx = torch.from_numpy(x).to(dev)
                temps = [synth.random_walk(128 + 32 * i, 60 + i) for i in range(8)]
                h.refine_templates_search(dx, temps, [(128 + 32 * i) // 10 for i in range(8)],
                                          200, steps=5)
            else:
                raise SystemExit(f"unknown profile case {name}")
            torch.cuda.synchronize()
    print("profile case done:", name)


def ctypes_peak(lib, h) -> float:
    import ctypes
    v = ctypes.c_double()
    st = lib.cdtw_calibrate_cell_rate(h._h, ctypes.byref(v))
    if st != 0:
        raise RuntimeError(lib.cdtw_last_error(h._h).decode())
    return v.value


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--profile",
                    choices=["search", "search1024", "topk", "pair", "refine", "refine_search",
                             "strip", "wide", "wide409", "batch_short"],
                    help="run one small case of that row twice (for ncu) and exit")
    ap.add_argument("--no-sub", action="store_true",
                    help="skip the pruned / batched search and pair fwd/bwd sub-results")
    ap.add_argument("--only-kernels", action="store_true",
                    help="device-timed steps only (no calibration, e2e or CPU baseline): "
                         "the target of ncu captures")
    args = ap.parse_args()
    if args.profile:
        profile_case(args.profile)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
