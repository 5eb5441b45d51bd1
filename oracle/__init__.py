"""CPU oracle -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``liboracle.so`` (an FP64 restatement of the CUDA-DTW
reference arithmetic, see cdtw_oracle.cpp) and runners for the reference's UCR
Suite binaries compiled from source into ``oracle/_ref``.  Only the tests,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference legs use
this package; the cudadtw_b200 product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None

_f64p = ctypes.POINTER(ctypes.c_double)
_f32p = ctypes.POINTER(ctypes.c_float)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i64 = ctypes.c_int64
_int = ctypes.c_int


def build() -> None:
    """Builds liboracle.so and, when the reference tree is present (its root
    in the CDTW_REFERENCE_DIR environment variable), the reference's UCR Suite
    binaries into _ref/ (kept when already built)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    refdir = os.environ.get("CDTW_REFERENCE_DIR", "")
    if refdir and os.path.isdir(refdir) and not all(
            os.path.exists(os.path.join(REF_DIR, b))
            for b in ("UCR_DTW_BIN", "UCR_ED_BIN", "UCR_DTW", "ref_ldtw")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFDIR={refdir}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        sigs = {
            "orc_znorm": (None, [_f64p, _int, _f64p]),
            "orc_window_stats": (None, [_f32p, _i64, _int, _f64p, _f64p]),
            "orc_cdtw_all": (None, [_f64p, _int, _f32p, _i64, _int, _int, _f64p]),
            "orc_cdtw_list": (None, [_f64p, _int, _f32p, _i64, _int, _int, _i64p, _i64, _f64p]),
            "orc_cdtw_pair": (ctypes.c_double, [_f64p, _f64p, _int, _int, _int]),
            "orc_argmin": (None, [_f64p, _i64, _i64p, _f64p]),
            "orc_envelope": (None, [_f64p, _int, _int, _f64p, _f64p]),
            "orc_lb_kim": (None, [_f64p, _int, _f32p, _i64, _int, _f64p]),
            "orc_lb_keogh": (None, [_f64p, _int, _int, _f32p, _i64, _int, _f64p]),
            "orc_lb_keogh_rev": (None, [_f64p, _int, _int, _f32p, _i64, _int, _f64p]),
            "orc_ldtw_all": (None, [_f64p, _int, _f32p, _i64, _int, _int, _f64p]),
            "orc_ed_all": (None, [_f64p, _int, _f64p, _i64, _f64p]),
            "orc_cdtw_ref_f32": (None, [_f32p, _int, _f32p, _f32p, _f32p, _i64p, _i64, _int,
                                        _int, _f32p]),
            "orc_pair_fwdbwd": (None, [_f32p, _f32p, _i64, _int, _int, _int, _int, _int, _f32p,
                                       _f64p, _f64p, _f64p, _f64p]),
            "orc_pair_fwdbwd64": (None, [_f64p, _f64p, _i64, _int, _int, _int, _int, _f64p, _f64p,
                                         _f64p, _f64p]),
            "orc_pair_path_grad": (None, [_f32p, _f32p, _i64, _int, _int, _int, _int, _u32p, _u32p,
                                          _f32p, _f64p, _f64p, _f64p, _i32p]),
            "orc_max_threads": (_int, []),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def znorm(q) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.empty_like(q)
    lib().orc_znorm(_p(q, _f64p), q.size, _p(out, _f64p))
    return out


def window_stats(x: np.ndarray, m: int):
    x = np.ascontiguousarray(x, dtype=np.float32)
    nw = x.size - m + 1
    mu = np.empty(nw, np.float64)
    sd = np.empty(nw, np.float64)
    lib().orc_window_stats(_p(x, _f32p), x.size, m, _p(mu, _f64p), _p(sd, _f64p))
    return mu, sd


def cdtw_all(query: np.ndarray, x: np.ndarray, w: int, euclid: bool = True) -> np.ndarray:
    """Squared (or absolute) cDTW of the z-normalised query vs every window."""
    zq = znorm(query)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.size - zq.size + 1, np.float64)
    lib().orc_cdtw_all(_p(zq, _f64p), zq.size, _p(x, _f32p), x.size, w, int(euclid),
                       _p(out, _f64p))
    return out


def cdtw_list(query, x, w, idx, euclid=True) -> np.ndarray:
    zq = znorm(query)
    x = np.ascontiguousarray(x, dtype=np.float32)
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    out = np.empty(idx.size, np.float64)
    lib().orc_cdtw_list(_p(zq, _f64p), zq.size, _p(x, _f32p), x.size, w, int(euclid),
                        _p(idx, _i64p), idx.size, _p(out, _f64p))
    return out


def cdtw_pair(a, b, w, euclid=True) -> float:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return lib().orc_cdtw_pair(_p(a, _f64p), _p(b, _f64p), a.size, w, int(euclid))


def argmin(v: np.ndarray):
    v = np.ascontiguousarray(v, dtype=np.float64)
    i = ctypes.c_int64()
    val = ctypes.c_double()
    lib().orc_argmin(_p(v, _f64p), v.size, ctypes.byref(i), ctypes.byref(val))
    return i.value, val.value


def envelope(q, w):
    q = np.ascontiguousarray(q, dtype=np.float64)
    lo = np.empty_like(q)
    hi = np.empty_like(q)
    lib().orc_envelope(_p(q, _f64p), q.size, w, _p(lo, _f64p), _p(hi, _f64p))
    return lo, hi


def lb_kim(query, x, euclid=True):
    zq = znorm(query)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.size - zq.size + 1, np.float64)
    lib().orc_lb_kim(_p(zq, _f64p), zq.size, _p(x, _f32p), x.size, int(euclid), _p(out, _f64p))
    return out


def lb_keogh(query, x, w, euclid=True):
    zq = znorm(query)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.size - zq.size + 1, np.float64)
    lib().orc_lb_keogh(_p(zq, _f64p), zq.size, w, _p(x, _f32p), x.size, int(euclid),
                       _p(out, _f64p))
    return out


def lb_keogh_rev(query, x, w, euclid=True):
    zq = znorm(query)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.size - zq.size + 1, np.float64)
    lib().orc_lb_keogh_rev(_p(zq, _f64p), zq.size, w, _p(x, _f32p), x.size, int(euclid),
                           _p(out, _f64p))
    return out


def ldtw_all(query, x, w, euclid=True):
    zq = znorm(query)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.size - zq.size + 1, np.float64)
    lib().orc_ldtw_all(_p(zq, _f64p), zq.size, _p(x, _f32p), x.size, w, int(euclid),
                       _p(out, _f64p))
    return out


def ed_all(query, x):
    zq = znorm(query)
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(x.size - zq.size + 1, np.float64)
    lib().orc_ed_all(_p(zq, _f64p), zq.size, _p(x, _f64p), x.size, _p(out, _f64p))
    return out


def cdtw_ref_f32(zq32, x, avg32, sd32, idx, w, nthreads):
    """The reference's FP32 OpenMP all-windows cDTW (timing baseline)."""
    zq32 = np.ascontiguousarray(zq32, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    avg32 = np.ascontiguousarray(avg32, dtype=np.float32)
    sd32 = np.ascontiguousarray(sd32, dtype=np.float32)
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    out = np.empty(idx.size, np.float32)
    lib().orc_cdtw_ref_f32(_p(zq32, _f32p), zq32.size, _p(x, _f32p), _p(avg32, _f32p),
                           _p(sd32, _f32p), _p(idx, _i64p), idx.size, w, nthreads,
                           _p(out, _f32p))
    return out


def max_threads() -> int:
    return lib().orc_max_threads()


_LOC = re.compile(r"Location\s*:\s*(-?\d+)")
_DIST = re.compile(r"Distance\s*:\s*([-+0-9.eEinfa]+)")
_TIME = re.compile(r"Total Execution Time\s*:\s*([0-9.eE+-]+)")


def _run_ucr(binary: str, args: list[str]):
    path = os.path.join(REF_DIR, binary)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the "
                                "reference sources are available")
    out = subprocess.run([path] + args, check=True, stdout=subprocess.PIPE,
                         stderr=subprocess.DEVNULL, text=True).stdout
    loc = int(_LOC.search(out).group(1))
    dist = float(_DIST.search(out).group(1))
    tm = _TIME.search(out)
    return loc, dist, (float(tm.group(1)) if tm else None), out


def ucr_dtw(x: np.ndarray, q: np.ndarray, r_arg: str):
    """Run the reference UCR_DTW_BIN (argv: data query m R n; R<=1 is a band
    fraction, R>1 an absolute band, UCR_DTW_BIN.cpp:417-425) on exact FP64
    widenings of the float32 inputs.  Returns (location, distance, cpu_s, stdout)."""
    with tempfile.TemporaryDirectory() as d:
        xp, qp = os.path.join(d, "data.f64"), os.path.join(d, "query.f64")
        x.astype(np.float64).tofile(xp)
        q.astype(np.float64).tofile(qp)
        return _run_ucr("UCR_DTW_BIN", [xp, qp, str(q.size), r_arg, str(x.size)])


def ucr_band_arg(w: int, m: int) -> str:
    """UCR_DTW_BIN's R argument for an absolute band w: R > 1 is taken as the
    band itself (UCR_DTW_BIN.cpp:420-423); w <= 1 is passed as the fraction
    w / m, which UCR floors back to w."""
    if w > 1:
        return str(int(w))
    return repr((w + 0.5) / m) if w == 1 else "0"


class UcrShards:
    """UCR_DTW_BIN over `shards` concurrent processes on one stream: shard s
    covers its share of the windows of the longest query `max_m` plus the
    samples that follow (the halo), written once as exact FP64 widenings of
    the float32 samples.  ``search(q, w)`` runs every shard on its windows
    (UCR reads only the n samples it is given) and combines the shard results
    by the FP64 oracle's distance at each shard's location, lowest location
    on ties (UCR prints 6 significant digits).  Use as a context manager."""

    def __init__(self, x: np.ndarray, shards: int | None = None, max_m: int = 8192):
        self.x = x
        self.path = os.path.join(REF_DIR, "UCR_DTW_BIN")
        if not os.path.exists(self.path):
            raise FileNotFoundError(f"{self.path} missing: run `make -C oracle ref`")
        self.shards = max(1, min(shards or (os.cpu_count() or 1), x.size))
        self.bounds = [x.size * s // self.shards for s in range(self.shards + 1)]
        self.dir = tempfile.TemporaryDirectory()
        self.files = []
        for s in range(self.shards):
            a = self.bounds[s]
            fp = os.path.join(self.dir.name, f"data{s}.f64")
            x[a:min(x.size, self.bounds[s + 1] + max_m - 1)].astype(np.float64).tofile(fp)
            self.files.append(fp)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.dir.cleanup()

    def search(self, q: np.ndarray, w: int):
        """Returns (location, distance as UCR printed it, wall seconds,
        [per-shard clock() seconds])."""
        import time
        m = q.size
        nw = self.x.size - m + 1
        qp = os.path.join(self.dir.name, "query.f64")
        q.astype(np.float64).tofile(qp)
        jobs = []
        for s in range(self.shards):
            a, b = self.bounds[s], min(self.bounds[s + 1], nw)
            if b > a:
                jobs.append((a, self.files[s], b - a + m - 1))
        t0 = time.perf_counter()
        procs = [subprocess.Popen([self.path, fp, qp, str(m), ucr_band_arg(w, m), str(n)],
                                  stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                 for _, fp, n in jobs]
        outs = [p.communicate()[0] for p in procs]
        wall = time.perf_counter() - t0
        if any(p.returncode != 0 for p in procs):
            raise RuntimeError("UCR_DTW_BIN failed on a shard")
        locs, dists, cpus = [], [], []
        for (a, _, _), out in zip(jobs, outs):
            locs.append(a + int(_LOC.search(out).group(1)))
            dists.append(float(_DIST.search(out).group(1)))
            tm = _TIME.search(out)
            cpus.append(float(tm.group(1)) if tm else None)
        exact = cdtw_list(q, self.x, w, np.array(locs, dtype=np.int64))
        best = min(range(len(jobs)), key=lambda s: (exact[s], locs[s]))
        return locs[best], dists[best], wall, cpus


def write_text(path: str, v: np.ndarray) -> None:
    """One value per line, each float32 printed exactly (9 significant digits
    round-trip), so a text reader recovers the float32 values."""
    np.savetxt(path, np.asarray(v, np.float32).astype(np.float64), fmt="%.9g")


def ucr_dtw_text(data_path: str, query_path: str, m: int, r_arg: str):
    """Run the reference UCR_DTW (text input, UCR_DTW.cpp:381-427) on files.
    Returns (location, distance, cpu_s, stdout)."""
    return _run_ucr("UCR_DTW", [data_path, query_path, str(m), r_arg])


def ref_ldtw(q: np.ndarray, x: np.ndarray, w: int, znorm: bool = True):
    """The reference's own LDTW host code (z_serial_ldtw / serial_ldtw of
    include/ldtw.cuh, built into _ref/ref_ldtw) on every window, with the
    inputs its GPU-ldtw.cu makes (FP32 query z-normalisation, avg_std window
    statistics).  Returns (float32 costs per window, determine_min's index)."""
    path = os.path.join(REF_DIR, "ref_ldtw")
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
    with tempfile.TemporaryDirectory() as d:
        qp, xp, rp = (os.path.join(d, n) for n in ("q.bin", "s.bin", "r.bin"))
        np.ascontiguousarray(q, np.float32).tofile(qp)
        np.ascontiguousarray(x, np.float32).tofile(xp)
        out = subprocess.run([path, qp, xp, str(q.size), str(x.size), str(w),
                              "z" if znorm else "raw", rp], check=True, stdout=subprocess.PIPE,
                             text=True).stdout
        r = np.fromfile(rp, dtype=np.float32)
    loc = int(re.search(r"found at index (\d+)", out).group(1))
    return r, loc


def ucr_ed(x: np.ndarray, q: np.ndarray):
    """Run the reference UCR_ED_BIN (argv: data query m n, UCR_ED_BIN.cpp:115-135)."""
    with tempfile.TemporaryDirectory() as d:
        xp, qp = os.path.join(d, "data.f64"), os.path.join(d, "query.f64")
        x.astype(np.float64).tofile(xp)
        q.astype(np.float64).tofile(qp)
        return _run_ucr("UCR_ED_BIN", [xp, qp, str(q.size), str(x.size)])


def pair_fwdbwd(q, s, W: int, euclid: bool = True, znorm: bool = True, f32: bool = False,
                dD=None):
    """Pairwise cDTW forward/backward (orc_pair_fwdbwd).  q, s: (n, L) float32.
    Returns D (n,), dq (n, L), ds (n, L), margin (n,)."""
    q = np.ascontiguousarray(q, dtype=np.float32)
    s = np.ascontiguousarray(s, dtype=np.float32)
    n, L = q.shape
    D = np.empty(n)
    dq = np.empty((n, L))
    ds = np.empty((n, L))
    mg = np.empty(n)
    up = None if dD is None else np.ascontiguousarray(dD, dtype=np.float32)
    lib().orc_pair_fwdbwd(_p(q, _f32p), _p(s, _f32p), n, L, W, int(euclid), int(znorm), int(f32),
                          None if up is None else _p(up, _f32p), _p(D, _f64p), _p(dq, _f64p),
                          _p(ds, _f64p), _p(mg, _f64p))
    return D, dq, ds, mg


def pair_fwdbwd64(q, s, W: int, euclid: bool = True, znorm: bool = True):
    """FP64 forward/backward on float64 inputs (orc_pair_fwdbwd64), for
    finite-difference checks.  Returns D, dq, ds, margin."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    s = np.ascontiguousarray(s, dtype=np.float64)
    n, L = q.shape
    D = np.empty(n)
    dq = np.empty((n, L))
    ds = np.empty((n, L))
    mg = np.empty(n)
    lib().orc_pair_fwdbwd64(_p(q, _f64p), _p(s, _f64p), n, L, W, int(euclid), int(znorm),
                            _p(D, _f64p), _p(dq, _f64p), _p(ds, _f64p), _p(mg, _f64p))
    return D, dq, ds, mg


def pair_path_grad(q, s, W: int, rows, cols, euclid: bool = True, znorm: bool = True, dD=None):
    """FP64 cost and gradient along a given path (device path-record runs).
    Returns cost (n,), dq, ds (n, L), valid (n,) bool."""
    q = np.ascontiguousarray(q, dtype=np.float32)
    s = np.ascontiguousarray(s, dtype=np.float32)
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    n, L = q.shape
    cost = np.empty(n)
    dq = np.empty((n, L))
    ds = np.empty((n, L))
    ok = np.empty(n, np.int32)
    up = None if dD is None else np.ascontiguousarray(dD, dtype=np.float32)
    lib().orc_pair_path_grad(_p(q, _f32p), _p(s, _f32p), n, L, W, int(euclid), int(znorm),
                             _p(rows, _u32p), _p(cols, _u32p),
                             None if up is None else _p(up, _f32p), _p(cost, _f64p),
                             _p(dq, _f64p), _p(ds, _f64p), _p(ok, _i32p))
    return cost, dq, ds, ok.astype(bool)
