"""ctypes binding of libcudadtw.so (the C ABI declared in include/cudadtw.h).

The shared library is built in-tree (cudadtw_b200/libcudadtw.so).  There is no
fallback: if it is missing or fails to load, importing the compute API raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcudadtw.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "cudadtw.h")

c_int, c_i64, c_vp, c_f32p = ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_f64p = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); every device/host buffer is passed as c_void_p
SIGNATURES = {
    "cdtw_create": (c_int, [ctypes.POINTER(c_vp), c_int]),
    "cdtw_destroy": (c_int, [c_vp]),
    "cdtw_set_stream": (c_int, [c_vp, c_vp]),
    "cdtw_last_error": (ctypes.c_char_p, [c_vp]),
    "cdtw_status_string": (ctypes.c_char_p, [c_int]),
    "cdtw_band_from_percent": (c_int, [c_int, c_int]),
    "cdtw_avg_std": (c_int, [c_vp, c_vp, c_i64, c_int, c_vp, c_vp]),
    "cdtw_set_query": (c_int, [c_vp, c_vp, c_int, c_int, c_int]),
    "cdtw_gpu_cdtw": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_i64, c_int, c_vp]),
    "cdtw_all_windows_host": (c_int, [c_vp, c_vp, c_int, c_vp, c_i64, c_int, c_int, c_vp]),
    "cdtw_calibrate_cell_rate": (c_int, [c_vp, c_f64p]),
    "cdtw_lb_kim": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_i64, c_int, c_vp]),
    "cdtw_lb_keogh": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_i64, c_int, c_vp, c_vp]),
    "cdtw_prune_cdtw": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_int, c_i64p, c_f32p]),
    "cdtw_search_host": (c_int, [c_vp, c_vp, c_int, c_vp, c_i64, c_int, c_int, c_i64p, c_f32p]),
    "cdtw_search_counts": (c_int, [c_vp, c_i64p]),
    "cdtw_search_flag": (c_int, [c_vp, ctypes.POINTER(c_int)]),
    "cdtw_set_memory_limit": (c_int, [c_vp, ctypes.c_size_t]),
    "cdtw_stream_begin": (c_int, [c_vp, c_vp, c_int, c_int, c_int, c_i64]),
    "cdtw_stream_push": (c_int, [c_vp, c_vp, c_i64]),
    "cdtw_stream_end": (c_int, [c_vp, c_i64p, c_f32p, c_i64p]),
    "cdtw_topk": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_int, c_int, c_vp, c_vp,
                          ctypes.POINTER(c_int)]),
    "cdtw_topk_device": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_int, c_int, c_vp, c_vp,
                                 ctypes.POINTER(c_int)]),
    "cdtw_set_band_variant": (c_int, [c_vp, c_int, c_int, c_int]),
    "cdtw_search_batched": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_int, c_int, c_vp, c_vp,
                                    c_vp, c_vp]),
    "ed_all_windows": (c_int, [c_vp, c_vp, c_int, c_vp, c_i64, c_vp]),
    "ed_search_host": (c_int, [c_vp, c_vp, c_int, c_vp, c_i64, c_i64p, c_f64p]),
    "ldtw_all_windows": (c_int, [c_vp, c_vp, c_i64, c_int, c_vp]),
    "ldtw_search_host": (c_int, [c_vp, c_vp, c_int, c_vp, c_i64, c_int, c_int, c_i64p, c_f64p]),
    "ldtw_ref_all_windows": (c_int, [c_vp, c_vp, c_i64, c_int, c_int, c_vp]),
    "ldtw_ref_search_host": (c_int, [c_vp, c_vp, c_int, c_vp, c_i64, c_int, c_int, c_int, c_i64p,
                                     c_f32p]),
    "cdtw_all_windows_noalloc": (c_int, [c_vp, c_int, c_vp, c_i64, c_int, c_int, c_vp, c_vp,
                                         ctypes.c_char_p, c_int]),
    "cdtw_pair_path_bytes": (ctypes.c_size_t, [c_i64, c_int]),
    "cdtw_refine_templates": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_int, c_vp, c_int,
                                      c_int, ctypes.c_float, c_int, c_vp]),
    "cdtw_refine_templates_search": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_int, c_int,
                                             c_int, ctypes.c_float, c_int, c_vp, c_vp]),
    "cdtw_pair_workspace_bytes": (ctypes.c_size_t, [c_i64, c_int, c_int, c_int, c_int]),
    "cdtw_pair_last_mode": (c_int, [c_vp, ctypes.POINTER(c_int)]),
    "cdtw_pair_fwd": (c_int, [c_vp, c_vp, c_vp, c_i64, c_int, c_int, c_int, c_int, c_vp, c_vp]),
    "cdtw_pair_bwd": (c_int, [c_vp, c_vp, c_vp, c_i64, c_int, c_int, c_int, c_vp, c_vp, c_vp,
                              c_vp]),
}

_lib = None


class CudaDTWError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -c 'import __graft_entry__ as g; "
                          "g.build()'` (or `make -C cudadtw_b200/csrc`)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def declared_symbols() -> list[str]:
    """Every function declared in include/cudadtw.h (parsed from the header)."""
    import re
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*|void|size_t)\s+(\w+)\s*\(", text, re.M)))
