"""CPU tests of the C ABI library: it loads, exports every symbol that
include/cudadtw.h declares, and its host-only logic behaves (no GPU work)."""
import ctypes

from cudadtw_b200 import _lib


def test_library_loads_and_exports_header_symbols():
    lib = _lib.load()
    declared = _lib.declared_symbols()
    assert "cdtw_gpu_cdtw" in declared and "cdtw_create" in declared
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in cudadtw.h but not exported"
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_band_from_percent_matches_driver_formula():
    lib = _lib.load()
    for m in (64, 100, 128, 256, 1000, 1024, 4096):
        for p in (0, 1, 5, 7, 10, 20, 33, 100):
            assert lib.cdtw_band_from_percent(m, p) == int(m * (p * 0.01))


def test_status_strings_and_null_handle():
    lib = _lib.load()
    assert lib.cdtw_status_string(0) == b"ok"
    assert lib.cdtw_status_string(4) == b"device wait timed out"
    assert lib.cdtw_destroy(None) == 1  # CDTW_EINVAL, no crash
    assert lib.cdtw_create(None, 0) == 1


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    lib = _lib.load()
    h = ctypes.c_void_p()
    st = lib.cdtw_create(ctypes.byref(h), 0)
    assert st in (1, 3) and not h.value


def test_drivers_usage_and_argument_checks_without_gpu():
    """The drop-in drivers keep the reference's usage line and return 1 on
    bad arguments before touching a GPU."""
    import os
    import subprocess
    d = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                     "cudadtw_b200", "drivers")
    for name, nargs in (("GPU-DTW", 5), ("GPU-ED", 4), ("GPU-LDTW", 5)):
        exe = os.path.join(d, name)
        if not os.path.exists(exe):
            continue
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 1 and r.stdout.startswith("call")
    exe = os.path.join(d, "GPU-DTW")
    if os.path.exists(exe):
        r = subprocess.run([exe, "q", "s", "8", "100", "10"], capture_output=True, text=True)
        assert r.returncode == 1 and "window = 0" in r.stdout  # M < 11 refused
