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


def test_pair_sizes():
    """Path record and direction scratch sizes (host-only sizing calls)."""
    lib = _lib.load()
    # path record: 4 doubles + row and column runs (2 x L words) per pair
    for L in (1, 256, 2048):
        assert lib.cdtw_pair_path_bytes(3, L) == 3 * (32 + 8 * L)
    # short pairs keep the direction record in shared memory: only the
    # z-normalised copies (2 x n x L floats, 256-byte slices) are scratch
    assert lib.cdtw_pair_workspace_bytes(1, 256, 25, 0, 1) == 0
    assert lib.cdtw_pair_workspace_bytes(4096, 256, 25, 1, 1) == 2 * 4096 * 256 * 4
    # long pairs: 2 bits per band cell in whole 64-byte-per-lane chunks of
    # 16 anti-diagonals (32 lanes of 13 slots, 32-bit elements)
    assert lib.cdtw_pair_workspace_bytes(1, 2048, 409, 0, 1) == 256 * 64 * 32
    assert lib.cdtw_pair_workspace_bytes(1, 2048, 409, 0, 0) == 0
    assert lib.cdtw_pair_workspace_bytes(0, 256, 25, 0, 1) == 0  # invalid size


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
