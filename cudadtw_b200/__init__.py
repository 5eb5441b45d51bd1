"""cudadtw_b200: B200-native z-normalised subsequence search under a
Sakoe-Chiba band (the hot path of CUDA-DTW), hand-written sm_100a kernels
behind the C ABI of include/cudadtw.h.

``synth`` (seeded synthetic streams) imports without a GPU; the compute API
(``Handle`` and friends) loads libcudadtw.so on first use and raises if it is
missing -- there is no CPU fallback.
"""
from . import synth  # noqa: F401

__all__ = ["Handle", "band_from_percent", "EUCLIDEAN", "MANHATTAN", "CudaDTWError", "synth"]


def __getattr__(name):
    if name in ("Handle", "band_from_percent", "EUCLIDEAN", "MANHATTAN"):
        from . import api
        return getattr(api, name)
    if name == "CudaDTWError":
        from ._lib import CudaDTWError
        return CudaDTWError
    raise AttributeError(name)
