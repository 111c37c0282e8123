"""hush_b200: B200-native re-implementation of the Hush denoise path (temporal reprojection, moments, a half-res
parameter MLP, a 5-level edge-aware a-trous pyramid and TAA) as sm_100a CUDA kernels behind the reference's
``Hush`` / ``SVGF`` surface.

The compute path is libhush_b200.so (C ABI in include/hush.h); this package is its host-side mirror.
"""
from .hush import Hush, HushError, HushTimer, builtin_weights, decode_weights, hiddenOf  # noqa: F401
from .post import Post  # noqa: F401
from .svgf import SVGF  # noqa: F401

__all__ = ["Hush", "HushError", "HushTimer", "Post", "SVGF", "hiddenOf", "builtin_weights", "decode_weights"]
