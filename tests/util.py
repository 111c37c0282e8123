"""Shared helpers of the tests: tolerance checks and oracle <-> CUDA state transfer."""
import numpy as np

# Parity bound: |cuda - oracle| <= 2e-3 * max(|oracle|, floor) per channel, floor = 1e-2 of the
# frame's mean absolute value (relative error on near-zero values is meaningless).
REL_TOL = 2e-3
FLOOR_FRAC = 1e-2


def mismatch(cuda: np.ndarray, ref: np.ndarray, rel: float = REL_TOL, floor_frac: float = FLOOR_FRAC,
             channels=slice(None)):
    """Fraction of values outside the bound, the largest scaled error, and the bound floor."""
    a = np.asarray(cuda, dtype=np.float64)[..., channels]
    b = np.asarray(ref, dtype=np.float64)[..., channels]
    finite = np.isfinite(b)
    floor = floor_frac * max(float(np.mean(np.abs(b[finite]))) if finite.any() else 0.0, 1e-6)
    scale = np.maximum(np.abs(b), floor)
    err = np.abs(a - b) / scale
    err[~finite & (a == b)] = 0.0
    err[~np.isfinite(err)] = np.inf
    bad = err > rel
    return float(bad.mean()) if bad.size else 0.0, float(err.max()) if err.size else 0.0, floor


def to_f32(x):
    try:
        import torch

        if isinstance(x, torch.Tensor):
            return x.detach().float().cpu().numpy()
    except ImportError:
        pass
    return np.asarray(x, dtype=np.float32)
