"""Generates tests/golden/oracle_seq.npz: a small seeded G-buffer sequence and the oracle's outputs on it.

The reference ships no golden vectors for this path (no tests, no fixtures; its golden test against a PyTorch twin is
not published, src/denoise/hush.js:6-7) and cannot run here, so this fixture pins the oracle to itself: it catches
regressions of the CPU restatement and gives the GPU tests a committed target. Inputs come from the host scene
generator (hush_b200.scene), outputs from the f32 oracle with the built-in weights.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hush_b200 import builtin_weights, scene  # noqa: E402
import oracle  # noqa: E402

W, H, FRAMES, SEED = 40, 24, 4, 7


def main():
    cfg = scene.SceneConfig(W, H, FRAMES, n_objects=6, n_moving=2, pan_min=1.0, pan_max=3.0, seed=SEED)
    o = oracle.OracleHush(W, H, builtin_weights())
    out = {}
    for i in range(FRAMES):
        f = scene.frame_host(cfg, i)
        for k in oracle.INPUTS:
            out[f"in{i}_{k}"] = f[k]
        out[f"out{i}"] = o.denoise(f)
    for name in ("A0", "X", "BH0", "C0", "CG", "F0", "F1", "F2", "F3"):
        out[f"last_{name}"] = o.buffer(name).copy()
    out["weights_sha256"] = np.frombuffer(b"728d4cb712ee4bedbf87b12b263de19a0c6318e41b27d57dfbbc6b68388bd0b5",
                                          dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "oracle_seq.npz"), **out)
    print("wrote", os.path.join(HERE, "oracle_seq.npz"))


if __name__ == "__main__":
    main()
