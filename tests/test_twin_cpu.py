"""The FP64 training-twin restatement (oracle/twin.py) against the oracle's frame (CPU only): same graph without the
f16 storage rounding, so the TAA outputs agree to the rounding level."""
import numpy as np
import pytest

import oracle
from hush_b200 import builtin_weights, scene

torch = pytest.importorskip("torch")
from oracle import twin  # noqa: E402


def test_twin_forward_tracks_the_oracle():
    cfg = scene.SceneConfig(48, 32, 3, n_moving=1, seed=3)
    frames = [scene.frame_host(cfg, i, clean=True) for i in range(3)]
    w16 = builtin_weights()
    o = oracle.OracleHush(cfg.width, cfg.height, w16)
    for f in frames[:2]:
        o.denoise(f)
    f = frames[2]
    c = o.frame & 1
    for p in ("temporal", "infer", "mid2", "mid3", "coarse1", "coarse2", "fine_final", "taa"):
        o.run_pass(p, f)
    st = {k: o.buffer(k).copy() for k in ("F0", "F1", "F2", "F3", "A0", "C0", "CG")}
    st["key"] = o.buffer(f"KEY{c}").copy()
    st["taa_prev"] = o.buffer(f"TAA{c ^ 1}").copy()
    for k in ("material", "emission", "motion"):
        st[k] = f[k]
    st["clean"] = f["clean"]
    theta = torch.tensor(w16.view(np.float16).astype(np.float64))
    loss, parts = twin.twin_loss(st, theta, return_all=True)
    ref = o.buffer(f"TAA{c}").astype(np.float64)[..., :3]
    out = parts["out"].numpy()
    rel = np.abs(out - ref) / (np.abs(ref) + 1e-2)
    assert np.mean(rel < 2e-2) > 0.99, np.mean(rel < 2e-2)
    par_ref = np.concatenate([o.buffer(f"PAR0_{c}"), o.buffer("PAR1"), o.buffer("PAR2")], -1).astype(np.float64)
    rp = np.abs(parts["par"].numpy() - par_ref) / (np.abs(par_ref) + 1e-3)
    assert np.mean(rp < 5e-3) > 0.99
    assert np.isfinite(loss.item()) and loss.item() > 0
