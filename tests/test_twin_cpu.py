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


def _temporal_case(W=48, H=32, seed=5):
    """The oracle two frames into a sequence, then frame 2's TEMPORAL pass alone: the previous frame's stored history
    (keys, colour, moments, par0) and frame 2's inputs and TEMPORAL outputs."""
    cfg = scene.SceneConfig(W, H, 3, n_moving=2, pan_min=1.0, pan_max=3.0, seed=seed)
    frames = [scene.frame_host(cfg, i, clean=True) for i in range(3)]
    o = oracle.OracleHush(W, H, builtin_weights())
    for f in frames[:2]:
        o.denoise(f)
    c = o.frame & 1
    prev = {k: o.buffer(f"{k}{c ^ 1}").copy() for k in ("KEY", "HIST", "MOM")}
    prev["PAR0"] = o.buffer(f"PAR0_{c ^ 1}").copy()
    f = frames[2]
    o.run_pass("temporal", f)
    st = {k: f[k] for k in ("radiance", "normalDepth", "motion", "material")}
    st["key_prev"] = prev["KEY"]
    return st, prev, o.buffer("A0").copy(), o.buffer(f"MOM{c}").copy()


def _f64(a):
    return torch.tensor(np.asarray(a, np.float32).astype(np.float64))


def test_temporal_restatement_tracks_the_oracle_pass():
    """oracle/twin.temporal (float64, the reference of the TEMPORAL adjoint) against the oracle's f32 TEMPORAL pass on
    the same history: equal to the f16 storage rounding."""
    st, prev, A0, mom = _temporal_case()
    A0t, momt = twin.temporal(st, _f64(prev["HIST"]), _f64(prev["MOM"]), _f64(prev["PAR0"]))
    for got, ref in ((A0t.numpy(), A0.astype(np.float64)), (momt.numpy(), mom.astype(np.float64))):
        rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-2 * np.abs(ref).mean())
        assert np.mean(rel <= 2e-3) > 0.995, np.mean(rel <= 2e-3)


def test_temporal_restatement_gradient_matches_central_differences():
    """The float64 TEMPORAL's autograd gradient (the reference the CUDA adjoint is checked against) against its own
    central differences on the history (colour, moments) and alpha / gamma, skipping entries at a kink."""
    st, prev, _, _ = _temporal_case(W=32, H=24, seed=9)
    ins = [_f64(prev["HIST"]).requires_grad_(True), _f64(prev["MOM"]).requires_grad_(True),
           _f64(prev["PAR0"]).requires_grad_(True)]
    rng = np.random.default_rng(3)
    sA = torch.tensor(rng.normal(size=(24, 32, 4)))
    sM = torch.tensor(rng.normal(size=(24, 32, 4)))

    def obj(h, m, p):
        A0, mom = twin.temporal(st, h, m, p)
        return (sA * A0).sum() + (sM * mom).sum()

    grads = torch.autograd.grad(obj(*ins), ins)
    checked = 0
    for k, (x, g) in enumerate(zip(ins, grads)):
        flat = g.reshape(-1).abs()
        idx = torch.argsort(flat, descending=True)[:6].tolist() + rng.choice(flat.numel(), 6).tolist()
        for i in idx:
            base = [t.detach().clone() for t in ins]
            h = 1e-6 * max(1.0, abs(base[k].reshape(-1)[i].item()))
            vals = []
            for d in (-h, 0.0, h):
                b = [t.clone() for t in base]
                b[k].reshape(-1)[i] += d
                vals.append(obj(*b).item())
            fm, f0, fp = vals
            left, right = (f0 - fm) / h, (fp - f0) / h
            if abs(left - right) > 0.05 * max(abs(left), abs(right), 1e-12):
                continue  # a kink (clamp, max, branch) inside the interval
            fd = (fp - fm) / (2 * h)
            ga = g.reshape(-1)[i].item()
            assert abs(fd - ga) <= 1e-5 * max(abs(fd), flat.max().item()), (k, i, fd, ga)
            checked += 1
    assert checked >= 20


def test_coarse_restatement_tracks_the_oracle_passes():
    """oracle/twin.coarse1 / coarse2 (float64, the references of the coarse adjoints: down() without the f16 rounding,
    then the 5x5 a-trous of steps 1 and 2) against the oracle's f32 COARSE1 and coarse2 passes on the same frame: equal
    to the f16 rounding of down() and of the stored levels."""
    cfg = scene.SceneConfig(64, 48, 3, n_moving=2, seed=8)
    frames = [scene.frame_host(cfg, i, clean=True) for i in range(3)]
    o = oracle.OracleHush(cfg.width, cfg.height, builtin_weights())
    for f in frames[:2]:
        o.denoise(f)
    f = frames[2]
    for p in ("temporal", "infer", "coarse1", "coarse2"):
        o.run_pass(p, f)
    F2, F3 = twin.unpack_half(o.buffer("F2")), twin.unpack_half(o.buffer("F3"))
    Gq = twin.coarse_guide(o.buffer("CG"))
    c1 = twin.coarse1(F2[..., 4:8], F3[..., 3], Gq)
    c0 = twin.coarse2(c1, Gq)
    for got, name in ((c1, "C1"), (c0, "C0")):
        ref = o.buffer(name).astype(np.float64)
        rel = np.abs(got.numpy() - ref) / np.maximum(np.abs(ref), 1e-2 * np.abs(ref).mean())
        assert np.mean(rel <= 2e-3) > 0.995, (name, np.mean(rel <= 2e-3))


def test_block_means_restatement_tracks_the_oracle():
    """oracle/twin.block_means (float64, the window gradient's path from TEMPORAL's A0 into the block means) against
    the block means the oracle's TEMPORAL pass stores (F2.zw: the mean of the f16 A0 over a block's surface pixels,
    then stored as f16 rounded toward zero): equal to that rounding, zero on blocks without a surface."""
    cfg = scene.SceneConfig(64, 48, 3, n_moving=2, seed=9)
    frames = [scene.frame_host(cfg, i, clean=True) for i in range(3)]
    o = oracle.OracleHush(cfg.width, cfg.height, builtin_weights())
    for f in frames[:2]:
        o.denoise(f)
    f = frames[2]
    o.run_pass("temporal", f)
    c = o.frame & 1
    A0 = torch.tensor(o.buffer("A0").astype(np.float64))
    surf = torch.tensor(o.buffer(f"KEY{c}").astype(np.float64)[..., 2] >= 0)
    got = twin.block_means(A0, surf).numpy()
    ref = twin.unpack_half(o.buffer("F2"))[..., 4:8].numpy()
    none = twin.unpack_half(o.buffer("F3"))[..., 3].numpy() <= 0
    assert none.any() and (~none).any()
    assert np.all(got[none] == 0.0) and np.all(ref[none] == 0.0)
    rel = np.abs(got[~none] - ref[~none]) / np.maximum(np.abs(ref[~none]), 1e-2 * np.abs(ref[~none]).mean())
    assert rel.max() <= 2 ** -9, rel.max()
