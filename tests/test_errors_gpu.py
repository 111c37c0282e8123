"""Error report of the MLP forms on the 1920x1080 sequence (3 moving objects, pan U[0,4] px/frame), on a B200:
the FP32 plain form, the BF16 and F16 tensor-core forms and plain SVGF against the FP64 oracle and against the
noise-free radiance, and the MLP's 12 predicted parameters per output against the FP64 oracle's, each form started
from the oracle's exact history. Prints the tables it asserts on (pytest -s)."""
import numpy as np
import pytest

import oracle
from hush_b200 import SVGF, Hush, builtin_weights, scene

from .util import mismatch, to_f32

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FORMS = ("fp32", "bf16", "f16")
PARAMS = ["alpha", "gamma", "beta", "kappa", "s0", "s1", "s2", "s3", "c0", "c1", "c2", "c3"]
N_FRAMES = 6


def _clipped_rel(out, clean):
    d = clean.abs() + 1e-2
    return torch.clamp((out - clean).abs() / d, max=1.0).mean().item()


def _flicker(out, prev_out, clean, prev_clean):
    d = clean.abs() + 1e-2
    return torch.clamp(((out - prev_out) - (clean - prev_clean)).abs() / d, max=1.0).mean().item()


def test_mlp_forms_at_1080p_against_fp64_and_clean():
    cfg = scene.CONFIG_1080P
    W, H = cfg.width, cfg.height
    w16 = builtin_weights()
    o64 = oracle.OracleHush(W, H, w16, fp64=True)
    forms = {m: Hush(0, {"width": W, "height": H, "mlp": m}) for m in FORMS}
    svgf = SVGF(0, W, H)
    rows = {k: [] for k in FORMS + ("svgf", "oracle_f64")}
    flick = {k: [] for k in rows}
    beyond = {m: [] for m in FORMS}
    prev = {}
    prev_frame = None
    for i in range(N_FRAMES):
        fr = scene.frame_device(cfg, i, clean=True)
        clean = fr["clean"]
        host = {k: fr[k].cpu().numpy() for k in oracle.INPUTS}
        ref = o64.denoise(host).astype(np.float32)
        outs = {"oracle_f64": torch.from_numpy(ref).cuda()[..., :3]}
        for m, g in forms.items():
            got = g.denoise(fr)
            torch.cuda.synchronize()
            got32 = to_f32(got)
            beyond[m].append((mismatch(got32, ref)[0], mismatch(got32, ref, rel=5e-2)[0]))
            outs[m] = got.float()[..., :3].clone()
        sv = dict(fr)
        sv["prevNormalDepth"] = prev_frame["normalDepth"] if prev_frame else fr["normalDepth"]
        sv["prevMotion"] = prev_frame["motion"] if prev_frame else fr["motion"]
        outs["svgf"] = svgf.encode(sv).float()[..., :3].clone()
        if i > 0:  # frame 0 has no history on any side
            for k, o in outs.items():
                rows[k].append(_clipped_rel(o, clean))
                flick[k].append(_flicker(o, prev[k], clean, prev_frame["clean"]))
        prev = outs
        prev_frame = fr

    print(f"\n1920x1080, frames 1..{N_FRAMES - 1} (frame 0 has no history)")
    print("| form | values beyond 2e-3 rel. of the f64 oracle (mean over frames / last) | beyond 5e-2 | clipped rel-L1 "
          "to clean | temporal flicker |")
    print("|---|---|---|---|---|")
    for k in rows:
        b = beyond.get(k)
        c1 = f"{np.mean([x[0] for x in b]):.2e} / {b[-1][0]:.2e}" if b else "—"
        c2 = f"{np.mean([x[1] for x in b]):.2e}" if b else "—"
        print(f"| {k} | {c1} | {c2} | {np.mean(rows[k]):.4f} | {np.mean(flick[k]):.4f} |")

    # the MLP's outputs: one more frame with every form started from the FP64 oracle's exact state (the history
    # buffers uploaded, the frame parity aligned), so that each form's parameters and the oracle's come from the
    # same history and inputs
    k = N_FRAMES
    fr = scene.frame_device(cfg, k)
    host = {n: fr[n].cpu().numpy() for n in oracle.INPUTS}
    state = {n: torch.from_numpy(o64.buffer(n).copy()).cuda() for n in oracle.BUF_NAMES}
    o64.denoise(host)
    c = k & 1
    ref_p = np.concatenate([o64.buffer(f"PAR0_{c}"), o64.buffer("PAR1"), o64.buffer("PAR2")], -1).astype(np.float64)
    sky = o64.buffer("F3")[..., 2].astype(np.float32) < 0
    print(f"\nMLP parameters of frame {k} against the FP64 oracle from the same state "
          "(|a - b| / (|b| + 1e-3) over non-sky rows; both sides stored as f16)")
    print("| output | " + " | ".join(f"{m} mean / max" for m in FORMS) + " |")
    print("|---|" + "---|" * len(FORMS))
    stats = {}
    for m in FORMS:
        g = Hush(0, {"width": W, "height": H, "mlp": m})
        for _ in range(k):
            g.end_frame()
        for n, t in state.items():
            g.buffer(n).copy_(t)
        g.denoise(fr)
        torch.cuda.synchronize()
        got_p = np.concatenate([g.buffer(n).cpu().numpy() for n in (f"PAR0_{c}", "PAR1", "PAR2")], -1)
        a, b = got_p[~sky].astype(np.float64), ref_p[~sky]
        rel = np.abs(a - b) / (np.abs(b) + 1e-3)
        stats[m] = (rel.mean(0), rel.max(0))
        g.destroy()
    for j, p in enumerate(PARAMS):
        print(f"| {p} | " + " | ".join(f"{stats[m][0][j]:.1e} / {stats[m][1][j]:.1e}" for m in FORMS) + " |")

    # bounds: every form (FP32, and the split-precision F16 / BF16 tensor-core forms) inside the per-channel 2e-3
    # bound of the FP64 oracle on all but 1e-3 of values; BF16 no worse than FP32 against the noise-free image; the
    # 12 MLP outputs of every form within 1e-3 (mean) of the FP64 oracle's
    for m in ("fp32", "f16", "bf16"):
        assert max(x[0] for x in beyond[m]) <= 1e-3, (m, beyond[m])
    assert np.mean(rows["bf16"]) <= np.mean(rows["fp32"]) * 1.01
    assert abs(np.mean(rows["fp32"]) - np.mean(rows["oracle_f64"])) <= 1e-3
    for m in FORMS:
        assert stats[m][0].max() <= 1e-3, (m, stats[m][0])


def test_4k_bf16_against_fp32_and_clean():
    """The 3840x2160 configuration (32 objects, 8 moving, 20% sky, pan U[0,6] px/frame, 2% fireflies x100), every
    frame replayed as one CUDA graph: the BF16 tensor-core form against the FP32 plain form and both against the
    noise-free radiance over 6 frames."""
    cfg = scene.CONFIG_4K
    W, H = cfg.width, cfg.height
    forms = {m: Hush(0, {"width": W, "height": H, "mlp": m, "graph": True}) for m in ("fp32", "bf16")}
    rel = {m: [] for m in forms}
    flick = {m: [] for m in forms}
    diff = []
    prev, prev_clean = {}, None
    for i in range(6):
        fr = scene.frame_device(cfg, i, clean=True)
        outs = {m: g.denoise(fr).float()[..., :3].clone() for m, g in forms.items()}
        torch.cuda.synchronize()
        a, b = outs["bf16"].cpu().numpy(), outs["fp32"].cpu().numpy()
        diff.append((mismatch(a, b)[0], mismatch(a, b, rel=5e-2)[0]))
        if i > 0:
            for m in forms:
                rel[m].append(_clipped_rel(outs[m], fr["clean"]))
                flick[m].append(_flicker(outs[m], prev[m], fr["clean"], prev_clean))
        prev, prev_clean = outs, fr["clean"]
    print(f"\n3840x2160, frames 1..5")
    print("| form | clipped rel-L1 to clean | temporal flicker |")
    print("|---|---|---|")
    for m in forms:
        print(f"| {m} | {np.mean(rel[m]):.4f} | {np.mean(flick[m]):.4f} |")
    print(f"BF16 against FP32: values beyond 2e-3 rel. {np.mean([d[0] for d in diff]):.2e} (mean over frames), "
          f"beyond 5e-2 {np.mean([d[1] for d in diff]):.2e}")
    for g in forms.values():
        assert g.kernel_status() == 0
        g.destroy()
    assert np.mean(rel["bf16"]) <= np.mean(rel["fp32"]) * 1.01
    assert max(d[0] for d in diff) <= 1e-3
