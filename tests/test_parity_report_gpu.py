"""Parity report on a B200 (pytest -s prints the tables it asserts on): every pass of the pass-by-pass schedule
started from the CPU oracle's exact state, at 640 x 360 and 1920 x 1080, and the fused frame over a short sequence
at 1920 x 1080 (3 moving objects, pan U[0,4] px/frame). Per output image: the fraction of values bit-identical to the
oracle's (both stored as f16), the fraction beyond the 2e-3 per-channel bound, and the largest scaled error."""
import numpy as np
import pytest

import oracle
from hush_b200 import Hush, builtin_weights, scene

from .test_parity_gpu import PASS_FRAC, PASS_OUTPUTS, SEQ_FRAC, _dev, _download, _upload
from .util import mismatch, to_f32

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _row(name, got, ref):
    same = float(np.mean(got.astype(np.float16).view(np.uint16) == ref.astype(np.float16).view(np.uint16)))
    frac, worst, _ = mismatch(got.astype(np.float32), ref.astype(np.float32))
    print(f"| {name} | {same:.5f} | {frac:.2e} | {worst:.2e} |")
    return frac


@pytest.mark.parametrize("size", [(640, 360), (1920, 1080)])
def test_pass_parity_report(size):
    W, H = size
    cfg = scene.SceneConfig(W, H, 4, n_moving=3, pan_min=0.0, pan_max=4.0, seed=77)
    frames = [scene.frame_host(cfg, i) for i in range(cfg.frames)]
    o = oracle.OracleHush(W, H, builtin_weights())
    for f in frames[:3]:
        o.denoise(f)
    g = Hush(0, {"width": W, "height": H, "schedule": "passes"})
    for _ in range(3):
        g.end_frame()
    f = frames[3]
    fd = _dev(f)
    c = o.frame & 1
    print(f"\n{W} x {H}, frame 3, each pass from the oracle's state")
    print("| pass / output | bit-identical | beyond 2e-3 | worst scaled error |")
    print("|---|---|---|---|")
    worst_frac = 0.0
    for p in oracle.PASS_NAMES:
        _upload(o, g)
        o.run_pass(p, f)
        g.run_pass(p, fd)
        torch.cuda.synchronize()
        for name in PASS_OUTPUTS[p]:
            name = name.format(c=c)
            worst_frac = max(worst_frac, _row(f"{p} / {name}", _download(g, name), o.buffer(name)))
    g.destroy()
    assert worst_frac <= PASS_FRAC


def test_fused_sequence_parity_report_1080p():
    cfg = scene.SceneConfig(1920, 1080, 5, n_moving=3, pan_min=0.0, pan_max=4.0, seed=78)
    o = oracle.OracleHush(cfg.width, cfg.height, builtin_weights())
    g = Hush(0, {"width": cfg.width, "height": cfg.height})
    print("\n1920 x 1080, fused schedule against the oracle, each side on its own history")
    print("| frame | bit-identical | beyond 2e-3 | worst scaled error |")
    print("|---|---|---|---|")
    fracs = []
    for i in range(cfg.frames):
        f = scene.frame_host(cfg, i)
        ref = o.denoise(f)
        got = to_f32(g.denoise(_dev(f)))
        fracs.append(_row(str(i), got, ref.astype(np.float32)))
    g.destroy()
    assert max(fracs) <= SEQ_FRAC
