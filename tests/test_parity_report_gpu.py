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


def _key_margins(nd, mv, key_prev):
    """The history tests TEMPORAL applies per pixel (hush.js:103-105, 149-187), evaluated in float64 from the stored
    values, with how close each comes to its threshold: over the bilinear footprint at p + mv (taps with weight > 0
    inside the image) and the 3x3 fallback around the nearest pixel, whether any tap's depth test (|z - zPrev| against
    0.05 zPrev + 0.01, relative margin) or normal test (n . n_prev against 0.9) lies within `eps` of its threshold,
    and whether the bilinear weight sum of the passing taps lies within 1e-6 of the 0.01 cut. The object-id test is
    an exact comparison of integers stored in f16 and has no margin. Also returns the decision itself (a surface pixel
    takes history when the passing bilinear taps weigh at least 0.01 or a fallback tap passes)."""
    from oracle import twin

    eps = 1e-4
    H, W = nd.shape[:2]
    ys, xs = np.mgrid[0:H, 0:W]
    n = nd[..., :3].astype(np.float64)
    ppx = xs.astype(np.float32) + mv[..., 0].astype(np.float32)
    ppy = ys.astype(np.float32) + mv[..., 1].astype(np.float32)
    bx, by = np.floor(ppx), np.floor(ppy)
    fx, fy = (ppx - bx).astype(np.float32), (ppy - by).astype(np.float32)
    kn = twin.oct_dec(torch.from_numpy(key_prev[..., 0].astype(np.float64)),
                      torch.from_numpy(key_prev[..., 1].astype(np.float64))).numpy()
    zp, obj = mv[..., 3].astype(np.float64), mv[..., 2]
    tol = 0.05 * zp + 0.01

    def tap(qx, qy):
        inside = (qx >= 0) & (qy >= 0) & (qx < W) & (qy < H)
        cx, cy = np.clip(qx, 0, W - 1).astype(np.int64), np.clip(qy, 0, H - 1).astype(np.int64)
        k = key_prev[cy, cx].astype(np.float64)
        cand = inside & (k[..., 2] >= 0) & (k[..., 3] == obj)
        mz = (tol - np.abs(k[..., 2] - zp)) / tol
        mn = (kn[cy, cx] * n).sum(-1) - 0.9
        ok = cand & (mz >= 0) & (mn >= 0)
        return ok, cand & (np.abs(mz) < eps), cand & (mz >= 0) & (np.abs(mn) < eps)

    sum_w = np.zeros((H, W))
    near_z = np.zeros((H, W), bool)
    near_n = np.zeros((H, W), bool)
    for i in range(4):
        w = ((fx if i & 1 else 1 - fx) * (fy if i >> 1 else 1 - fy)).astype(np.float32)
        ok, z, nn = tap(bx + (i & 1), by + (i >> 1))
        sum_w += np.where(ok & (w > 0), w, 0.0)
        near_z |= z & (w > 0)
        near_n |= nn & (w > 0)
    cxn, cyn = np.floor(ppx + np.float32(0.5)), np.floor(ppy + np.float32(0.5))
    fb = sum_w < 0.01
    n_fb = np.zeros((H, W), np.int64)
    for j in range(9):
        ok, z, nn = tap(cxn + j % 3 - 1, cyn + j // 3 - 1)
        n_fb += ok
        near_z |= z & fb
        near_n |= nn & fb
    near_w = np.abs(sum_w - 0.01) < 1e-6
    has = (nd[..., 3] >= 0) & (~fb | (n_fb > 0))
    return has, near_z, near_n, near_w


@pytest.mark.parametrize("size", [(640, 360), (1920, 1080)])
def test_temporal_branch_flip_report(size):
    """TEMPORAL's history decision per pixel (hush.js:149-190: history taken or not; a pixel with history stores a
    length above 1, one without stores 1, sky 0), CUDA against the oracle from the oracle's exact state (frame 3 of
    the seeded sequence): the pixels whose decision flips, each attributed to the test that sits at its threshold
    (key-test depth tolerance, the 0.9 normal threshold, the 0.01 bilinear weight-sum cut; object-id equality is exact
    and cannot flip), and the A0 values beyond the bound over all pixels and over the pixels without a flip. Every
    flip must sit at a threshold (a last-ulp difference of the two f32 evaluations), not come from different
    arithmetic."""
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
    c = o.frame & 1
    key_prev = o.buffer(f"KEY{c ^ 1}").astype(np.float32)
    _upload(o, g)
    o.run_pass("temporal", f)
    g.run_pass("temporal", _dev(f))
    torch.cuda.synchronize()
    mom_o, mom_g = o.buffer(f"MOM{c}").astype(np.float32), _download(g, f"MOM{c}")
    has_o, has_g = mom_o[..., 3] > 1.0, mom_g[..., 3] > 1.0
    flip = has_o != has_g
    has64, near_z, near_n, near_w = _key_margins(f["normalDepth"].astype(np.float32),
                                                 f["motion"].astype(np.float32), key_prev)
    near = near_z | near_n | near_w
    # the float64 restatement of the decisions agrees with the oracle's away from the thresholds
    assert not np.any((has64 != has_o) & ~near)
    at_z, at_n, at_w = int((flip & near_z).sum()), int((flip & near_n).sum()), int((flip & near_w).sum())
    unexplained = int((flip & ~near).sum())
    a0_o, a0_g = o.buffer("A0").astype(np.float32), _download(g, "A0")
    frac_all, _, _ = mismatch(a0_g, a0_o)
    keep = ~flip
    frac_kept, _, _ = mismatch(a0_g[keep], a0_o[keep])
    n_flip = int(flip.sum())
    print(f"\n{W} x {H}, frame 3, TEMPORAL from the oracle's state: history decisions")
    print("| pixels | with history (oracle) | decision flips | at the depth tolerance | at the 0.9 normal threshold "
          "| at the 0.01 weight sum | elsewhere | A0 beyond 2e-3, all pixels | A0 beyond 2e-3, pixels without a flip |")
    print("|---|---|---|---|---|---|---|---|---|")
    print(f"| {W * H} | {int(has_o.sum())} | {n_flip} | {at_z} | {at_n} | {at_w} | {unexplained} | {frac_all:.2e} "
          f"| {frac_kept:.2e} |")
    g.destroy()
    assert unexplained == 0
    assert n_flip <= 1e-4 * W * H
    assert frac_kept <= PASS_FRAC
