"""TEMPORAL's adjoint and backpropagation through time over a window, through the C ABI on a B200.

* hush_temporal_fwd / hush_temporal_bwd: the forward against the float64 restatement of pixel() (oracle/twin.temporal)
  on the same stored history, the adjoint (dA0, dMOM -> the previous frame's colour history, moments, alpha / gamma)
  against that restatement's autograd vector-Jacobian product (whose own central differences tests/test_twin_cpu.py
  checks).
* the fine adjoint's input gradient dA0 and its history seed dA1 against the float64 fine level.
* hush_trainer_window_bptt: the weight gradient of a 4-frame window against the float64 window loss with the same
  gradient paths (oracle/twin.window_loss); the alpha / gamma heads (rows 0-1 of W3 and b3), which the per-frame
  (truncated) gradient leaves at zero, get their gradient through time.
"""
import numpy as np
import pytest

import oracle
from hush_b200 import Hush, scene
from hush_b200.train import Trainer, xavier_init

from .test_passes_gpu import Frame

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from oracle import twin  # noqa: E402

W3o, B3o = 608, 800
AG_IDX = list(range(W3o, W3o + 32)) + [B3o, B3o + 1]  # the weights that feed alpha and gamma only


def _f64(t):
    return torch.tensor(np.asarray(t, np.float32).astype(np.float64))


def _frac_beyond(got, ref, rel=1e-3):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    scale = max(np.abs(ref).max(), 1e-30)
    return float(np.mean(np.abs(got - ref) > rel * scale)), float(np.abs(got - ref).max() / scale)


@pytest.fixture(scope="module")
def frame():
    return Frame()


def _prev_state(fr):
    c = fr.g.frame & 1
    return {k: fr.g.buffer(f"{k}{c ^ 1}").cpu().numpy() for k in ("KEY", "HIST", "MOM")} | {
        "PAR0": fr.g.buffer(f"PAR0_{c ^ 1}").cpu().numpy()}


def _st(fr, prev):
    st = {k: fr.host[2][k] for k in ("radiance", "normalDepth", "motion", "material")}
    st["key_prev"] = prev["KEY"]
    return st


def test_temporal_forward_matches_fp64(frame):
    fr = frame
    prev = _prev_state(fr)
    fr.tr.fwd("temporal")
    torch.cuda.synchronize()
    A0t, momt = twin.temporal(_st(fr, prev), _f64(prev["HIST"]), _f64(prev["MOM"]), _f64(prev["PAR0"]))
    c = fr.g.frame & 1
    for got, ref in ((fr.g.buffer("A0").float().cpu().numpy(), A0t.numpy()),
                     (fr.g.buffer(f"MOM{c}").float().cpu().numpy(), momt.numpy())):
        rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-2 * np.abs(ref).mean())
        assert np.mean(rel <= 2e-3) > 0.995, np.mean(rel <= 2e-3)


def test_temporal_adjoint_matches_fp64_vjp(frame):
    fr = frame
    prev = _prev_state(fr)
    gen = torch.Generator().manual_seed(5)
    sA = torch.randn(fr.b("DA0").shape, generator=gen, dtype=torch.float64)
    sM = torch.randn(fr.b("DMOM").shape, generator=gen, dtype=torch.float64)
    fr.tr.zero_adjoints()
    fr.b("DA0").copy_(sA.float().cuda())
    fr.b("DMOM").copy_(sM.float().cuda())
    fr.tr.bwd("temporal")
    torch.cuda.synchronize()
    ins = [_f64(prev["HIST"]).requires_grad_(True), _f64(prev["MOM"]).requires_grad_(True),
           _f64(prev["PAR0"]).requires_grad_(True)]
    A0, mom = twin.temporal(_st(fr, prev), *ins)
    ref = torch.autograd.grad((sA * A0).sum() + (sM * mom).sum(), ins)
    got = {"DHIST": fr.b("DHIST").double().cpu(), "DMOM_PREV": fr.b("DMOM_PREV").double().cpu(),
           "DAG": fr.b("DAG").double().cpu()}
    pairs = [("DHIST", got["DHIST"][..., :3], ref[0][..., :3]), ("DMOM_PREV", got["DMOM_PREV"], ref[1]),
             ("DAG", got["DAG"], ref[2][..., :2])]
    for name, g, r in pairs:
        assert r.abs().max().item() > 0, name
        frac, worst = _frac_beyond(g.numpy(), r.numpy())
        print(f"temporal adjoint {name}: {frac:.2e} of entries beyond 1e-3 of the largest, worst {worst:.2e}")
        # a pixel whose key test or history threshold falls on the other side in FP32 takes another branch
        assert frac <= 2e-3 and worst <= 5e-2, (name, frac, worst)
    # in the sum over the image those branch flips are a small part
    for name, g, r in pairs:
        assert abs(g.sum().item() - r.sum().item()) <= 1e-3 * r.abs().sum().item(), name


def test_fine_adjoint_input_and_history_seed_match_fp64(frame):
    fr = frame
    gen = torch.Generator().manual_seed(6)
    sX = torch.randn(fr.b("DX").shape, generator=gen, dtype=torch.float64)
    sX[..., 3] = 0.0
    sH = torch.randn(fr.b("DA1").shape, generator=gen, dtype=torch.float64)
    fr.tr.zero_adjoints()
    fr.b("DX").copy_(sX.float().cuda())
    fr.b("DA1").copy_(sH.float().cuda())
    fr.tr.bwd("fine")
    torch.cuda.synchronize()
    got = fr.b("DA0").double().cpu()
    A0 = _f64(fr.st["A0"]).requires_grad_(True)
    par, b3 = fr.f64("PAR"), fr.f64("B3")
    A1, X = twin.fine(fr.st, par, b3, fr.Gh, fr.sky_h, fr.Ah, A0=A0)
    sky = _f64(fr.st["key"])[..., 2] < 0
    A1 = torch.where(sky[..., None], torch.zeros_like(A1), A1)
    (ref,) = torch.autograd.grad((sX[..., :3] * X).sum() + (sH * A1).sum(), [A0])
    frac, worst = _frac_beyond(got.numpy(), ref.numpy())
    print(f"fine adjoint dA0: {frac:.2e} beyond 1e-3 of the largest, worst {worst:.2e}")
    assert worst <= 1e-3, worst


def _window(W=64, H=48, n=4, seed=11):
    cfg = scene.SceneConfig(W, H, n, n_moving=2, pan_min=1.0, pan_max=3.0, seed=seed)
    frames = []
    for i in range(n):
        h = scene.frame_host(cfg, i, clean=True)
        d = {k: torch.from_numpy(np.ascontiguousarray(h[k])).cuda() for k in oracle.INPUTS}
        d["clean"] = torch.from_numpy(h["clean"]).cuda()
        frames.append((h, d))
    return frames


def test_window_bptt_matches_the_fp64_window_gradient():
    W, H, lam = 64, 48, 0.5
    frames = _window(W, H)
    g = Hush(0, {"width": W, "height": H, "schedule": "passes"})
    tr = Trainer(g, xavier_init(11))
    # the window's forward frame by frame, keeping each frame's state for the float64 reference
    tr.reset()
    states = []
    tr.zero_grad()
    for i, (h, d) in enumerate(frames):
        tr.frame(d, d["clean"], frames[i - 1][1]["clean"] if i else None, lam, backward=True)
        torch.cuda.synchronize()
        c = g.frame & 1
        st = {k: g.buffer(k).cpu().numpy() for k in ("F0", "F1", "F2", "F3", "A0", "C0", "C1", "CG")}
        st.update({"key": g.buffer(f"KEY{c}").cpu().numpy(), "key_prev": g.buffer(f"KEY{c ^ 1}").cpu().numpy(),
                   "mom": g.buffer(f"MOM{c}").cpu().numpy(), "hist": g.buffer(f"HIST{c}").cpu().numpy(),
                   "par0": g.buffer(f"PAR0_{c}").cpu().numpy(), "taa_prev": g.buffer(f"TAA{c ^ 1}").cpu().numpy(),
                   "out_prev": tr.buffer("OUT_PREV").cpu().numpy() if i else None, "reset": i == 0})
        for k in ("radiance", "normalDepth", "motion", "material", "emission"):
            st[k] = h[k]
        st["clean"] = h["clean"]
        st["clean_prev"] = frames[i - 1][0]["clean"] if i else None
        states.append(st)
        tr.end_frame()
    truncated = tr.grad()
    # the same window through time on the device
    tr.zero_grad()
    tr.window_bptt([d for _, d in frames], lam)
    torch.cuda.synchronize()
    got = tr.grad()
    theta = torch.tensor(tr.theta.astype(np.float64), requires_grad=True)
    (ref,) = torch.autograd.grad(twin.window_loss(states, theta, lam), [theta])
    ref = ref.numpy()
    scale = np.abs(ref).max()
    err = np.abs(got - ref)
    print(f"window BPTT: max |cuda - fp64| / max |fp64| = {err.max() / scale:.2e}; alpha/gamma rows: "
          f"cuda {np.abs(got[AG_IDX]).max():.3e}, fp64 {np.abs(ref[AG_IDX]).max():.3e}, "
          f"truncated {np.abs(truncated[AG_IDX]).max():.3e}")
    assert err.max() <= 1e-3 * scale, err.max() / scale
    # the alpha / gamma heads: no gradient frame by frame, a gradient through time that matches the reference
    assert np.abs(truncated[AG_IDX]).max() == 0.0
    ag = np.abs(ref[AG_IDX]).max()
    assert ag > 1e-6 * scale
    assert np.abs(got[AG_IDX] - ref[AG_IDX]).max() <= 1e-2 * ag
    # away from alpha / gamma, the through-time gradient adds to the per-frame one
    assert not np.allclose(got, truncated)
    tr.destroy()
    g.destroy()


def test_native_windows_through_time_match_the_window_calls():
    """hush_trainer_windows_bptt (generation on the device, windows on concurrent lanes, each window's forward and
    reverse sweep replayed as a CUDA graph) accumulates the same loss and gradient as hush_trainer_window_bptt called
    window by window on the same generated windows, in both MLP forms (the loss to 1e-12, the gradient to 1e-5 of its
    largest value). Batches of three windows of three frames: the
    first batch captures each lane's graph, the next ones replay it; a one-window batch runs on the caller's stream.
    The alpha / gamma heads get their gradient through time on this path too."""
    from hush_b200.train import TrainConfig, window, window_scene

    cfg = TrainConfig(size=64, frames=3)
    theta = xavier_init(9)
    a = Trainer(Hush(0, {"width": 64, "height": 64, "schedule": "passes"}), theta)
    b = Trainer(Hush(0, {"width": 64, "height": 64, "schedule": "passes"}), theta)

    def calls(seeds):
        b.zero_grad()
        b.loss_sum()
        for s in seeds:
            b.window_bptt(window(cfg, s), 0.5)
        return b.loss_sum(), b.grad()

    for mlp in ("fp32", "bf16"):
        a.set_mlp(mlp)
        b.set_mlp(mlp)
        for seeds in ([11, 12, 13], [14, 15, 16], [17, 18, 19], [20]):
            a.zero_grad()
            a.loss_sum()
            a.windows_bptt(window_scene(cfg), seeds, cfg.frames, 0.5)
            la, ga = a.loss_sum(), a.grad()
            lb, gb = calls(seeds)
            assert la == pytest.approx(lb, rel=1e-12), (mlp, seeds)
            # the adjoints' FP32 atomics add in a different order: differences at FP32 rounding level, carried
            # through the frames of the window
            assert np.abs(ga - gb).max() <= 1e-5 * np.abs(gb).max(), (mlp, seeds)
            assert np.abs(ga[AG_IDX]).max() > 1e-6 * np.abs(ga).max(), (mlp, seeds)
    a.destroy()
    b.destroy()
