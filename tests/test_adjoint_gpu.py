"""The hand-written adjoint of the training twin on a B200: against the FP64 autograd gradient of the same graph
(oracle/twin.py) and against central finite differences (h = 1e-3) of the CUDA twin itself."""
import numpy as np
import pytest

import oracle
from hush_b200 import Hush, scene
from hush_b200.train import Trainer, xavier_init

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from oracle import twin  # noqa: E402


def _dev(f):
    return {k: torch.from_numpy(np.ascontiguousarray(f[k])).cuda() for k in oracle.INPUTS}


def _setup(W=64, H=48, frames=3, seed=3, theta=None, lambda_t=0.5):
    cfg = scene.SceneConfig(W, H, frames, n_moving=2, pan_min=1.0, pan_max=3.0, seed=seed)
    host = [scene.frame_host(cfg, i, clean=True) for i in range(frames)]
    g = Hush(0, {"width": W, "height": H, "schedule": "passes"})
    tr = Trainer(g, xavier_init(seed) if theta is None else theta)
    cleans = [torch.from_numpy(h["clean"]).cuda() for h in host]
    for t in range(frames - 1):
        tr.frame(_dev(host[t]), cleans[t], cleans[t - 1] if t else None, lambda_t, backward=False)
        tr.end_frame()
    t = frames - 1
    return g, tr, host, cleans, t


def _capture(g, tr, host, t, lambda_t):
    c = g.frame & 1
    st = {k: g.buffer(k).cpu().numpy() for k in ("F0", "F1", "F2", "F3", "A0", "C0", "CG")}
    st["key"] = g.buffer(f"KEY{c}").cpu().numpy()
    st["taa_prev"] = g.buffer(f"TAA{c ^ 1}").cpu().numpy()
    for k, name in (("material", "material"), ("emission", "emission"), ("motion", "motion")):
        st[k] = host[t][name]
    st["clean"] = host[t]["clean"]
    st["clean_prev"] = host[t - 1]["clean"]
    st["reset"] = False
    return st


def test_adjoint_matches_fp64_autograd():
    lam = 0.5
    g, tr, host, cleans, t = _setup(lambda_t=lam)
    tr.zero_grad()
    loss = tr.frame(_dev(host[t]), cleans[t], cleans[t - 1], lam, backward=True)
    torch.cuda.synchronize()
    d_cuda = tr.grad()
    par_c, dpar_c = tr.par()
    st = _capture(g, tr, host, t, lam)
    # the temporal term (lambda > 0) is covered by the finite-difference test; here lambda = 0 on both sides
    theta = torch.tensor(tr.theta.astype(np.float64), requires_grad=True)
    tr.zero_grad()
    loss0 = tr.frame(_dev(host[t]), cleans[t], None, 0.0, backward=True)
    d_cuda0 = tr.grad()
    lt, parts = twin.twin_loss(st, theta, 0.0, return_all=True)
    parts["par_raw"].retain_grad()
    lt.backward()
    d_ref = theta.grad.numpy()
    assert np.isfinite(d_ref).all() and np.isfinite(d_cuda0).all()
    assert abs(loss0 - lt.item()) <= 1e-4 * abs(lt.item()), (loss0, lt.item())
    scale = np.abs(d_ref).max()
    err = np.abs(d_cuda0 - d_ref)
    assert err.max() <= 1e-3 * scale, (err.max() / scale, np.argmax(err))
    big = np.abs(d_ref) > 0.05 * scale
    rel = err[big] / np.abs(d_ref[big])
    assert rel.max() <= 1e-2, rel.max()
    # parameter gradient (12 per half-res pixel)
    sky = (g.buffer("F3").cpu().numpy()[..., 2].astype(np.float32) < 0)[..., None]
    dpar_ref = np.where(sky, 0.0, parts["par_raw"].grad.numpy())
    _, dpar_c0 = tr.par()
    sp = np.abs(dpar_ref).max()
    assert np.abs(dpar_c0 - dpar_ref).max() <= 2e-3 * sp
    assert np.isfinite(loss) and loss > loss0 * 0.5


def test_adjoint_matches_central_differences():
    lam = 0.5
    g, tr, host, cleans, t = _setup(seed=4, lambda_t=lam)
    tr.zero_grad()
    tr.frame(_dev(host[t]), cleans[t], cleans[t - 1], lam, backward=True)
    d = tr.grad()
    theta0 = tr.theta.copy()
    h = 1e-3
    idx = np.argsort(-np.abs(d))[:12]
    fd = []
    for i in idx:
        tp, tm_ = theta0.copy(), theta0.copy()
        tp[i] += h
        tm_[i] -= h
        tr.theta = tp
        lp = tr.frame(_dev(host[t]), cleans[t], cleans[t - 1], lam, backward=False)
        tr.theta = tm_
        lm = tr.frame(_dev(host[t]), cleans[t], cleans[t - 1], lam, backward=False)
        fd.append((lp - lm) / (2 * h))
    tr.theta = theta0
    fd = np.array(fd)
    rel = np.abs(fd - d[idx]) / np.abs(d[idx])
    # FP32 forward: the loss differences carry ~1e-7 relative rounding, so the largest gradients agree to ~1e-3
    assert np.median(rel) <= 1e-2 and rel.max() <= 5e-2, (rel, fd, d[idx])


def test_fp64_reference_matches_its_own_finite_differences():
    g, tr, host, cleans, t = _setup(W=32, H=24, seed=5)
    tr.frame(_dev(host[t]), cleans[t], None, 0.0, backward=False)
    st = _capture(g, tr, host, t, 0.0)
    theta = torch.tensor(tr.theta.astype(np.float64), requires_grad=True)
    lt = twin.twin_loss(st, theta)
    lt.backward()
    gref = theta.grad.numpy()
    h = 1e-3
    for i in np.argsort(-np.abs(gref))[:6]:
        tp, tm_ = theta.detach().clone(), theta.detach().clone()
        tp[i] += h
        tm_[i] -= h
        fd = (twin.twin_loss(st, tp).item() - twin.twin_loss(st, tm_).item()) / (2 * h)
        assert abs(fd - gref[i]) <= 1e-3 * abs(gref[i]) + 1e-9, (i, fd, gref[i])


def test_training_steps_reduce_the_loss():
    from hush_b200.train import TrainConfig, train

    cfg = TrainConfig(size=64, frames=4, seeds=8, batch=2, steps=60, lr=1e-3, lambda_t=0.25)
    tr, hush, hist = train(cfg)
    first = np.mean([h["loss"] for h in hist[:10]])
    last = np.mean([h["loss"] for h in hist[-10:]])
    assert np.isfinite(last) and last < first, (first, last)
    blob = tr.export()
    assert blob.dtype == np.uint16 and blob.size == 812 and hush.hidden == 16


def test_accumulator_views_alias_the_device_gradient():
    """The device views used by data-parallel training read and write the trainer's own accumulators."""
    g, tr, host, cleans, t = _setup()
    tr.zero_grad()
    tr.loss_sum()  # restart the loss sum (the set-up frames added theirs)
    loss = tr.frame(_dev(host[t]), cleans[t], cleans[t - 1], 0.5, backward=True)
    grad, loss_acc = tr.accumulators()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(grad.cpu().numpy(), tr.grad())
    assert loss_acc.item() == pytest.approx(loss, rel=1e-12)
    grad.mul_(0.5)  # what the all-reduce mean does in place with one rank contributing half
    torch.cuda.synchronize()
    np.testing.assert_array_equal(tr.grad(), grad.cpu().numpy())
    assert tr.loss_sum() == pytest.approx(loss, rel=1e-12)
    assert loss_acc.item() == 0.0


def test_native_windows_match_the_per_frame_loop():
    """hush_trainer_windows (generation and frames on the device, windows on concurrent lanes, each window's frames
    replayed as a CUDA graph) accumulates the same loss and gradient as the per-frame loop over the same generated
    windows. Batches of three windows of three frames: the first two batches capture each lane's graphs for both
    frame parities, the third replays them; a one-window batch runs on the caller's stream."""
    from hush_b200.train import TrainConfig, window, window_scene

    cfg = TrainConfig(size=64, frames=3)
    theta = xavier_init(9)
    a = Trainer(Hush(0, {"width": 64, "height": 64, "schedule": "passes"}), theta)
    b = Trainer(Hush(0, {"width": 64, "height": 64, "schedule": "passes"}), theta)

    def loop(seeds):
        b.zero_grad()
        b.loss_sum()
        for s in seeds:
            win = window(cfg, s)
            b.reset()
            for t, fr in enumerate(win):
                b.frame(fr, fr["clean"], win[t - 1]["clean"] if t else None, 0.5, backward=True, sync=False)
                b.end_frame()
        return b.loss_sum(), b.grad()

    for seeds in ([11, 12, 13], [14, 15, 16], [17, 18, 19], [20]):
        a.zero_grad()
        a.loss_sum()
        a.windows(window_scene(cfg), seeds, cfg.frames, 0.5)
        la, ga = a.loss_sum(), a.grad()
        lb, gb = loop(seeds)
        assert la == pytest.approx(lb, rel=1e-12), seeds
        assert np.abs(ga - gb).max() <= 1e-5 * np.abs(gb).max(), seeds
        assert np.abs(gb).max() > 0
