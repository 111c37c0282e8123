"""Each pass of the training twin, the coarse levels included, as a forward / adjoint pair through the C ABI
(hush_<pass>_fwd / hush_<pass>_bwd) on a B200: the forward against the FP64 restatement of the same pass
(oracle/twin.py) at the pass's own inputs, the adjoint against that restatement's FP64 autograd vector-Jacobian
product and against central finite differences (h = 1e-3) of the CUDA forward, and the chain of adjoints against the
fused frame's gradient."""
import ctypes as C

import numpy as np
import pytest

import oracle
from hush_b200 import Hush, HushError, scene
from hush_b200 import _lib as L
from hush_b200.train import Trainer, xavier_init

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from oracle import twin  # noqa: E402

ORDER = ["mlp", "mid1", "mid2", "mid3", "fine", "taa", "loss"]
COARSE = ["coarse1", "coarse2"]  # the coarse levels: no learnable input; their adjoints carry the input-level gradient
H_FD = 1e-3
# COARSE1's input (the block means) enters through down()'s 2x2 weighted means, so its gradients are a fraction of
# the level's and the FP32 rounding of the forward over +-1e-3 dominates its differences: the coarse passes take a
# step of 1e-2 for the differences of the CUDA forward (the FP64 differences keep 1e-3)
H_FD_CUDA = {"coarse1": 1e-2, "coarse2": 1e-2}


def _dev(f):
    return {k: torch.from_numpy(np.ascontiguousarray(f[k])).cuda() for k in oracle.INPUTS}


class Frame:
    """A trainer two frames into a window, with the third frame begun and its forward chain run."""

    def __init__(self, W=64, H=48, seed=3, lam=0.5):
        cfg = scene.SceneConfig(W, H, 3, n_moving=2, pan_min=1.0, pan_max=3.0, seed=seed)
        self.host = [scene.frame_host(cfg, i, clean=True) for i in range(3)]
        self.g = Hush(0, {"width": W, "height": H, "schedule": "passes"})
        self.tr = Trainer(self.g, xavier_init(seed))
        self.cleans = [torch.from_numpy(h["clean"]).cuda() for h in self.host]
        self.lam = lam
        for t in range(2):
            self.tr.frame(_dev(self.host[t]), self.cleans[t], self.cleans[t - 1] if t else None, lam, backward=False)
            self.tr.end_frame()
        self.inputs = _dev(self.host[2])
        self.tr.begin(self.inputs, self.cleans[2], self.cleans[1], lam)
        for p in ORDER + COARSE:
            self.tr.fwd(p)
        torch.cuda.synchronize()
        c = self.g.frame & 1
        st = {k: self.g.buffer(k).cpu().numpy() for k in ("F0", "F1", "F2", "F3", "A0", "C0", "CG")}
        st["key"] = self.g.buffer(f"KEY{c}").cpu().numpy()
        st["taa_prev"] = self.g.buffer(f"TAA{c ^ 1}").cpu().numpy()
        for k in ("material", "emission", "motion"):
            st[k] = self.host[2][k]
        st["clean"] = self.host[2]["clean"]
        st["clean_prev"] = self.host[1]["clean"]
        st["out_prev"] = self.b("OUT_PREV").cpu().numpy()
        st["reset"] = False
        self.st = st
        self.feats, self.Gh, self.sky_h, self.Ah = twin.half_inputs(st)
        self.cnt_h = twin.unpack_half(st["F3"])[..., 3]  # the blocks' pixel counts (down()'s weights)
        self.Gq = twin.coarse_guide(st["CG"])

    def b(self, name):
        return self.tr.buffer(name)

    def f64(self, name, rgb=False):
        v = self.b(name).double().cpu()
        return (v[..., :3] if rgb else v).clone().requires_grad_(True)


# per pass: (output buffer, seed buffer, channels of the output that carry the seed, {input buffer: gradient buffer})
SPEC = {
    "mlp": ("PAR", "DPAR", 12, {"THETA": "GRAD"}),
    "mid1": ("B1", "DB1", 4, {"PAR": "DPAR"}),
    "mid2": ("B2", "DB2", 4, {"B1": "DB1", "PAR": "DPAR"}),
    "mid3": ("B3", "DB3", 4, {"B2": "DB2", "PAR": "DPAR"}),
    "fine": ("X", "DX", 3, {"B3": "DB3", "PAR": "DPAR"}),
    "taa": ("OUT", "DOUT", 3, {"X": "DX"}),
    "loss": ("LOSS", None, 1, {"OUT": "DOUT"}),
    "coarse1": ("C1", "DC1", 4, {"AH": "DAH"}),
    "coarse2": ("C0", "DC0", 4, {"C1": "DC1"}),
}
# PAR components each pass reads (alpha gamma beta kappa | s0..s3 | c0..c3)
PAR_USED = {"mid1": (5, 9), "mid2": (6, 10), "mid3": (7, 11), "fine": (2, 3, 4, 8)}


def _seed(fr, name, gen):
    out, seed, ch, _ = SPEC[name]
    if seed is None:
        return None
    s = fr.b(seed)
    z = torch.randn(s.shape, generator=gen, dtype=torch.float64).float()
    if ch < s.shape[-1]:
        z[..., ch:] = 0.0
    return z.cuda()


def _run_bwd(fr, name, seed):
    """Adjoint of one pass from `seed` (written into its seed buffer) with every gradient cleared first."""
    fr.tr.zero_adjoints()
    fr.tr.zero_grad()
    if seed is not None:
        fr.b(SPEC[name][1]).copy_(seed)
    fr.tr.bwd(name)
    torch.cuda.synchronize()
    return {g: fr.b(g).double().cpu().clone() for g in SPEC[name][3].values()}


def _objective(fr, name, seed):
    """<seed, pass output> in FP64 (the loss itself for the loss pass)."""
    out = fr.b(SPEC[name][0]).double()
    return out.sum().item() if seed is None else (seed.double() * out).sum().item()


def _reference(fr, name, seed):
    """FP64 forward of the pass at the CUDA pass's own inputs and its vector-Jacobian product with the seed."""
    if name == "mlp":
        th = fr.f64("THETA")
        _, y = twin.mlp(fr.feats, th, fr.sky_h)
        ins = {"THETA": th}
    elif name.startswith("mid"):
        k = int(name[-1])
        par = fr.f64("PAR")
        src = fr.Ah if k == 1 else fr.f64(f"B{k - 1}")
        y = twin.mid(k, src, fr.Gh, fr.sky_h, par)
        ins = {"PAR": par} if k == 1 else {f"B{k - 1}": src, "PAR": par}
    elif name == "fine":
        par, b3 = fr.f64("PAR"), fr.f64("B3")
        _, y = twin.fine(fr.st, par, b3, fr.Gh, fr.sky_h, fr.Ah)
        ins = {"B3": b3, "PAR": par}
    elif name == "coarse1":
        ah = fr.f64("AH")
        y = twin.coarse1(ah, fr.cnt_h, fr.Gq)
        ins = {"AH": ah}
    elif name == "coarse2":
        c1 = fr.f64("C1")
        y = twin.coarse2(c1, fr.Gq)
        ins = {"C1": c1}
    elif name == "taa":
        x = fr.f64("X", rgb=True)
        y = twin.taa(fr.st, x)
        ins = {"X": x}
    else:
        o = fr.f64("OUT", rgb=True)
        y = twin.loss_of(fr.st, o, fr.lam)
        ins = {"OUT": o}
    s = y.sum() if seed is None else (seed.double().cpu()[..., :y.shape[-1]] * y).sum()
    grads = torch.autograd.grad(s, list(ins.values()))
    return y.detach(), dict(zip(ins, grads))


def _as_full(gref, like):
    """An FP64 gradient of rgb-only inputs padded to the buffer's 4 channels."""
    if gref.shape == like.shape:
        return gref
    pad = torch.zeros(like.shape, dtype=torch.float64)
    pad[..., :gref.shape[-1]] = gref
    return pad


@pytest.fixture(scope="module")
def frame():
    return Frame()


@pytest.mark.parametrize("name", ORDER + COARSE)
def test_pass_forward_matches_fp64(frame, name):
    seed = _seed(frame, name, torch.Generator().manual_seed(1))
    frame.tr.fwd(name)
    torch.cuda.synchronize()
    y_ref, _ = _reference(frame, name, seed)
    y = frame.b(SPEC[name][0]).double().cpu()
    y = y[..., :y_ref.shape[-1]] if y_ref.dim() else y.reshape(())
    err = (y - y_ref).abs()
    scale = y_ref.abs().max().item()
    # FP32 arithmetic against FP64 on identical inputs
    assert err.max().item() <= 1e-4 * max(scale, 1e-6), (name, err.max().item(), scale)


@pytest.mark.parametrize("name", ORDER + COARSE)
def test_pass_adjoint_matches_fp64_vjp(frame, name):
    seed = _seed(frame, name, torch.Generator().manual_seed(2))
    got = _run_bwd(frame, name, seed)
    _, ref = _reference(frame, name, seed)
    for inp, gname in SPEC[name][3].items():
        g = got[gname]
        r = _as_full(ref[inp], g)
        if inp == "PAR":  # this pass's components only (the others belong to other passes and stay zero)
            used = list(PAR_USED[name])
            assert g[..., [c for c in range(12) if c not in used]].abs().max().item() == 0.0
            g, r = g[..., used], r[..., used]
        if gname == "GRAD":
            g, r = g.view(-1), r.view(-1)
        scale = r.abs().max().item()
        assert scale > 0, (name, inp)
        err = (g - r).abs()
        print(f"{name} d{inp}: max |cuda - fp64| / max |fp64| = {err.max().item() / scale:.2e}")
        assert err.max().item() <= 1e-3 * scale, (name, inp, err.max().item() / scale)


@pytest.mark.parametrize("name", ORDER + COARSE)
def test_pass_adjoint_matches_central_differences(frame, name):
    seed = _seed(frame, name, torch.Generator().manual_seed(3))
    got = _run_bwd(frame, name, seed)
    rng = np.random.default_rng(4)
    frame.tr.fwd(name)
    s0 = _objective(frame, name, seed)
    rels, kinks = [], 0
    for inp, gname in SPEC[name][3].items():
        g = got[gname].reshape(-1)
        if inp == "PAR":
            mask = torch.zeros(got[gname].shape, dtype=torch.bool)
            mask[..., list(PAR_USED[name])] = True
            g = torch.where(mask.reshape(-1), g, torch.zeros_like(g))
        if inp in ("X", "OUT"):  # the rgb channels only (alpha is a constant)
            mask = torch.zeros(got[gname].shape, dtype=torch.bool)
            mask[..., :3] = True
            g = torch.where(mask.reshape(-1), g, torch.zeros_like(g))
        top = torch.argsort(-g.abs())[:8].numpy()
        nz = torch.nonzero(g.abs() > 1e-3 * g.abs().max()).view(-1).numpy()
        pick = np.unique(np.concatenate([top, rng.choice(nz, size=min(16, nz.size), replace=False)]))
        buf = frame.b(inp).view(-1)
        h_fd = H_FD_CUDA.get(name, H_FD)
        for i in pick:
            v0 = buf[i].item()
            buf[i] = v0 + h_fd
            vp = buf[i].item()  # the FP32 value actually stored
            frame.tr.fwd(name)
            sp = _objective(frame, name, seed)
            buf[i] = v0 - h_fd
            vm = buf[i].item()
            frame.tr.fwd(name)
            sm = _objective(frame, name, seed)
            buf[i] = v0
            # a central difference is only meaningful where the pass is differentiable across [v - h, v + h]: where
            # the two one-sided differences disagree, the interval holds a kink (a clip of the loss, the TAA box or
            # the heads, a relu, |x| at 0) and the entry is skipped
            up, down = (sp - s0) / (vp - v0), (s0 - sm) / (v0 - vm)
            if abs(up - down) > 0.05 * max(abs(up), abs(down)):
                kinks += 1
                continue
            fd = (sp - sm) / (vp - vm)
            rels.append(abs(fd - g[i].item()) / abs(g[i].item()))
    frame.tr.fwd(name)  # restore the pass's output
    rels = np.array(rels)
    print(f"{name}: {rels.size} entries, {kinks} across a kink, relative error median {np.median(rels):.2e} "
          f"max {rels.max():.2e}")
    assert rels.size >= 8 and kinks <= rels.size, (name, rels.size, kinks)
    # FP32 outputs: the differences carry ~1e-7 relative rounding over h = 1e-3
    assert np.median(rels) <= 1e-3 and np.mean(rels <= 1e-2) >= 0.9, (name, np.sort(rels))


def test_chain_of_pass_adjoints_is_the_frame_gradient():
    fr = Frame(seed=5)
    tr = fr.tr
    tr.zero_adjoints()
    tr.zero_grad()
    for p in reversed(ORDER):
        tr.bwd(p)
    torch.cuda.synchronize()
    g_chain = tr.grad()
    _, dpar_chain = tr.par()
    tr.zero_grad()
    tr.frame(fr.inputs, fr.cleans[2], fr.cleans[1], fr.lam, backward=True)
    g_frame = tr.grad()
    _, dpar_frame = tr.par()
    # same kernels; only the order of the atomic additions differs
    assert np.abs(g_chain - g_frame).max() <= 1e-5 * np.abs(g_frame).max()
    assert np.abs(dpar_chain - dpar_frame).max() <= 1e-5 * np.abs(dpar_frame).max()


def test_pass_calls_check_their_arguments():
    g = Hush(0, {"width": 32, "height": 24, "schedule": "passes"})
    tr = Trainer(g, xavier_init(0))
    with pytest.raises(HushError, match="hush_trainer_begin first"):
        tr.fwd("mlp")
    assert L.lib().hush_trainer_pass(tr._t, len(L.TWIN_PASSES), 0, None) == L.HUSH_ERR_ARG
    assert L.lib().hush_trainer_pass(tr._t, -1, 1, None) == L.HUSH_ERR_ARG
    p = C.c_void_p()
    assert L.lib().hush_trainer_buffer(tr._t, len(L.TWIN_BUF_NAMES), C.byref(p), None, None, None) == L.HUSH_ERR_ARG
    cfg = scene.SceneConfig(32, 24, 1, seed=1)
    f = scene.frame_host(cfg, 0, clean=True)
    clean = torch.from_numpy(f["clean"]).cuda()
    tr.begin(_dev(f), clean)
    tr.fwd("mlp")
    tr.end_frame()
    with pytest.raises(HushError, match="hush_trainer_begin first"):
        tr.bwd("mlp")
    g.resize(48, 32)
    with pytest.raises(HushError, match="resized"):
        tr.begin(_dev(f), clean)


def test_train_step_is_the_training_loop():
    W, H, nw, nf = 48, 32, 2, 3
    wins = []
    for s in range(nw):
        cfg = scene.SceneConfig(W, H, nf, n_moving=1, seed=20 + s)
        win = []
        for i in range(nf):
            f = scene.frame_host(cfg, i, clean=True)
            d = _dev(f)
            d["clean"] = torch.from_numpy(f["clean"]).cuda()
            win.append(d)
        wins.append(win)
    theta = xavier_init(7)
    a = Trainer(Hush(0, {"width": W, "height": H, "schedule": "passes"}), theta)
    loss_a, gn_a = a.train_step(wins, lambda_t=0.5, lr=1e-3, clip=1.0)
    b = Trainer(Hush(0, {"width": W, "height": H, "schedule": "passes"}), theta)
    for win in wins:
        b.reset()
        for i, fr in enumerate(win):
            b.frame(fr, fr["clean"], win[i - 1]["clean"] if i else None, 0.5, backward=True, sync=False)
            b.end_frame()
    loss_b = b.loss_sum() / (nw * nf)
    gn_b = b.step(1e-3, clip=1.0)
    assert loss_a == pytest.approx(loss_b, rel=1e-12)
    assert gn_a == pytest.approx(gn_b, rel=1e-5)
    # the gradients differ only in the order of atomic additions; Adam's first step moves each weight by about
    # lr * sign(g), so a weight whose gradient is rounding noise may step the other way
    d = np.abs(a.theta - b.theta)
    assert np.mean(d <= 1e-6) >= 0.99 and d.max() <= 2.1e-3, (np.mean(d <= 1e-6), d.max())
    assert not np.array_equal(a.theta, theta)


@pytest.mark.parametrize("name", ORDER + COARSE)
def test_pass_adjoint_matches_fp64_central_differences(frame, name):
    """The CUDA adjoint of each pass against central differences (h = 1e-3) of the same pass evaluated in FP64 at the
    CUDA pass's inputs: free of the FP32 rounding of the forward. Every entry whose +-h interval is smooth agrees to
    1e-3 relative where the entry is at least 1e-2 of the largest gradient; smaller entries, whose FP32 accumulation
    over the rows can cancel, to 1e-5 of the largest gradient in absolute terms."""
    seed = _seed(frame, name, torch.Generator().manual_seed(5))
    got = _run_bwd(frame, name, seed)
    sd = None if seed is None else seed.double().cpu()

    def objective(inputs):
        with torch.no_grad():
            if name == "mlp":
                _, y = twin.mlp(frame.feats, inputs["THETA"], frame.sky_h)
            elif name.startswith("mid"):
                k = int(name[-1])
                src = frame.Ah if k == 1 else inputs[f"B{k - 1}"]
                y = twin.mid(k, src, frame.Gh, frame.sky_h, inputs["PAR"])
            elif name == "fine":
                _, y = twin.fine(frame.st, inputs["PAR"], inputs["B3"], frame.Gh, frame.sky_h, frame.Ah)
            elif name == "taa":
                y = twin.taa(frame.st, inputs["X"][..., :3])
            elif name == "coarse1":
                y = twin.coarse1(inputs["AH"], frame.cnt_h, frame.Gq)
            elif name == "coarse2":
                y = twin.coarse2(inputs["C1"], frame.Gq)
            else:
                y = twin.loss_of(frame.st, inputs["OUT"][..., :3], frame.lam)
            return y.sum().item() if sd is None else (sd[..., :y.shape[-1]] * y).sum().item()

    def mlp_pattern(theta):
        """The MLP's piecewise-linear switches over the non-sky rows: both ReLU masks and the heads' clamps. A weight
        perturbation that flips any of them crosses a kink in one row of many, which the one-sided test misses."""
        w = theta
        live = ~frame.sky_h
        x = frame.feats[live]
        a1 = x @ w[twin.W1o:twin.B1o].view(16, 20).T + w[twin.B1o:twin.W2o]
        h1 = torch.relu(a1)
        a2 = h1 @ w[twin.W2o:twin.B2o].view(16, 16).T + w[twin.B2o:twin.W3o]
        o = torch.relu(a2) @ w[twin.W3o:twin.B3o].view(12, 16).T + w[twin.B3o:twin.B3o + 12]
        return torch.cat([a1 > 0, a2 > 0, o[:, 4:8].abs() < 5, o[:, 8:12].abs() < 4], 1)

    base = {inp: frame.b(inp).double().cpu().clone() for inp in SPEC[name][3]}
    rng = np.random.default_rng(6)
    rels, kinks = [], 0
    f0 = objective(base)
    for inp, gname in SPEC[name][3].items():
        g = got[gname].reshape(-1)
        gmax = g.abs().max().item()
        if inp == "PAR":
            mask = torch.zeros(got[gname].shape, dtype=torch.bool)
            mask[..., list(PAR_USED[name])] = True
            g = torch.where(mask.reshape(-1), g, torch.zeros_like(g))
        if inp in ("X", "OUT"):
            mask = torch.zeros(got[gname].shape, dtype=torch.bool)
            mask[..., :3] = True
            g = torch.where(mask.reshape(-1), g, torch.zeros_like(g))
        top = torch.argsort(-g.abs())[:16].numpy()
        nz = torch.nonzero(g.abs() > 1e-3 * g.abs().max()).view(-1).numpy()
        pick = np.unique(np.concatenate([top, rng.choice(nz, size=min(16, nz.size), replace=False)]))
        for i in pick:
            xs = {k: v.clone() for k, v in base.items()}
            flat = xs[inp].view(-1)
            v0 = flat[i].item()
            flat[i] = v0 + H_FD
            fp = objective(xs)
            flat[i] = v0 - H_FD
            fm = objective(xs)
            up, down = (fp - f0) / H_FD, (f0 - fm) / H_FD
            switched = False
            if name == "mlp":
                with torch.no_grad():
                    p0 = mlp_pattern(base["THETA"])
                    for dv in (H_FD, -H_FD):
                        t = base["THETA"].clone()
                        t[i] += dv
                        switched |= bool((mlp_pattern(t) != p0).any())
            if switched or abs(up - down) > 0.05 * max(abs(up), abs(down)):
                kinks += 1
                continue
            fd = (fp - fm) / (2 * H_FD)
            gi = g[i].item()
            # the error in units of the bound: 1e-3 of the entry, or 1e-5 of the largest gradient for small entries
            bound = 1e-3 * abs(gi) if abs(gi) >= 1e-2 * gmax else 1e-5 * gmax
            rels.append((abs(fd - gi) / abs(gi), abs(fd - gi) / bound))
    rels = np.array(rels)
    print(f"{name}: {len(rels)} entries against FP64 differences, {kinks} across a kink, relative error median "
          f"{np.median(rels[:, 0]):.2e} max {rels[:, 0].max():.2e}, worst / bound {rels[:, 1].max():.2f}")
    assert len(rels) >= 8, (name, len(rels), kinks)
    assert rels[:, 1].max() <= 1.0, (name, rels)
