"""On-device training of the parameter MLP through the hand-written adjoint kernels (hush_trainer_* in include/hush.h).

The reference's weights were trained offline by a PyTorch copy of its passes that is not shipped (README.md:137,
src/denoise/hush.js:6-7). Here the frames come from the synthetic scene generator on the device, the target is the
noise-free image, the loss is relative L1 of the TAA output plus a temporal-gradient term, and Adam updates FP32
master weights; the result exports to the reference's f16 blob format (W1 b1 W2 b2 W3 b3, hush.js:20-21).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .dp import DataParallel, finish_step
from .hush import Hush, HushError, _DevView, _fill_inputs, _stream_handle
from .scene import SceneConfig, frame_device

NW = 812


def xavier_init(seed: int = 0) -> np.ndarray:
    """Xavier-uniform weights and zero biases of the 20-16-16-12 network in the blob layout."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NW, np.float32)

    def xav(n_out, n_in):
        b = np.sqrt(6.0 / (n_in + n_out))
        return rng.uniform(-b, b, n_out * n_in).astype(np.float32)

    w[0:320] = xav(16, 20)
    w[336:592] = xav(16, 16)
    w[608:800] = xav(12, 16)
    return w


class Trainer:
    """Training twin bound to one Hush instance (FP32 master weights, Adam state, gradient accumulator)."""

    def __init__(self, hush: Hush, theta: np.ndarray | None = None):
        self.hush = hush
        self._theta = None if theta is None else np.ascontiguousarray(theta, np.float32)
        h = C.c_void_p()
        rc = L.lib().hush_trainer_create(hush._h, self._theta.ctypes.data if self._theta is not None else None,
                                         C.byref(h))
        if rc != L.HUSH_OK:
            raise HushError(L.lib().hush_last_error(hush._h).decode())
        self._t = h
        self._inp = L.HushInputs()

    def _check(self, rc):
        if rc != L.HUSH_OK:
            raise HushError(L.lib().hush_last_error(self.hush._h).decode())

    def frame(self, inputs: dict, clean, clean_prev=None, lambda_t: float = 0.0, backward: bool = True,
              stream=None, sync: bool = True):
        """One frame: forward, loss and (if backward) the gradient added to the accumulator. Does not advance.
        Returns the loss (synchronising) or None with sync=False (the loss is summed on the device)."""
        _fill_inputs(self._inp, inputs)
        loss = C.c_double()
        self._check(L.lib().hush_trainer_frame(self._t, C.byref(self._inp), clean.data_ptr(),
                                               clean_prev.data_ptr() if clean_prev is not None else None,
                                               float(lambda_t), 1 if backward else 0,
                                               C.c_void_p(_stream_handle(stream)), C.byref(loss) if sync else None))
        return loss.value if sync else None

    def set_mlp(self, mlp: str):
        """The twin's MLP arithmetic: "fp32" (per-thread FP32) or "bf16" / "f16" (tensor-core GEMM tiles)."""
        self._check(L.lib().hush_trainer_set_mlp(self._t, {"fp32": L.MLP_FP32, "bf16": L.MLP_BF16,
                                                           "f16": L.MLP_F16}[mlp]))

    def windows(self, scene_cfg: SceneConfig, seeds, n_frames: int, lambda_t: float = 0.0, stream=None):
        """hush_trainer_windows: for each seed, the n_frames frames of scene_cfg with that seed generated on the
        device and run forward + backward (history reset per window); gradient and loss accumulate, no step."""
        sc = scene_cfg.c()
        arr = (C.c_uint32 * len(seeds))(*[int(x) & 0xFFFFFFFF for x in seeds])
        self._check(L.lib().hush_trainer_windows(self._t, C.byref(sc), arr, len(seeds), int(n_frames),
                                                 float(lambda_t), C.c_void_p(_stream_handle(stream))))

    def windows_bptt(self, scene_cfg: SceneConfig, seeds, n_frames: int, lambda_t: float = 0.0, stream=None):
        """hush_trainer_windows_bptt: for each seed, the n_frames frames of scene_cfg with that seed generated on the
        device and run forward and backward through time (window_bptt) on concurrent lanes, each window replayed as a
        CUDA graph; gradient and loss accumulate, no step."""
        sc = scene_cfg.c()
        arr = (C.c_uint32 * len(seeds))(*[int(x) & 0xFFFFFFFF for x in seeds])
        self._check(L.lib().hush_trainer_windows_bptt(self._t, C.byref(sc), arr, len(seeds), int(n_frames),
                                                      float(lambda_t), C.c_void_p(_stream_handle(stream))))

    def loss_sum(self, stream=None) -> float:
        """Sum of the frame losses since the previous call."""
        v = C.c_double()
        self._check(L.lib().hush_trainer_loss_sum(self._t, C.c_void_p(_stream_handle(stream)), C.byref(v)))
        return v.value

    def end_frame(self):
        self._check(L.lib().hush_trainer_end_frame(self._t))

    def reset(self):
        self._check(L.lib().hush_trainer_reset(self._t))

    def zero_grad(self, stream=None):
        self._check(L.lib().hush_trainer_zero_grad(self._t, C.c_void_p(_stream_handle(stream))))

    def grad(self) -> np.ndarray:
        g = np.zeros(NW, np.float64)
        self._check(L.lib().hush_trainer_grad(self._t, g.ctypes.data))
        return g

    def accumulators(self):
        """(grad, loss_sum): torch views of the device gradient accumulator (812 float64) and loss sum (1 float64)."""
        import torch

        g, l = C.c_void_p(), C.c_void_p()
        self._check(L.lib().hush_trainer_accumulators(self._t, C.byref(g), C.byref(l)))
        dev = torch.device("cuda", self.hush.device)
        return (torch.as_tensor(_DevView(g.value, 1, 1, NW, "<f8"), device=dev).view(NW),
                torch.as_tensor(_DevView(l.value, 1, 1, 1, "<f8"), device=dev).view(1))

    @property
    def theta(self) -> np.ndarray:
        t = np.zeros(NW, np.float32)
        self._check(L.lib().hush_trainer_theta(self._t, t.ctypes.data, None))
        return t

    @theta.setter
    def theta(self, v):
        v = np.ascontiguousarray(v, np.float32)
        self._check(L.lib().hush_trainer_theta(self._t, None, v.ctypes.data))

    def par(self):
        """(par, dpar): (h, w, 12) FP32 parameters of the last frame and their gradient."""
        H2, W2 = (self.hush.height + 1) // 2, (self.hush.width + 1) // 2
        p = np.zeros((H2, W2, 12), np.float32)
        d = np.zeros((H2, W2, 12), np.float32)
        self._check(L.lib().hush_trainer_par(self._t, p.ctypes.data, d.ctypes.data))
        return p, d

    def output(self) -> np.ndarray:
        o = np.zeros((self.hush.height, self.hush.width, 4), np.float32)
        self._check(L.lib().hush_trainer_output(self._t, o.ctypes.data))
        return o

    def step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, clip=1.0, stream=None) -> float:
        n = C.c_double()
        self._check(L.lib().hush_trainer_step(self._t, lr, beta1, beta2, eps, clip,
                                              C.c_void_p(_stream_handle(stream)), C.byref(n)))
        return n.value

    def export(self) -> np.ndarray:
        b = np.zeros(NW, np.uint16)
        self._check(L.lib().hush_trainer_export(self._t, b.ctypes.data))
        return b

    # ---- the passes as forward / adjoint pairs (hush_trainer_begin, hush_<pass>_fwd / _bwd) ----
    def begin(self, inputs: dict, clean, clean_prev=None, lambda_t: float = 0.0, stream=None):
        """TEMPORAL and the coarse levels for the frame; fixes the frame for fwd() / bwd(). The tensors must stay
        alive until the frame's last pass call."""
        _fill_inputs(self._inp, inputs)
        self._begun = (inputs, clean, clean_prev)
        self._check(L.lib().hush_trainer_begin(self._t, C.byref(self._inp), clean.data_ptr(),
                                               clean_prev.data_ptr() if clean_prev is not None else None,
                                               float(lambda_t), C.c_void_p(_stream_handle(stream))))

    def fwd(self, name: str, stream=None):
        """Forward of one pass ("mlp", "mid1", "mid2", "mid3", "fine", "taa", "loss", "temporal", "coarse1",
        "coarse2")."""
        self._check(getattr(L.lib(), f"hush_{name}_fwd")(self._t, C.c_void_p(_stream_handle(stream))))

    def bwd(self, name: str, stream=None):
        """Adjoint of one pass: adds into the gradients of its inputs (the loss adjoint sets dOUT)."""
        self._check(getattr(L.lib(), f"hush_{name}_bwd")(self._t, C.c_void_p(_stream_handle(stream))))

    def zero_adjoints(self, stream=None):
        self._check(L.lib().hush_trainer_zero_adjoints(self._t, C.c_void_p(_stream_handle(stream))))

    def buffer(self, name: str):
        """Torch view of a trainer buffer (hush_trainer_buf): THETA / GRAD (812,), LOSS (1,), PAR / DPAR (h, w, 12),
        B1..B3 / DB1..DB3 (h, w, 4), A1 / X / DX / OUT / OUT_PREV / DOUT (H, W, 4), AH / DAH (h, w, 4), C1 / DC1 /
        C0 / DC0 (quarter resolution, 4 channels)."""
        import torch

        ptr, w, h, c = C.c_void_p(), C.c_int(), C.c_int(), C.c_int()
        self._check(L.lib().hush_trainer_buffer(self._t, L.TWIN_BUF_NAMES.index(name), C.byref(ptr), C.byref(w),
                                                C.byref(h), C.byref(c)))
        ts = "<f8" if name in ("GRAD", "LOSS") else "<f4"
        v = torch.as_tensor(_DevView(ptr.value, h.value, w.value, c.value, ts),
                            device=torch.device("cuda", self.hush.device))
        return v.view(-1) if h.value == 1 and c.value == 1 else v

    def window_bptt(self, window, lambda_t: float = 0.5, stream=None):
        """hush_trainer_window_bptt: backpropagation through time over one window, a list of input dicts each with a
        "clean" (H, W, 3) float32 CUDA tensor. Adds into the gradient and loss accumulators (no optimiser step)."""
        n = len(window)
        ins = (L.HushInputs * n)()
        cl = (C.c_void_p * n)()
        for i, fr in enumerate(window):
            _fill_inputs(ins[i], fr)
            cl[i] = fr["clean"].data_ptr()
        self._check(L.lib().hush_trainer_window_bptt(self._t, ins, cl, n, float(lambda_t),
                                                     C.c_void_p(_stream_handle(stream))))

    def train_step(self, windows, lambda_t=0.5, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, clip=1.0, stream=None):
        """hush_train_step over a batch: windows = list of windows, each a list of input dicts with a "clean" (H, W, 3)
        float32 CUDA tensor. Returns (mean frame loss, gradient norm)."""
        nw, nf = len(windows), len(windows[0])
        if any(len(w) != nf for w in windows):
            raise HushError("train_step: windows must have the same number of frames")
        ins = (L.HushInputs * (nw * nf))()
        cl = (C.c_void_p * (nw * nf))()
        for i, fr in enumerate(f for w in windows for f in w):
            _fill_inputs(ins[i], fr)
            cl[i] = fr["clean"].data_ptr()
        loss, gn = C.c_double(), C.c_double()
        self._check(L.lib().hush_train_step(self._t, ins, cl, nw, nf, float(lambda_t), lr, beta1, beta2, eps, clip,
                                            C.c_void_p(_stream_handle(stream)), C.byref(loss), C.byref(gn)))
        return loss.value, gn.value

    def destroy(self):
        if getattr(self, "_t", None) and self._t.value:
            L.lib().hush_trainer_destroy(self._t)
            self._t = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.destroy()
        except Exception:
            pass


# W3 rows 0-1 and b3[0:2] in the weight blob (W1 b1 W2 b2 W3 b3, hush.js:20-21): the alpha and gamma heads' weights
AG_IDX = list(range(608, 640)) + [800, 801]


@dataclass
class TrainConfig:
    """The training workload: windows of `frames` frames at `size`^2 from `seeds` generator seeds."""
    size: int = 384
    frames: int = 8
    seeds: int = 2048
    batch: int = 16
    steps: int = 5000
    lr: float = 1e-3
    lambda_t: float = 0.5
    clip: float = 1.0
    init_seed: int = 0
    mlp: str = "fp32"  # the twin's MLP: "fp32", or "bf16" / "f16" tensor-core tiles
    bptt: bool = False  # gradient through time over each window (hush_trainer_window_bptt): alpha / gamma train


def window_scene(cfg: TrainConfig, seed: int = 0) -> SceneConfig:
    """The generator configuration of a training window: 3 independently moving objects, pan U[0,4] px/frame."""
    return SceneConfig(cfg.size, cfg.size, cfg.frames, seed=seed, pan_min=0.0, pan_max=4.0, n_moving=3)


def window(cfg: TrainConfig, seed: int, buf=None):
    """One training window generated on the device: list of (inputs, clean) for `frames` frames."""
    sc = window_scene(cfg, seed)
    out = []
    for t in range(cfg.frames):
        out.append(frame_device(sc, t, out=None if buf is None else buf[t], clean=True))
    return out


def train(cfg: TrainConfig, log_every: int = 100, on_log=None, time_budget_s: float | None = None,
          dp: DataParallel | None = None, device: int = 0):
    """Runs the training loop; returns (trainer, hush, history). A step = `batch` windows of `frames` frames on each
    rank; with dp (one process per GPU) the ranks draw disjoint window seeds and average gradient and loss before
    the shared Adam step, so the global batch is batch x world windows."""
    import torch

    dp = dp or DataParallel()
    hush = Hush(device, {"width": cfg.size, "height": cfg.size, "schedule": "passes"})
    tr = Trainer(hush, xavier_init(cfg.init_seed))
    tr.set_mlp(cfg.mlp)
    if dp.world > 1:  # every rank starts from rank 0's weights
        th = torch.from_numpy(tr.theta).cuda(device)
        dp.broadcast_(th)
        tr.theta = th.cpu().numpy()
    rng = dp.seed_rng(cfg.init_seed + 1)
    sc = window_scene(cfg)
    hist = []
    t0 = time.time()
    for step in range(cfg.steps):
        ts = time.perf_counter()
        seeds = [dp.window_seed(rng, cfg.seeds) for _ in range(cfg.batch)]
        if cfg.bptt:  # generation + forward + backward through time of every window
            tr.windows_bptt(sc, seeds, cfg.frames, cfg.lambda_t)
        else:
            tr.windows(sc, seeds, cfg.frames, cfg.lambda_t)  # generation + forward + adjoint of every frame
        loss, gn = finish_step(tr, dp, cfg.batch * cfg.frames, cfg.lr, cfg.clip)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - ts) * 1e3
        rec = {"step": step, "loss": loss, "grad_norm": gn, "step_ms": ms}
        hist.append(rec)
        if on_log and (step % log_every == 0 or step == cfg.steps - 1):
            on_log(rec)
        stop = bool(time_budget_s and time.time() - t0 > time_budget_s)
        if dp.world > 1:  # every rank stops at the same step
            flag = torch.tensor([1.0 if stop else 0.0], device=f"cuda:{device}")
            dp.average_(flag)
            stop = flag.item() > 0
        if stop:
            break
    return tr, hush, hist


def evaluate(weights_blob: np.ndarray | None, seeds, size: int = 384, frames: int = 8, svgf: bool = False):
    """Error of the inference path on held-out windows: clipped relative L1 against the noise-free image and temporal
    flicker (clipped relative L1 of frame differences), averaged over frames 1.. of each window. weights_blob = None
    uses the built-in weights; svgf = True runs the SVGF baseline instead."""
    import torch

    from .svgf import SVGF

    cfg = TrainConfig(size=size, frames=frames)
    rel, flick = [], []
    for seed in seeds:
        win = window(cfg, int(seed))
        if svgf:
            den = SVGF(0, size, size)
        else:
            opts = {"width": size, "height": size}
            if weights_blob is not None:
                opts["weights"] = weights_blob.tobytes()
            den = Hush(0, opts)
        prev_out, prev_clean = None, None
        for t, fr in enumerate(win):
            if svgf:
                g = dict(fr)
                g["prevNormalDepth"] = win[t - 1]["normalDepth"] if t else fr["normalDepth"]
                g["prevMotion"] = win[t - 1]["motion"] if t else fr["motion"]
                out = den.encode(g).float()[..., :3]
            else:
                out = den.denoise(fr).float()[..., :3]
            clean = fr["clean"]
            d = clean.abs() + 1e-2
            if t > 0:
                rel.append(torch.clamp((out - clean).abs() / d, max=1.0).mean().item())
                flick.append(torch.clamp(((out - prev_out) - (clean - prev_clean)).abs() / d, max=1.0).mean().item())
            prev_out, prev_clean = out.clone(), clean
        den.destroy()
    return {"rel_l1": float(np.mean(rel)), "flicker": float(np.mean(flick)), "windows": len(seeds)}


def main(argv=None):
    """Command line. Under torchrun (WORLD_SIZE > 1) it trains data-parallel over NCCL, one GPU per rank; rank 0
    evaluates and writes the outputs."""
    import argparse
    import datetime
    import json
    import os

    import torch
    import torch.distributed as dist

    ap = argparse.ArgumentParser(description="train the parameter MLP on device and evaluate against SVGF")
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--batch", type=int, default=16, help="windows per step on each rank")
    ap.add_argument("--size", type=int, default=384)
    ap.add_argument("--frames", type=int, default=8)
    ap.add_argument("--seeds", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--mlp", default="fp32", choices=["fp32", "bf16", "f16"], help="the twin's MLP arithmetic")
    ap.add_argument("--bptt", action="store_true",
                    help="backpropagate through time over each window (the alpha / gamma heads train)")
    ap.add_argument("--time-budget", type=float, default=None, help="stop after this many seconds of training")
    ap.add_argument("--eval-seeds", type=int, default=64)
    ap.add_argument("--out", default=None, help="write the summary JSON here")
    ap.add_argument("--weights-out", default=None, help="write the trained f16 blob here")
    a = ap.parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dp = DataParallel()
    cfg = TrainConfig(size=a.size, frames=a.frames, seeds=a.seeds, batch=a.batch, steps=a.steps, lr=a.lr, mlp=a.mlp,
                      bptt=a.bptt)
    log = []

    def on_log(rec):
        log.append(rec)
        if dp.rank == 0:
            print(json.dumps(rec), flush=True)

    tr, hush, hist = train(cfg, log_every=50, on_log=on_log, time_budget_s=a.time_budget, dp=dp, device=local)
    blob = tr.export()
    div = dp.max_divergence(torch.from_numpy(tr.theta).cuda(local))
    if dp.rank != 0:
        tr.destroy()
        hush.destroy()
        dist.destroy_process_group()
        return 0
    if a.weights_out:
        blob.tofile(a.weights_out)
    held_out = [1_000_000 + i for i in range(a.eval_seeds)]
    res = {
        "config": vars(a),
        "world": dp.world,
        "steps_run": len(hist),
        "theta_max_divergence_over_ranks": div,
        "train_step_ms_median": float(np.median([h["step_ms"] for h in hist[1:]] or [hist[0]["step_ms"]])),
        "loss_first": hist[0]["loss"], "loss_last": float(np.mean([h["loss"] for h in hist[-20:]])),
        "eval_trained": evaluate(blob, held_out, a.size, a.frames),
        "eval_builtin": evaluate(None, held_out, a.size, a.frames),
        "eval_svgf": evaluate(None, held_out, a.size, a.frames, svgf=True),
        # the weights that feed only alpha and gamma (rows 0-1 of W3 and b3): they move only with --bptt
        "alpha_gamma_weights_max_change": float(np.abs(tr.theta[AG_IDX] - xavier_init(cfg.init_seed)[AG_IDX]).max()),
        "log": log,
    }
    print(json.dumps({k: v for k, v in res.items() if k != "log"}), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    if dp.world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    import sys

    sys.exit(main())
