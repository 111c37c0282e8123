"""Benchmark of the Hush denoise path on synthetic 1080p G-buffer sequences.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mlp fp32|bf16|f16]
                    [--no-graph] [--workload 1080p|4k]

A step is one denoised 1920x1080 frame of the seeded 64-frame sequence (3 independently moving objects, camera pan
U[0,4] px/frame with 0.2 deg/frame yaw, a camera cut and reset() at frame 32); longer runs loop over the sequence
with a reset() at every restart. Each frame is replayed as one CUDA graph (re-captured and updated in place when
the input buffers change; --no-graph launches the eight kernels directly). Inputs are generated on the device
before timing, so the timed region starts with them resident in HBM; every frame reads its own 83 MB of inputs plus
~230 MB of state, more than the 126 MB L2, so no L2 flush is needed between frames. --workload 4k runs the 3840x2160
workload instead (BF16 MLP, one graph per frame).

Prints one JSON line (rank 0). For N > 1 every rank denoises its own independent sequence on its own GPU (replicas:
the path has no cross-GPU exchange); value = max-over-ranks time / total frames. `--gpus N` under torchrun uses its
ranks; without one, bench.py starts the N ranks itself through torch.distributed.run.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1080p ms/frame + %HBM roofline, BF16-MLP vs FP32 plain; train-step ms at equal error"
W, H, SEQ = 1920, 1080, 64
WORKLOAD = "1920x1080 64-frame sequence, 3 moving objects, pan U[0,4] px/frame, cut at 32 (reset)"
L2_NOTE = "no flush: each frame reads 83 MB of fresh inputs + ~230 MB of state (> 126 MB L2)"


def _config(mlp: str, world: int) -> dict:
    """The workload as both arms print it (implementation details such as the schedule go in "setup")."""
    return {"workload": WORKLOAD, "width": W, "height": H, "mlp": mlp, "l2": L2_NOTE,
            "parallelism": f"replicas x{world}"}


def _scene_cfg():
    from hush_b200 import scene

    return scene.CONFIG_1080P if W == 1920 else scene.CONFIG_4K

# Algorithmic bytes per launch of each fused stage at this build's formats (8 B per rgba16float texel), per
# full-res pixel (P), half-res pixel (h) and quarter-res pixel (q): unique global reads + writes.
STAGE_BYTES = {
    # unique global bytes per launch at this build's formats: P full, h half, q quarter pixels
    "temporal+mlp": lambda P, h, q: P * (32 + 24 + 24) + h * (8 + 56),  # rad nd mv mat; key hist mom gathers; A0 mom
                                                                        # key | prev par0; par0..2 Ah Gh Gd
    "mid1+coarse1": lambda P, h, q: h * (40 + 8 + 8) + q * 32,           # Ah Gd par1 par2 -> Bh0, Gh | -> C1 CG CGd
    "mid2+coarse2": lambda P, h, q: h * (40 + 8) + q * 32,               # Bh0 Gd par1 par2 -> Bh1 | C1 CGd -> C0
    "mid3": lambda P, h, q: h * (40 + 8),                                # Bh1 Gd par1 par2 -> Bh0
    "fine+final": lambda P, h, q: P * (32 + 16) + h * 56 + q * 24,       # A0 key mat emi -> hist X | Gd Ah Bh0 par0..2
                                                                        # | CGd C0
    "taa": lambda P, h, q: P * 32,                                       # X motion prevTaa -> taa
}


def _env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary (profiles/traffic.json)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return {}
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # wait for the first sample so that the timed region is covered from its start
            t0 = time.time()
            while time.time() - t0 < 5 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def _cpu_baseline_sample(frames: int = 3):
    """The oracle (f32 restatement of the reference's passes, OpenMP over rows) on frames of the bench's sequence:
    ms/frame over the frames after the first, all host threads."""
    import numpy as np  # noqa: F401

    import oracle

    oracle.set_threads(0)
    cores = os.cpu_count() or 1
    cfg = _scene_cfg()
    o = oracle.OracleHush(W, H, oracle.builtin_weights())
    times = []
    for i in range(frames):
        f = oracle.scene_frame(cfg, i)
        t = time.perf_counter()
        o.denoise(f)
        times.append(time.perf_counter() - t)
    ms = 1000.0 * statistics.mean(times[1:] if len(times) > 1 else times)
    return {"value": round(ms, 3), "unit": "ms/frame", "cores": cores, "kind": "port",
            "sample": f"{frames} frames of the {W}x{H} sequence (frame 0 untimed), oracle f32, {cores} threads",
            "per_pass_ms": _cpu_per_pass_sizes()}


def _cpu_per_pass_sizes():
    out = {}
    for w, h in ((W, H), (640, 360)):
        try:
            out[f"{w}x{h}"] = _cpu_per_pass(w, h)
        except Exception as e:  # pragma: no cover - reported, not fatal
            out[f"{w}x{h}"] = f"failed: {e}"
    return out


def _cpu_per_pass(w, h, warm=2, timed=5):
    """The oracle's passes one by one (f32, all host threads): the median ms per pass over `timed` frames of the
    sequence at w x h after `warm` frames."""
    import oracle

    cfg = _scene_cfg().with_(width=w, height=h, frames=warm + timed, cut_frame=-1)
    o = oracle.OracleHush(w, h, oracle.builtin_weights())
    per = {p: [] for p in oracle.PASS_NAMES}
    for i in range(warm + timed):
        f = oracle.scene_frame(cfg, i)
        for p in oracle.PASS_NAMES:
            t = time.perf_counter()
            o.run_pass(p, f)
            if i >= warm:
                per[p].append(1000.0 * (time.perf_counter() - t))
        o.end_frame()
    return {p: round(statistics.median(v), 3) for p, v in per.items()}


def run_reference(args):
    rank, _, world = _env_rank()
    if rank != 0:
        return 0
    import oracle  # the CPU arm loads only the oracle library: frames, weights and passes all come from it

    oracle.set_threads(0)
    cores = os.cpu_count() or 1
    cfg = _scene_cfg()
    o = oracle.OracleHush(W, H, oracle.builtin_weights())
    # bounded sample: the CPU takes ~0.3 s per 1080p frame, so at most 2 warm-up and 24 timed frames
    warm, steps = min(args.warmup, 2), min(args.steps, 24)
    n = warm + steps
    frames = {}
    times = []
    for i in range(n):
        k = i % SEQ
        if k not in frames:
            frames[k] = oracle.scene_frame(cfg, k)
        if k == 32 or (k == 0 and i > 0):
            o.reset()
        t = time.perf_counter()
        o.denoise(frames[k])
        if i >= warm:
            times.append(time.perf_counter() - t)
        if len(frames) > 4:
            frames.pop(min(frames))
    ms = 1000.0 * sum(times) / max(len(times), 1)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(ms, 3), "unit": "ms/frame", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": _config(args.mlp, world),
        "setup": {"inputs": "generated on the host by the oracle library before each frame's timing",
                  "arithmetic": "f32 oracle, OpenMP over rows"},
        "cpu_baseline": {"value": round(ms, 3), "unit": "ms/frame", "cores": cores, "kind": "port",
                         "sample": f"{steps} full {W}x{H} frames of the sequence after {warm} warm-up frames; the "
                                   "reference's WGSL cannot run here (no WebGPU / Dawn / node), its scalar "
                                   "restatement (oracle/) stands in"},
        "e2e": {"value": round(ms, 3), "unit": "ms/frame", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    from hush_b200 import Hush, scene

    rank, local, world = _env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    cfg = _scene_cfg().with_(seed=1 + rank)
    nseq = min(SEQ, args.warmup + args.steps)
    # the sequence, generated on the device (untimed)
    frames = [scene.frame_device(cfg, i) for i in range(nseq)]
    torch.cuda.synchronize()
    hush = Hush(local, {"width": W, "height": H, "mlp": args.mlp, "schedule": args.schedule,
                        "graph": args.graph})
    stream = torch.cuda.current_stream()

    def step(i):
        k = i % nseq
        if k == 32 or (k == 0 and i > 0):
            hush.reset()
        return hush.denoise(frames[k], stream=stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world > 1:
            t = torch.tensor([x], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    # ---- headline: device-resident inputs
    for i in range(args.warmup):
        step(i)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for i in range(args.warmup, args.warmup + args.steps):
            step(i)
        e1.record(stream)
        barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1))
    ms_frame = ms_total / args.steps
    clocks = clk.summary()

    # ---- per-kernel breakdown: the same frames with CUDA events between the stages
    stage_ms = {}
    hush_timer_frames = min(args.steps, 16)
    from hush_b200 import HushTimer

    for i in range(args.warmup + args.steps, args.warmup + args.steps + hush_timer_frames):
        k = i % nseq
        if k == 32 or k == 0:
            hush.reset()
        t = HushTimer()
        hush.denoise(frames[k], timer=t, stream=stream)
        for label, ms in t.last:
            stage_ms.setdefault(label, []).append(ms)
    stage_avg = {k: statistics.mean(v) for k, v in stage_ms.items()}

    # ---- end to end through the public API with host buffers: Hush.denoise_host copies the five pinned host inputs
    # in and the output back every step (the copies of adjacent frames overlap the kernels)
    host = []
    for k in range(min(nseq, 8)):
        host.append({n: frames[k][n].cpu().pin_memory() for n in scene.NAMES})
    outs = [torch.empty((H, W, 4), dtype=torch.float16).pin_memory() for _ in range(2)]
    hush.reset()
    e2e_steps = min(args.steps, 32)
    for i in range(3):
        hush.denoise_host(host[i % len(host)], outs[i & 1], stream=stream)
    hush.host_join(stream)
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for i in range(e2e_steps):
        hush.denoise_host(host[i % len(host)], outs[i & 1], stream=stream)
    hush.host_join(stream)
    f1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1)) / e2e_steps
    h2d = sum(host[0][n].numel() * 2 for n in scene.NAMES)
    d2h = outs[0].numel() * 2
    # the PCIe bound of e2e: the same five pinned input copies alone, back to back on one stream (CUDA events)
    staging = {n: torch.empty_like(frames[0][n]) for n in scene.NAMES}
    for _ in range(3):
        for n in scene.NAMES:
            staging[n].copy_(host[0][n], non_blocking=True)
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    for i in range(10):
        for n in scene.NAMES:
            staging[n].copy_(host[i % len(host)][n], non_blocking=True)
    c1.record(stream)
    torch.cuda.synchronize()
    h2d_peak_gbs = h2d * 10 / (c0.elapsed_time(c1) * 1e-3) / 1e9
    del staging

    # ---- the other MLP form on the same frames, device-resident inputs (BF16 tensor-core MLP vs FP32 plain MLP)
    alt = "bf16" if args.mlp != "bf16" else "fp32"
    hush_alt = Hush(local, {"width": W, "height": H, "mlp": alt, "schedule": args.schedule, "graph": args.graph})
    n_alt = min(args.steps, 512)

    def step_alt(i):
        k = i % nseq
        if k == 32 or (k == 0 and i > 0):
            hush_alt.reset()
        return hush_alt.denoise(frames[k], stream=stream)

    for i in range(args.warmup):
        step_alt(i)
    barrier()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for i in range(args.warmup, args.warmup + n_alt):
        step_alt(i)
    g1.record(stream)
    barrier()
    alt_ms = max_over_ranks(g0.elapsed_time(g1)) / n_alt
    hush_alt.destroy()

    # ---- one training step of the parameter MLP (data-parallel over the ranks when N > 1)
    train_ms = None
    if not args.no_train:  # the BF16 tensor-core form (the training configuration's), the FP32 form beside it
        train_ms = _train_step_ms(local, stream, barrier, max_over_ranks, mlp="bf16")
        train_ms["fp32_step_ms"] = _train_step_ms(local, stream, barrier, max_over_ranks, mlp="fp32")["step_ms"]
        # backpropagation through time over each window (alpha / gamma heads trained), one window after another
        train_ms["bptt_step_ms"] = _train_step_ms(local, stream, barrier, max_over_ranks, mlp="bf16",
                                                  bptt=True)["step_ms"]

    if rank != 0:
        hush.destroy()
        if world > 1:
            dist.destroy_process_group()
        return 0

    P, h, q = W * H, ((W + 1) // 2) * ((H + 1) // 2), ((W + 3) // 4) * ((H + 3) // 4)
    peak, peak_kind = _peaks()
    per_stage = {}
    for label, ms in stage_avg.items():
        nbytes = STAGE_BYTES[label](P, h, q) if label in STAGE_BYTES else None
        per_stage[label] = {"ms": round(ms, 4),
                            "gbs": round(nbytes / (ms * 1e-3) / 1e9, 1) if nbytes else None,
                            "bytes": nbytes}
    dominant = max(stage_avg, key=stage_avg.get) if stage_avg else None
    tr = _traffic().get(dominant) if dominant else None
    roof = None
    if dominant and dominant in STAGE_BYTES:
        ach = per_stage[dominant]["gbs"]
        roof = {"kernel": dominant, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "peak_source": peak_kind,
                # the captures are of 1920 x 1080 launches; other sizes scale them by the pixels processed (the
                # kernels stream their images, so DRAM bytes grow in proportion)
                "traffic": (round(tr["bytes_per_launch"] * P / (1920 * 1080)) if tr and "bytes_per_launch" in tr
                            else None),
                "traffic_source": (("ncu capture at 1920x1080" if P == 1920 * 1080
                                    else "ncu capture at 1920x1080 scaled by the pixel count") if tr else None),
                "algorithmic_bytes_per_launch": per_stage[dominant]["bytes"]}
    filt_bytes = sum(v["bytes"] for v in per_stage.values() if v["bytes"])
    filt_ms = sum(v["ms"] for v in per_stage.values())
    # the filter passes alone (every stage after TEMPORAL + MLP): their summed bytes over their summed time
    fp = [v for k, v in per_stage.items() if k != "temporal+mlp" and v["bytes"]]
    fp_bytes, fp_ms = sum(v["bytes"] for v in fp), sum(v["ms"] for v in fp)
    n_kernels = 8  # fused: stage 0, mid1-3, COARSE1, coarse2, FINE_FINAL, TAA; passes: the reference's 8 passes
    line = {
        "metric": METRIC, "value": round(ms_frame / world, 4), "unit": "ms/frame", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_frame, 4), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": _config(args.mlp, world),
        "setup": {"inputs": "generated on the device before timing", "schedule": args.schedule,
                  "graph": bool(args.graph)},
        "roofline": roof,
        "frame_hbm": {"bytes_per_frame": filt_bytes, "sum_stage_ms": round(filt_ms, 4),
                      "gbs": round(filt_bytes / (filt_ms * 1e-3) / 1e9, 1) if filt_ms else None,
                      "frac": round(filt_bytes / (filt_ms * 1e-3) / 1e9 / peak, 4) if filt_ms else None,
                      "compulsory_108B_per_px_ms": round(108 * P / (peak * 1e9) * 1e3, 4)},
        "filter_passes": {"stages": [k for k in per_stage if k != "temporal+mlp"], "bytes": fp_bytes,
                          "ms": round(fp_ms, 4),
                          "gbs": round(fp_bytes / (fp_ms * 1e-3) / 1e9, 1) if fp_ms else None,
                          "frac": round(fp_bytes / (fp_ms * 1e-3) / 1e9 / peak, 4) if fp_ms else None},
        "stages": per_stage,
        "clocks": clocks,
        "e2e": {"value": round(e2e_ms / world, 4), "unit": "ms/frame", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                # host -> device rate of the timed e2e steps against the same copies timed alone
                "h2d_gbs": round(h2d / (e2e_ms * 1e-3) / 1e9, 1), "h2d_copy_peak_gbs": round(h2d_peak_gbs, 1)},
        "gpu_launches": n_kernels * args.steps,
        "kernel_status": hush.kernel_status(),  # the error word of the bounded waits after the run (0 = none gave up)
        "mlp_forms": {args.mlp: {"ms_per_frame": round(ms_frame, 4)},
                      alt: {"ms_per_frame": round(alt_ms, 4), "frames": n_alt}},
    }
    if train_ms is not None:
        line["train"] = train_ms
    if not args.no_extras:
        line["extras"] = _extras_ms(frames, stream)
    if not args.no_cpu_baseline and world == 1:  # the CPU baseline is timed on rank 0 of single-GPU runs only
        line["cpu_baseline"] = _cpu_baseline_sample()
    print(json.dumps(line), flush=True)
    hush.destroy()
    if world > 1:
        dist.destroy_process_group()
    return 0


def _extras_ms(frames, stream, n=32, warmup=4):
    """Per-frame device time of the pieces around the denoiser at the workload's size, each timed alone with CUDA
    events on the launching stream: plain SVGF (the fallback and judge, 5 a-trous iterations + TAA) on the same
    frames, the path tracer (1 spp, 3 bounces, the demo scene) and the display post (bloom, vignette, AgX, sRGB into
    an rgba8 target). A failure is reported in place of the time."""
    import torch

    from hush_b200 import SVGF, Post, pt

    H, W = frames[0]["radiance"].shape[:2]
    out = {}

    def timed(step):
        for i in range(warmup):
            step(i)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(n):
            step(warmup + i)
        e1.record(stream)
        torch.cuda.synchronize()
        return round(e0.elapsed_time(e1) / n, 4)

    try:
        sv = SVGF(0, W, H)

        def svgf_step(i):
            k = i % len(frames)
            g = dict(frames[k])
            g["prevNormalDepth"] = frames[k - 1]["normalDepth"] if k else frames[k]["normalDepth"]
            g["prevMotion"] = frames[k - 1]["motion"] if k else frames[k]["motion"]
            sv.encode(g, stream=stream)

        out["svgf_ms_per_frame"] = timed(svgf_step)
        sv.destroy()
    except Exception as e:  # pragma: no cover - reported, not fatal
        out["svgf_ms_per_frame"] = f"failed: {e}"
    try:
        sc, env, mover = pt.demo_scene(0, seed=0, n_objects=32)
        tracer = pt.PathTracer(0, sc, W, H)
        cam = pt.Camera(position=(0.0, 4.0, 13.0), target=(0.0, 0.8, 0.0), fov=50, aspect=W / H)
        state = {"vp": None}

        def pt_step(i):
            state["vp"] = tracer.write_uniforms(camera=cam, prev_view_proj=state["vp"], frame=i, mode=0,
                                                jitter=pt.JITTER[i % 16], env=env)
            tracer.encode(i & 1, stream=stream)

        out["pt_ms_per_frame"] = timed(pt_step)
        out["pt_config"] = "demo scene, 32 objects, 1 spp, 3 bounces, NEE + MIS, env map"
        tracer.destroy()
    except Exception as e:  # pragma: no cover
        out["pt_ms_per_frame"] = f"failed: {e}"
    try:
        post = Post(0, "rgba8unorm")
        den = frames[0]["radiance"]

        def post_step(i):
            post.encode(frames[i % len(frames)]["radiance"], den, split=0.5, stream=stream)

        out["post_ms_per_frame"] = timed(post_step)
        post.destroy()
    except Exception as e:  # pragma: no cover
        out["post_ms_per_frame"] = f"failed: {e}"
    return out


def _train_step_ms(local, stream, barrier, max_over_ranks, warmup=2, steps=5, mlp="bf16", bptt=False):
    """Device time of one training step: 16 windows x 8 frames of 384x384 generated on the device, the twin's
    forward + adjoint per frame (MLP as bf16 tensor-core GEMM tiles, or FP32) or, with bptt, each window forward and
    backward through time, the gradient / loss all-reduce across ranks (N > 1) and the Adam step."""
    import torch

    from hush_b200 import Hush
    from hush_b200.dp import DataParallel, finish_step
    from hush_b200.train import TrainConfig, Trainer, window_scene, xavier_init

    cfg = TrainConfig(mlp=mlp, bptt=bptt)
    dp = DataParallel()
    th = Hush(local, {"width": cfg.size, "height": cfg.size, "schedule": "passes"})
    tr = Trainer(th, xavier_init(cfg.init_seed))
    tr.set_mlp(cfg.mlp)
    rng = dp.seed_rng(cfg.init_seed + 1)
    sc = window_scene(cfg)

    def one():
        seeds = [dp.window_seed(rng, cfg.seeds) for _ in range(cfg.batch)]
        if bptt:
            tr.windows_bptt(sc, seeds, cfg.frames, cfg.lambda_t, stream=stream)
        else:
            tr.windows(sc, seeds, cfg.frames, cfg.lambda_t, stream=stream)
        return finish_step(tr, dp, cfg.batch * cfg.frames, cfg.lr, cfg.clip)

    for _ in range(warmup):
        one()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    losses = [one()[0] for _ in range(steps)]
    e1.record(stream)
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1)) / steps
    tr.destroy()
    th.destroy()
    return {"step_ms": round(ms, 3), "mlp": cfg.mlp, "steps": steps, "warmup": warmup, "world": dp.world,
            "windows_per_step": cfg.batch * dp.world, "frames_per_step": cfg.batch * cfg.frames * dp.world,
            "size": f"{cfg.size}x{cfg.size}", "loss_last": round(losses[-1], 5),
            "note": "window generation, twin forward + adjoint of every frame, gradient all-reduce (N > 1), Adam"}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2048)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mlp", default="fp32", choices=["fp32", "bf16", "f16"])
    ap.add_argument("--schedule", default="fused", choices=["fused", "passes"])
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="launch the eight kernels of each frame directly instead of replaying the frame as a CUDA graph")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-train", action="store_true", help="skip the training-step timing")
    ap.add_argument("--no-extras", action="store_true", help="skip the SVGF / path tracer / post timings")
    ap.add_argument("--dry-run", action="store_true",
                    help="run only the rank plumbing on the CPU (gloo) and print the rank fields of the line")
    ap.add_argument("--workload", default="1080p", choices=["1080p", "4k"],
                    help="4k: the 3840x2160 workload (32 objects, 8 moving, 20%% sky, pan U[0,6], 2%% fireflies x100) "
                         "with the BF16 MLP and each frame replayed as one CUDA graph")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    if args.workload == "4k":
        global W, H, SEQ, WORKLOAD
        W, H, SEQ = 3840, 2160, 16
        WORKLOAD = ("3840x2160 sequence (16 frames resident, looped with reset), 32 objects, 8 moving, 20% sky, "
                    "pan U[0,6] px/frame, 2% fireflies x100; BF16 MLP, one CUDA graph per frame")
        if "--mlp" not in (argv or sys.argv):
            args.mlp = "bf16"
        args.graph = True
        args.no_train = True
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return _launch_ranks(args.gpus, list(sys.argv[1:] if argv is None else argv))
    if args.dry_run:
        return run_dry(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


def _launch_ranks(n: int, argv) -> int:
    """`bench.py --gpus N` without an outer torchrun: re-run this script as N ranks on this node (one process per GPU,
    rendezvous on 127.0.0.1), bounded by `timeout -k 60` well above the run's own process-group timeouts."""
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__)] + argv
    return subprocess.call(cmd)


def run_dry(args) -> int:
    """--dry-run: the rank plumbing alone, on the CPU (gloo): every rank joins, one all-reduce counts them, rank 0
    prints the line's rank fields. No GPU work."""
    import datetime

    import torch
    import torch.distributed as dist

    rank, _, world = _env_rank()
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    t = torch.ones(1)
    if world > 1:
        dist.all_reduce(t)
    if rank == 0:
        print(json.dumps({"dry_run": True, "impl": args.impl, "metric": METRIC, "n_gpus": world,
                          "ranks_joined": int(t.item()), "config": _config(args.mlp, world)}), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
