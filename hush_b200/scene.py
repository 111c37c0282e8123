"""Seeded synthetic G-buffer sequences (the benchmark workloads; there is no public dataset for this path).

A ground plane plus spheres and y-rotated boxes ray-cast analytically (csrc/scene.h): normals, linear depth, depth -1
for sky, integer object ids < 2048, per-object albedo U[0.05, 0.9]^3 times an 8 x 8 checker factor 0.6 / 1.0,
roughness U[0, 1], one emissive sphere at 5.0. Clean radiance is Lambert shading under one directional light (hard
shadows) plus 0.1 ambient; the 1 spp radiance is clean x Exp(1) per pixel and channel with fireflies. The camera
yaws and pans; motion vectors and previous depth come from the analytic previous camera.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace

import numpy as np

from . import _lib as L

NAMES = ["radiance", "normalDepth", "motion", "material", "emission"]


@dataclass(frozen=True)
class SceneConfig:
    width: int
    height: int
    frames: int
    n_objects: int = 12
    n_moving: int = 0
    sky_frac: float = 0.10
    pan_min: float = 2.0
    pan_max: float = 2.0
    yaw_deg: float = 0.2
    firefly_rate: float = 0.005
    firefly_scale: float = 50.0
    cut_frame: int = -1
    seed: int = 1

    def with_(self, **kw) -> "SceneConfig":
        return replace(self, **kw)

    def c(self) -> "L.HushScene":
        return L.HushScene(self.width, self.height, self.n_objects, self.n_moving, self.sky_frac, self.pan_min,
                           self.pan_max, self.yaw_deg, self.firefly_rate, self.firefly_scale, self.cut_frame,
                           self.seed & 0xFFFFFFFF)


# The workloads: plain forward 640x360x8; 1080p x64 with 3 moving objects, pan U[0,4] and a cut at 32; 256^2 crops
# (adjoint check); 384^2 x 8 windows (training); 4K x 120 with 32 objects, 8 moving, 20% sky, pan U[0,6], 2% x100.
CONFIG_360P = SceneConfig(640, 360, 8)
CONFIG_1080P = SceneConfig(1920, 1080, 64, n_moving=3, pan_min=0.0, pan_max=4.0, cut_frame=32)
CONFIG_CROP = SceneConfig(256, 256, 4)
CONFIG_TRAIN = SceneConfig(384, 384, 8)
CONFIG_4K = SceneConfig(3840, 2160, 120, n_objects=32, n_moving=8, sky_frac=0.20, pan_min=0.0, pan_max=6.0,
                        firefly_rate=0.02, firefly_scale=100.0)


def frame_host(cfg: SceneConfig, frame: int, clean: bool = False):
    """One frame as numpy: dict of five (H, W, 4) float16 arrays (+ 'clean' (H, W, 3) float32)."""
    H, W = cfg.height, cfg.width
    bufs = {n: np.empty((H, W, 4), dtype=np.float16) for n in NAMES}
    cl = np.empty((H, W, 3), dtype=np.float32) if clean else None
    sc = cfg.c()
    rc = L.lib().hush_scene_frame_host(C.byref(sc), int(frame), *[bufs[n].ctypes.data for n in NAMES],
                                       cl.ctypes.data if clean else None)
    if rc != 0:
        raise RuntimeError(f"scene generation failed ({rc})")
    if clean:
        bufs["clean"] = cl
    return bufs


def frame_device(cfg: SceneConfig, frame: int, out: dict | None = None, clean: bool = False, stream=None):
    """One frame generated on the GPU into (H, W, 4) float16 CUDA tensors (allocated if ``out`` is None)."""
    import torch

    H, W = cfg.height, cfg.width
    if out is None:
        out = {n: torch.empty((H, W, 4), dtype=torch.float16, device="cuda") for n in NAMES}
        if clean:
            out["clean"] = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    sc = cfg.c()
    st = torch.cuda.current_stream().cuda_stream if stream is None else stream
    rc = L.lib().hush_scene_frame_device(C.byref(sc), int(frame), *[out[n].data_ptr() for n in NAMES],
                                         out["clean"].data_ptr() if "clean" in out else None, C.c_void_p(st))
    if rc != 0:
        raise RuntimeError(f"scene generation failed ({rc})")
    return out
