"""The path tracer (src/pt): SceneGPU, PathTracer, JITTER, prepareEnvMap / envSunLight, without three.js.

Meshes arrive as world-space numpy arrays; a small perspective Camera stands in for three.PerspectiveCamera (same
matrix conventions: column-major elements, the camera looks down -z). The tracer writes the five Hush inputs
(radiance, normalDepth, motion, material, emission) into one of two G-buffer slots per frame:

    scene = SceneGPU(0)
    m = scene.add_material(base=(0.8, 0.8, 0.8), roughness=0.6)
    scene.add_mesh(positions, indices, m, normals=normals)
    scene.build()
    pt = PathTracer(0, scene, 640, 360)
    vp = pt.write_uniforms(camera=cam, prev_view_proj=prev_vp, frame=i, mode=0, jitter=JITTER[i % 16], env=env)
    pt.encode(i & 1)
    gbuf = pt.gbuf[i & 1]          # dict of (H, W, 4) float16 CUDA views, ready for Hush.denoise
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib as L
from .hush import HushError, _DevView, _stream_handle

MAX_BLAS, MAX_LIGHTS = 8, 8
TEX_SIZE, TEX_MIPS = 1024, 11
ENV_GRID = (256, 128)
GBUF_NAMES = ["radiance", "normalDepth", "motion", "material", "emission"]
GROUP_DYNAMIC, GROUP_NO_SHADOW = 1, 2


class PtMaterial(C.Structure):
    _fields_ = [("base", C.c_float * 4), ("emissive", C.c_float * 4), ("pbr", C.c_float * 4),
                ("tex", C.c_int32 * 4), ("uv", C.c_float * 4)]


class PtBlas(C.Structure):
    _fields_ = [("node_offset", C.c_uint32), ("tri_offset", C.c_uint32), ("node_count", C.c_uint32),
                ("flags", C.c_uint32)]


class PtLight(C.Structure):
    _fields_ = [("pos", C.c_float * 4), ("prev_pos", C.c_float * 4), ("radiance", C.c_float * 4),
                ("params", C.c_float * 4)]


class PtFrame(C.Structure):
    _fields_ = [("cam_pos", C.c_float * 4), ("cam_right", C.c_float * 4), ("cam_up", C.c_float * 4),
                ("cam_fwd", C.c_float * 4), ("view_proj", C.c_float * 16), ("prev_view_proj", C.c_float * 16),
                ("size", C.c_uint32 * 2), ("frame", C.c_uint32), ("mode", C.c_uint32), ("jitter", C.c_float * 2),
                ("spp", C.c_uint32), ("max_bounces", C.c_uint32), ("sky_zenith", C.c_float * 4),
                ("sky_horizon", C.c_float * 4), ("ground", C.c_float * 4), ("counts", C.c_uint32 * 4),
                ("clamp_lum", C.c_float), ("pixel_angle", C.c_float), ("shadow_tau", C.c_float),
                ("clamp_direct", C.c_float), ("env", C.c_float * 4), ("blas", PtBlas * MAX_BLAS),
                ("lights", PtLight * MAX_LIGHTS)]


assert C.sizeof(PtFrame) == 960 and C.sizeof(PtMaterial) == 80

_P = C.c_void_p
_SIGS = {
    "hush_pt_material_default": (PtMaterial, []),
    "hush_pt_scene_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "hush_pt_scene_destroy": (None, [_P]),
    "hush_pt_scene_add_material": (C.c_int, [_P, C.POINTER(PtMaterial)]),
    "hush_pt_scene_add_texture": (C.c_int, [_P, _P, C.c_int, C.c_int]),
    "hush_pt_scene_add_group": (C.c_int, [_P, C.c_int, _P, _P, _P, C.c_int, _P, _P, C.c_int]),
    "hush_pt_scene_build": (C.c_int, [_P]),
    "hush_pt_scene_update": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "hush_pt_scene_blas": (C.c_int, [_P, C.POINTER(PtBlas), C.c_int]),
    "hush_pt_scene_info": (C.c_int, [_P] + [C.POINTER(C.c_int)] * 4),
    "hush_pt_scene_device": (C.c_int, [_P] + [C.POINTER(_P)] * 6),
    "hush_pt_bvh_build": (C.c_int, [_P, C.c_int, _P, _P, C.POINTER(C.c_int)]),
    "hush_pt_env_prepare": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_double, _P, _P, _P, _P]),
    "hush_pt_jitter": (None, [_P]),
    "hush_pt_create": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(_P)]),
    "hush_pt_destroy": (None, [_P]),
    "hush_pt_resize": (C.c_int, [_P, C.c_int, C.c_int]),
    "hush_pt_set_envmap": (C.c_int, [_P, _P, C.c_int, C.c_int, _P]),
    "hush_pt_encode": (C.c_int, [_P, C.POINTER(PtFrame), C.c_int, _P]),
    "hush_pt_gbuffer": (_P, [_P, C.c_int, C.c_int]),
    "hush_pt_accum": (_P, [_P]),
    "hush_pt_clear_accum": (C.c_int, [_P, _P]),
    "hush_pt_last_error": (C.c_char_p, []),
}
_bound = False


def lib():
    global _bound
    lb = L.lib()
    if not _bound:
        for name, (res, args) in _SIGS.items():
            fn = getattr(lb, name)
            fn.restype, fn.argtypes = res, args
        _bound = True
    return lb


def _check(rc, what=""):
    if rc != L.HUSH_OK:
        raise HushError((lib().hush_pt_last_error() or b"").decode() or f"{what} failed ({rc})")


def _halton(i: int, b: int) -> float:
    f, r = 1.0, 0.0
    while i > 0:
        f /= b
        r += f * (i % b)
        i //= b
    return r


# 16-phase Halton(2, 3) subpixel jitter in pixels, [-0.5, 0.5] (pathtracer.js:6-12)
JITTER = [(_halton(i + 1, 2) - 0.5, _halton(i + 1, 3) - 0.5) for i in range(16)]


# ------------------------------------------------------------------------------------------------ camera
class Camera:
    """Perspective camera with three.js conventions (fov in degrees, vertical; looks down -z in its frame)."""

    def __init__(self, position=(0, 0, 5), target=(0, 0, 0), up=(0, 1, 0), fov=50.0, aspect=16 / 9, near=0.1,
                 far=1000.0):
        self.fov, self.aspect, self.near, self.far = float(fov), float(aspect), float(near), float(far)
        self.look_at(position, target, up)

    def look_at(self, position, target, up=(0, 1, 0)):
        eye = np.asarray(position, np.float64)
        z = eye - np.asarray(target, np.float64)
        z = z / np.linalg.norm(z)
        x = np.cross(np.asarray(up, np.float64), z)
        x = x / np.linalg.norm(x)
        y = np.cross(z, x)
        m = np.eye(4)
        m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = x, y, z, eye
        self.matrix_world = m  # row-major numpy; .T.ravel() gives three.js elements
        return self

    @property
    def elements(self):
        return self.matrix_world.T.ravel()

    def projection(self) -> np.ndarray:
        top = self.near * math.tan(math.radians(0.5 * self.fov))
        h = 2 * top
        w = self.aspect * h
        left = -0.5 * w
        r, t, b = left + w, top, top - h
        n, f = self.near, self.far
        p = np.zeros((4, 4))
        p[0, 0], p[0, 2] = 2 * n / (r - left), (r + left) / (r - left)
        p[1, 1], p[1, 2] = 2 * n / (t - b), (t + b) / (t - b)
        p[2, 2], p[2, 3] = -(f + n) / (f - n), -2 * f * n / (f - n)
        p[3, 2] = -1.0
        return p

    def view_proj(self) -> np.ndarray:
        """projection * inverse(matrixWorld) as 16 column-major float32 elements."""
        vp = self.projection() @ np.linalg.inv(self.matrix_world)
        return vp.T.ravel().astype(np.float32)


# ------------------------------------------------------------------------------------------------ env map
@dataclass
class EnvMap:
    width: int
    height: int
    half: np.ndarray   # (H, W, 4) uint16 (rgba16float)
    table: np.ndarray  # (128, 256, 4) float32 alias table (threshold, alias bits, pmf, 0)
    sun: Optional[dict] = None


def prepare_env_map(data: np.ndarray, sun: bool = True, sun_cone_deg: float = 3.0) -> EnvMap:
    """prepareEnvMap (envmap.js:85-105) of an equirect float image (H, W, 4), row 0 = up."""
    img = np.ascontiguousarray(data, np.float32).copy()
    H, W = img.shape[:2]
    half = np.zeros((H, W, 4), np.uint16)
    table = np.zeros((ENV_GRID[1], ENV_GRID[0], 4), np.float32)
    d, e = (C.c_double * 3)(), (C.c_double * 3)()
    rc = lib().hush_pt_env_prepare(img.ctypes.data, W, H, 1 if sun else 0, float(sun_cone_deg), half.ctypes.data,
                                   table.ctypes.data, d, e)
    if rc < 0:
        raise HushError(lib().hush_pt_last_error().decode())
    s = {"dir": list(d), "irradiance": list(e)} if rc == 1 else None
    return EnvMap(W, H, half, table, s)


def env_sun_light(m: EnvMap, rotation: float = 0.0, angular_deg: float = 0.53, scale: float = 1.0,
                  tint=(1.0, 1.0, 1.0)):
    """envSunLight (envmap.js:114-122): the cut-out sun as a cone light, rotated like the map; None without a sun."""
    if not m.sun:
        return None
    x, y, z = m.sun["dir"]
    c, s = math.cos(rotation), math.sin(rotation)
    cos_max = math.cos(math.radians(angular_deg / 2))
    omega = 2 * math.pi * (1 - cos_max)
    return {"kind": 0, "dir": [c * x + s * z, y, -s * x + c * z], "cosMax": cos_max,
            "radiance": [e * scale * t / omega for e, t in zip(m.sun["irradiance"], tint)]}


# ------------------------------------------------------------------------------------------------ scene
@dataclass
class _Group:
    flags: int
    pos: list = field(default_factory=list)
    nrm: list = field(default_factory=list)
    uv: list = field(default_factory=list)
    idx: list = field(default_factory=list)
    mat: list = field(default_factory=list)
    n_verts: int = 0
    gid: int = -1


class SceneGPU:
    """SceneGPU (scene.js) from world-space meshes: group 0 holds the static meshes; add_group() makes a dynamic or
    no-shadow BLAS (at most 8 groups in all)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().hush_pt_scene_create(int(device), C.byref(h)), "SceneGPU")
        self._h, self.device = h, int(device)
        self._groups = [_Group(0)]
        self._mats = []
        self.built = False

    def add_material(self, base=(1, 1, 1), alpha_cutoff=0.0, emissive=(0, 0, 0), roughness=1.0, metalness=0.0,
                     transmission=0.0, ior=1.5, tex_base=-1, tex_normal=-1, tex_arm=-1, uv_scale=(1, 1),
                     normal_scale=1.0) -> int:
        m = PtMaterial()
        m.base[:] = [*base, alpha_cutoff]
        m.emissive[:] = [*emissive, 0.0]
        m.pbr[:] = [roughness, metalness, transmission, ior]
        m.tex[:] = [tex_base, tex_normal, tex_arm, 0]
        m.uv[:] = [uv_scale[0], uv_scale[1], normal_scale, 0.0]
        i = lib().hush_pt_scene_add_material(self._h, C.byref(m))
        if i < 0:
            _check(L.HUSH_ERR_ARG)
        self._mats.append(bytes(m))
        return i

    def materials_array(self) -> np.ndarray:
        """(M, 20) float32 material records as uploaded (texture layers stored as int32 bits)."""
        return np.frombuffer(b"".join(self._mats), np.float32).reshape(-1, 20).copy()

    def group_arrays(self) -> list:
        """The BLAS inputs in build order: dicts of flags and concatenated pos / nrm / uv / idx / mat arrays."""
        out = []
        for g in self._groups:
            if g.idx:
                out.append({"flags": g.flags, "pos": np.concatenate(g.pos), "nrm": np.concatenate(g.nrm),
                            "uv": np.concatenate(g.uv), "idx": np.concatenate(g.idx) - 0,
                            "mat": np.concatenate(g.mat)})
        return out

    def add_texture(self, rgba: np.ndarray) -> int:
        a = np.ascontiguousarray(rgba, np.uint8)
        i = lib().hush_pt_scene_add_texture(self._h, a.ctypes.data, a.shape[1], a.shape[0])
        if i < 0:
            _check(L.HUSH_ERR_ARG)
        return i

    def add_group(self, dynamic: bool = False, no_shadow: bool = False) -> int:
        """A new BLAS for meshes that move (dynamic) or that shadow rays skip (no_shadow); returns its handle."""
        if len(self._groups) >= MAX_BLAS:
            raise HushError("too many dynamic groups")
        self._groups.append(_Group((GROUP_DYNAMIC if dynamic else 0) | (GROUP_NO_SHADOW if no_shadow else 0)))
        return len(self._groups) - 1

    def add_mesh(self, positions, indices, material, normals=None, uvs=None, group: int = 0):
        g = self._groups[group]
        p = np.asarray(positions, np.float32).reshape(-1, 3)
        ix = np.asarray(indices, np.uint32).reshape(-1, 3)
        g.pos.append(p)
        g.nrm.append(np.tile([0, 1, 0], (len(p), 1)).astype(np.float32) if normals is None
                     else np.asarray(normals, np.float32).reshape(-1, 3))
        g.uv.append(np.zeros((len(p), 2), np.float32) if uvs is None else np.asarray(uvs, np.float32).reshape(-1, 2))
        g.idx.append(ix + g.n_verts)
        mat = np.broadcast_to(np.asarray(material, np.uint32), (len(ix),))
        g.mat.append(np.ascontiguousarray(mat))
        g.n_verts += len(p)

    def build(self):
        for g in self._groups:
            if not g.idx:
                continue
            pos, nrm, uv = (np.ascontiguousarray(np.concatenate(a)) for a in (g.pos, g.nrm, g.uv))
            idx, mat = np.ascontiguousarray(np.concatenate(g.idx)), np.ascontiguousarray(np.concatenate(g.mat))
            g.gid = lib().hush_pt_scene_add_group(self._h, g.flags, pos.ctypes.data, nrm.ctypes.data, uv.ctypes.data,
                                                  len(pos), idx.ctypes.data, mat.ctypes.data, len(idx))
            if g.gid < 0:
                _check(L.HUSH_ERR_ARG)
        _check(lib().hush_pt_scene_build(self._h), "SceneGPU.build")
        self.built = True

    def update(self, group: int, positions, normals=None, stream=None):
        """Re-poses a dynamic group: all of its vertices (in add_mesh order), normals or None for smooth normals."""
        g = self._groups[group]
        p = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        if len(p) != g.n_verts:
            raise HushError(f"SceneGPU.update: group {group} has {g.n_verts} vertices, got {len(p)}")
        n = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        _check(lib().hush_pt_scene_update(self._h, g.gid, p.ctypes.data, None if n is None else n.ctypes.data,
                                          C.c_void_p(_stream_handle(stream))), "SceneGPU.update")

    def blas_table(self):
        t = (PtBlas * MAX_BLAS)()
        n = lib().hush_pt_scene_blas(self._h, t, MAX_BLAS)
        return [t[i] for i in range(n)]

    @property
    def tri_total(self) -> int:
        v = [C.c_int() for _ in range(4)]
        _check(lib().hush_pt_scene_info(self._h, *[C.byref(x) for x in v]))
        return v[0].value

    def info(self) -> dict:
        v = [C.c_int() for _ in range(4)]
        _check(lib().hush_pt_scene_info(self._h, *[C.byref(x) for x in v]))
        return dict(zip(("tri_total", "node_total", "vert_total", "max_depth"), (x.value for x in v)))

    def device_buffers(self) -> dict:
        p = [C.c_void_p() for _ in range(6)]
        _check(lib().hush_pt_scene_device(self._h, *[C.byref(x) for x in p]))
        return dict(zip(("nodes", "tris", "tri_idx", "verts", "mats", "tex"), (x.value for x in p)))

    def destroy(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().hush_pt_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.destroy()
        except Exception:
            pass


def bvh_build(positions: np.ndarray):
    """The product's binned-SAH builder alone (bvh.js buildBVH): (nodes (n, 8) float32 build layout, order, depth)."""
    p = np.ascontiguousarray(positions, np.float32).reshape(-1, 9)
    n = len(p)
    nodes = np.zeros((max(1, 2 * n), 8), np.float32)
    order = np.zeros(max(1, n), np.uint32)
    depth = C.c_int()
    used = lib().hush_pt_bvh_build(p.ctypes.data, n, nodes.ctypes.data, order.ctypes.data, C.byref(depth))
    if used < 0:
        _check(L.HUSH_ERR_ARG)
    return nodes[:used], order[:n], depth.value


# ------------------------------------------------------------------------------------------------ tracer
def frame_uniforms(camera: Camera, prev_view_proj, frame: int, mode: int, jitter, width: int, height: int,
                   blas, env: dict, spp: int = 1, sample_offset: int = 0, max_bounces: int = 3,
                   clamp_lum: float = 16.0, shadow_tau: float = 0.0):
    """writeUniforms (pathtracer.js:105-149) as a PtFrame; returns (frame struct, this frame's view-projection)."""
    f = PtFrame()
    e = camera.elements
    th = math.tan(math.radians(camera.fov) / 2)
    right, up, fwd = e[0:3], e[4:7], -e[8:11]
    f.cam_pos[:] = [*e[12:15], 0.0]
    f.cam_right[:] = [*(right * th * camera.aspect), 0.0]
    f.cam_up[:] = [*(up * th), 0.0]
    f.cam_fwd[:] = [*fwd, 0.0]
    vp = camera.view_proj()
    f.view_proj[:] = list(vp)
    f.prev_view_proj[:] = list(vp if prev_view_proj is None else np.asarray(prev_view_proj, np.float32))
    f.size[:] = [width, height]
    f.frame, f.mode = frame & 0xffffffff, mode
    f.jitter[:] = list(jitter)
    f.spp, f.max_bounces = spp, max_bounces
    f.sky_zenith[:] = [*env.get("skyZenith", (0, 0, 0)), 0.0]
    f.sky_horizon[:] = [*env.get("skyHorizon", (0, 0, 0)), env.get("skyIntensity", 1.0)]
    f.ground[:] = [*env.get("ground", (0, 0, 0)), 0.0]
    lights = list(env.get("lights", []))[:MAX_LIGHTS]
    f.counts[:] = [len(blas), len(lights), sample_offset, 0]
    f.clamp_lum = env.get("clampLum", clamp_lum)
    f.pixel_angle = 2 * th / height
    f.shadow_tau = shadow_tau
    f.clamp_direct = env.get("clampDirect", 0.0) or 0.0
    rot = env.get("mapRotation", 0.0)
    f.env[:] = [env.get("mapIntensity", 1.0), math.cos(rot), math.sin(rot), 1.0 if env.get("map") else 0.0]
    for i, b in enumerate(blas):
        f.blas[i] = b
    for i, Lt in enumerate(lights):
        if Lt["kind"] == 0:
            f.lights[i].pos[:] = [*Lt["dir"], 0.0]
            f.lights[i].prev_pos[:] = [*Lt["dir"], 0.0]
            f.lights[i].radiance[:] = [*Lt["radiance"], 0.0]
            f.lights[i].params[:] = [0.0, Lt["cosMax"], 0.0, 0.0]
        else:
            f.lights[i].pos[:] = [*Lt["pos"], Lt["radius"]]
            f.lights[i].prev_pos[:] = [*Lt.get("prevPos", Lt["pos"]), Lt["radius"]]
            f.lights[i].radiance[:] = [*Lt["radiance"], 0.0]
            f.lights[i].params[:] = [1.0, 0.0, 0.0, 0.0]
    return f, vp


class PathTracer:
    """PathTracer (pathtracer.js:14-162): 1 spp + G-buffer (mode 0) or accumulated reference paths (mode 1)."""

    def __init__(self, device, scene: SceneGPU, width: int, height: int):
        if not scene.built:
            scene.build()
        h = C.c_void_p()
        _check(lib().hush_pt_create(scene._h, int(width), int(height), C.byref(h)), "PathTracer")
        self._h, self.scene, self.device = h, scene, scene.device
        self.width, self.height = int(width), int(height)
        self._frame = None
        self._env_map = None
        self._views()

    def _views(self):
        import torch

        dev = torch.device("cuda", self.device)
        self.gbuf = []
        for s in range(2):
            self.gbuf.append({n: torch.as_tensor(_DevView(lib().hush_pt_gbuffer(self._h, s, k), self.height,
                                                          self.width, 4, "<f2"), device=dev)
                              for k, n in enumerate(GBUF_NAMES)})
        self.accum = torch.as_tensor(_DevView(lib().hush_pt_accum(self._h), self.height, self.width, 4, "<f4"),
                                     device=dev)

    def resize(self, width: int, height: int):
        _check(lib().hush_pt_resize(self._h, int(width), int(height)), "PathTracer.resize")
        self.width, self.height = int(width), int(height)
        self._views()

    def set_env_map(self, m: Optional[EnvMap]):
        if m is self._env_map:
            return
        if m is None:
            _check(lib().hush_pt_set_envmap(self._h, None, 0, 0, None))
        else:
            _check(lib().hush_pt_set_envmap(self._h, m.half.ctypes.data, m.width, m.height, m.table.ctypes.data))
        self._env_map = m

    def write_uniforms(self, camera: Camera, prev_view_proj=None, frame: int = 0, mode: int = 0,
                       jitter=(0.0, 0.0), spp: int = 1, sample_offset: int = 0, max_bounces: int = 3,
                       clamp_lum: float = 16.0, shadow_tau: float = 0.0, env: Optional[dict] = None) -> np.ndarray:
        env = env or {}
        self.set_env_map(env.get("map"))
        self._frame, vp = frame_uniforms(camera, prev_view_proj, frame, mode, jitter, self.width, self.height,
                                         self.scene.blas_table(), env, spp, sample_offset, max_bounces, clamp_lum,
                                         shadow_tau)
        return vp

    def encode(self, slot: int = 0, stream=None):
        if self._frame is None:
            raise HushError("PathTracer.encode: call write_uniforms first")
        _check(lib().hush_pt_encode(self._h, C.byref(self._frame), int(slot), C.c_void_p(_stream_handle(stream))),
               "PathTracer.encode")
        return self.gbuf[slot]

    def clear_accum(self, stream=None):
        _check(lib().hush_pt_clear_accum(self._h, C.c_void_p(_stream_handle(stream))))

    def destroy(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().hush_pt_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.destroy()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------------ demo scenes
def box_mesh(center, size, rot_y=0.0):
    """Axis-aligned box (rotated about +y) as 24 vertices with face normals and 12 triangles."""
    c, s = math.cos(rot_y), math.sin(rot_y)
    R = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    pos, nrm, uv, idx = [], [], [], []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            n = np.zeros(3)
            n[axis] = sign
            u_ax, v_ax = [a for a in range(3) if a != axis]
            base = len(pos)
            for (a, b) in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                p = np.zeros(3)
                p[axis] = sign
                p[u_ax], p[v_ax] = a, b
                pos.append(R @ (p * np.asarray(size) * 0.5) + np.asarray(center))
                nrm.append(R @ n)
                uv.append(((a + 1) / 2, (b + 1) / 2))
            quad = [(0, 1, 2), (0, 2, 3)]
            # outward winding
            flip = (sign > 0) == ((axis == 1))
            for t in quad:
                idx.append([base + t[0], base + t[2], base + t[1]] if flip else [base + k for k in t])
    return (np.asarray(pos, np.float32), np.asarray(idx, np.uint32), np.asarray(nrm, np.float32),
            np.asarray(uv, np.float32))


def sphere_mesh(center, radius, seg=24, rings=12):
    pos, nrm, uv, idx = [], [], [], []
    for r in range(rings + 1):
        th = math.pi * r / rings
        for s in range(seg + 1):
            ph = 2 * math.pi * s / seg
            n = np.array([math.sin(th) * math.cos(ph), math.cos(th), math.sin(th) * math.sin(ph)])
            pos.append(np.asarray(center) + radius * n)
            nrm.append(n)
            uv.append((s / seg, r / rings))
    for r in range(rings):
        for s in range(seg):
            a, b = r * (seg + 1) + s, (r + 1) * (seg + 1) + s
            if r > 0:  # the pole rows would give zero-area triangles
                idx.append([a, a + 1, b])
            if r < rings - 1:
                idx.append([a + 1, b + 1, b])
    return (np.asarray(pos, np.float32), np.asarray(idx, np.uint32), np.asarray(nrm, np.float32),
            np.asarray(uv, np.float32))


def _textures(sc: SceneGPU):
    """A checker albedo, a leaf-like alpha cut-out, a bumpy normal map and an ARM map (roughness in g, metal in b)."""
    yy, xx = np.indices((64, 64))
    ch = (((xx // 8) + (yy // 8)) % 2).astype(np.float32)
    albedo = np.zeros((64, 64, 4), np.uint8)
    albedo[..., :3] = (150 + 105 * ch)[..., None]
    albedo[..., 3] = 255
    cut = albedo.copy()
    r = np.hypot(xx - 31.5, yy - 31.5)
    cut[..., 3] = np.where((r < 28) & ((xx + yy) % 16 > 3), 255, 0)
    nrm = np.zeros((64, 64, 4), np.uint8)
    nx, ny = 0.35 * np.sin(xx / 4.0), 0.35 * np.cos(yy / 5.0)
    nz = np.sqrt(np.clip(1 - nx ** 2 - ny ** 2, 0, 1))
    nrm[..., 0], nrm[..., 1], nrm[..., 2], nrm[..., 3] = ((nx + 1) * 127.5), ((ny + 1) * 127.5), ((nz + 1) * 127.5), 255
    arm = np.zeros((64, 64, 4), np.uint8)
    arm[..., 0], arm[..., 1], arm[..., 2], arm[..., 3] = 255, (80 + 170 * ch), (255 * (1 - ch)), 255
    return [sc.add_texture(t) for t in (albedo, cut, nrm, arm)]


def demo_scene(device: int = 0, seed: int = 0, n_objects: int = 12, textured: bool = True, dynamic: bool = True):
    """Ground plane plus boxes and spheres (diffuse, metal, glass, one emissive), textured materials (checker albedo,
    an alpha cut-out panel, a normal- and ARM-mapped box) and one moving box in a dynamic group. Returns (scene, env,
    mover) where mover(t) re-poses the dynamic group for frame t (None without a dynamic group)."""
    rng = np.random.default_rng(seed)
    sc = SceneGPU(device)
    t_alb = t_cut = t_nrm = t_arm = -1
    if textured:
        t_alb, t_cut, t_nrm, t_arm = _textures(sc)
    ground = sc.add_material(base=(0.7, 0.7, 0.7), roughness=0.8, tex_base=t_alb, uv_scale=(8, 8))
    gp = np.array([[-20, 0, -20], [20, 0, -20], [20, 0, 20], [-20, 0, 20]], np.float32)
    sc.add_mesh(gp, [[0, 2, 1], [0, 3, 2]], ground, normals=np.tile([0, 1, 0], (4, 1)),
                uvs=[[0, 0], [1, 0], [1, 1], [0, 1]])
    for i in range(n_objects):
        kind = i % 4
        base = tuple(rng.uniform(0.05, 0.9, 3))
        m = sc.add_material(base=base, roughness=float(rng.uniform(0.05, 1.0)),
                            metalness=1.0 if kind == 1 else 0.0, transmission=1.0 if kind == 3 and i % 8 == 3 else 0.0,
                            emissive=(5.0, 4.0, 3.0) if i == 0 else (0, 0, 0))
        r = float(rng.uniform(0.2, 1.5))
        c = (float(rng.uniform(-6, 6)), r, float(rng.uniform(-6, 6)))
        mesh = sphere_mesh(c, r) if kind % 2 == 0 else box_mesh(c, (2 * r, 2 * r, 2 * r), float(rng.uniform(0, 3)))
        sc.add_mesh(mesh[0], mesh[1], m, normals=mesh[2], uvs=mesh[3])
    if textured:
        cut = sc.add_material(base=(0.3, 0.8, 0.3, ), alpha_cutoff=0.5, roughness=0.7, tex_base=t_cut)
        q = np.array([[-2.5, 0.2, 2.0], [-0.5, 0.2, 2.0], [-0.5, 2.2, 2.0], [-2.5, 2.2, 2.0]], np.float32)
        sc.add_mesh(q, [[0, 1, 2], [0, 2, 3]], cut, normals=np.tile([0, 0, 1], (4, 1)),
                    uvs=[[0, 0], [1, 0], [1, 1], [0, 1]])
        bumpy = sc.add_material(base=(0.8, 0.7, 0.5), roughness=1.0, metalness=1.0, tex_normal=t_nrm, tex_arm=t_arm,
                                normal_scale=1.0)
        bm = box_mesh((2.5, 0.8, 2.5), (1.6, 1.6, 1.6), 0.4)
        sc.add_mesh(bm[0], bm[1], bumpy, normals=bm[2], uvs=bm[3])
    mover = None
    if dynamic:
        g = sc.add_group(dynamic=True)
        mm = sc.add_material(base=(0.9, 0.3, 0.2), roughness=0.3)
        p0, ix, n0, uv0 = box_mesh((0, 0.6, 0), (1.2, 1.2, 1.2))
        sc.add_mesh(p0, ix, mm, normals=n0, uvs=uv0, group=g)

        def mover(t):
            a = 0.15 * t
            c, s = math.cos(a), math.sin(a)
            R = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]], np.float32)
            off = np.array([3 * math.cos(0.1 * t), 0, 3 * math.sin(0.1 * t)], np.float32)
            pos, nrm = p0 @ R.T + off, n0 @ R.T
            sc.update(g, pos, nrm)
            return pos, nrm
        mover.group = g
    sc.build()
    env = {"skyZenith": (0.3, 0.45, 0.8), "skyHorizon": (0.8, 0.85, 0.9), "skyIntensity": 1.0,
           "ground": (0.3, 0.28, 0.25),
           "lights": [{"kind": 0, "dir": list(np.array([0.4, 0.8, 0.3]) / np.linalg.norm([0.4, 0.8, 0.3])),
                       "cosMax": math.cos(math.radians(0.53 / 2)), "radiance": [20000.0, 19000.0, 17000.0]},
                      {"kind": 1, "pos": [0.0, 3.0, 2.0], "radius": 0.2, "radiance": [40.0, 35.0, 30.0]}]}
    return sc, env, mover
