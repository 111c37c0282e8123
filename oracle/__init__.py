"""CPU oracle of the Hush denoise path: TEST INFRASTRUCTURE ONLY.

Loaded by the tests, by ``__graft_entry__.smoke()`` as the checker and by ``bench.py``'s CPU-baseline leg; never by
the product path (hush_b200). See hush_oracle.h for what it restates and its parity status (unpinned by reference
outputs: the reference ships no golden vectors and cannot run here).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_hush.so")

PASS_NAMES = ["temporal", "infer", "mid2", "mid3", "coarse1", "coarse2", "fine_final", "taa"]
BUF_NAMES = ["A0", "X", "BH0", "BH1", "MOM0", "MOM1", "KEY0", "KEY1", "HIST0", "HIST1", "TAA0", "TAA1",
             "PAR0_0", "PAR0_1", "PAR1", "PAR2", "F0", "F1", "F2", "F3", "C0", "C1", "CG"]
INPUTS = ["radiance", "normalDepth", "motion", "material", "emission"]


class _Inputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("radiance", "normal_depth", "motion", "material", "emission")]


class _SvgfOpts(C.Structure):
    _fields_ = [("iterations", C.c_int), ("sigma_l", C.c_float), ("sigma_n", C.c_float), ("sigma_z", C.c_float),
                ("alpha_color", C.c_float), ("alpha_moments", C.c_float), ("taa_alpha", C.c_float),
                ("taa", C.c_int)]


class _SvgfInputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("radiance", "normal_depth", "motion", "material", "emission",
                                           "prev_normal_depth", "prev_motion")]


class _PostArgs(C.Structure):
    _fields_ = [("left", C.c_void_p), ("right", C.c_void_p), ("mid", C.c_void_p), ("width", C.c_int),
                ("height", C.c_int), ("out_width", C.c_int), ("out_height", C.c_int), ("split", C.c_float),
                ("split2", C.c_float), ("exposure", C.c_float), ("line", C.c_float), ("bloom", C.c_float),
                ("vignette", C.c_float), ("same", C.c_int)]


class _SceneDesc(C.Structure):  # hs_desc of hush_b200/csrc/scene.h
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("n_objects", C.c_int), ("n_moving", C.c_int),
                ("sky_frac", C.c_float), ("pan_min", C.c_float), ("pan_max", C.c_float), ("yaw_deg", C.c_float),
                ("firefly_rate", C.c_float), ("firefly_scale", C.c_float), ("cut_frame", C.c_int),
                ("seed", C.c_uint32)]


POST_LEVELS = 6
WEIGHTS_PATH = os.path.join(os.path.dirname(HERE), "hush_b200", "data", "hush-weights.bin")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing at {LIB_PATH}; run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        sig = {
            "ho_hidden_of": (C.c_int, [C.c_long]),
            "ho_hush_create": (P, [C.c_int, C.c_int, C.c_float, P, C.c_long, C.c_int]),
            "ho_hush_destroy": (None, [P]),
            "ho_hush_reset": (None, [P]),
            "ho_hush_set_exposure": (None, [P, C.c_float]),
            "ho_hush_frame": (C.c_int, [P]),
            "ho_hush_denoise": (P, [P, C.POINTER(_Inputs)]),
            "ho_hush_pass": (C.c_int, [P, C.c_int, C.POINTER(_Inputs)]),
            "ho_hush_end_frame": (None, [P]),
            "ho_hush_buffer": (P, [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "ho_set_threads": (None, [C.c_int]),
            "ho_f2h_rz": (C.c_uint16, [C.c_float]),
            "ho_h2f": (C.c_float, [C.c_uint16]),
            "ho_qf16": (C.c_float, [C.c_float]),
            "ho_mlp": (None, [P, C.c_long, P, P, C.c_int]),
            "ho_svgf_create": (P, [C.c_int, C.c_int, C.POINTER(_SvgfOpts), C.c_int]),
            "ho_svgf_destroy": (None, [P]),
            "ho_svgf_reset": (None, [P]),
            "ho_svgf_encode": (P, [P, C.POINTER(_SvgfInputs)]),
            "ho_post_level_size": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "ho_post": (C.c_int, [C.POINTER(_PostArgs), P, P, P, P]),
            "ho_f2h_rne": (C.c_uint16, [C.c_float]),
            "ho_hush_set_mlp_half": (None, [P, C.c_int]),
            "ho_scene_frame": (C.c_int, [C.POINTER(_SceneDesc), C.c_int, P, P, P, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def set_threads(n: int = 0):
    lib().ho_set_threads(int(n))


def _as_u16(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a)
    return a.view(np.uint16) if a.dtype == np.float16 else a.astype(np.uint16)


class OracleHush:
    """The oracle's Hush instance (mode 0: f32 like the WGSL, mode 1: f64 arithmetic). f16=True is the reference's
    `f16` option: INFER's MLP in f16 arithmetic (hush.js:683-703, 740)."""

    def __init__(self, width, height, weights: np.ndarray, exposure=1.0, fp64=False, f16=False):
        self.w16 = np.ascontiguousarray(weights.astype(np.uint16))
        self.W, self.H = int(width), int(height)
        self._h = lib().ho_hush_create(self.W, self.H, float(exposure), self.w16.ctypes.data, self.w16.size,
                                       1 if fp64 else 0)
        if not self._h:
            raise ValueError("oracle: bad weights or size")
        if f16:
            lib().ho_hush_set_mlp_half(self._h, 1)
        self._keep = None

    def _inputs(self, inputs: dict) -> _Inputs:
        arrs = [np.ascontiguousarray(inputs[n]).view(np.uint16) for n in INPUTS]
        self._keep = arrs
        return _Inputs(*[a.ctypes.data for a in arrs])

    def denoise(self, inputs: dict) -> np.ndarray:
        inp = self._inputs(inputs)
        p = lib().ho_hush_denoise(self._h, C.byref(inp))
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint16)), (self.H, self.W, 4)).view(np.float16).copy()

    def run_pass(self, name: str, inputs: dict | None = None):
        inp = self._inputs(inputs) if inputs is not None else _Inputs()
        lib().ho_hush_pass(self._h, PASS_NAMES.index(name), C.byref(inp))

    def end_frame(self):
        lib().ho_hush_end_frame(self._h)

    def reset(self):
        lib().ho_hush_reset(self._h)

    def set_exposure(self, e):
        lib().ho_hush_set_exposure(self._h, float(e))

    @property
    def frame(self):
        return lib().ho_hush_frame(self._h)

    def buffer(self, name: str) -> np.ndarray:
        """Live view of a state buffer as float16 (h, w, channels)."""
        w, h, c = C.c_int(), C.c_int(), C.c_int()
        p = lib().ho_hush_buffer(self._h, BUF_NAMES.index(name), C.byref(w), C.byref(h), C.byref(c))
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint16)), (h.value, w.value, c.value)).view(np.float16)

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                lib().ho_hush_destroy(self._h)
                self._h = None
        except Exception:  # interpreter shutdown
            pass


class OracleSVGF:
    def __init__(self, width, height, options: dict | None = None, fp64=False):
        o = _SvgfOpts(5, 4.0, 128.0, 1.0, 0.2, 0.2, 0.1, 1)
        names = {"iterations": "iterations", "sigmaL": "sigma_l", "sigmaN": "sigma_n", "sigmaZ": "sigma_z",
                 "alphaColor": "alpha_color", "alphaMoments": "alpha_moments", "taaAlpha": "taa_alpha", "taa": "taa"}
        for k, v in (options or {}).items():
            setattr(o, names[k], int(v) if k in ("iterations", "taa") else float(v))
        self.W, self.H = int(width), int(height)
        self._h = lib().ho_svgf_create(self.W, self.H, C.byref(o), 1 if fp64 else 0)

    def encode(self, inputs: dict) -> np.ndarray:
        names = INPUTS + ["prevNormalDepth", "prevMotion"]
        arrs = [np.ascontiguousarray(inputs[n]).view(np.uint16) for n in names]
        inp = _SvgfInputs(*[a.ctypes.data for a in arrs])
        p = lib().ho_svgf_encode(self._h, C.byref(inp))
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint16)), (self.H, self.W, 4)).view(np.float16).copy()

    def reset(self):
        lib().ho_svgf_reset(self._h)

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                lib().ho_svgf_destroy(self._h)
                self._h = None
        except Exception:  # interpreter shutdown
            pass


def builtin_weights() -> np.ndarray:
    """The reference's built-in weight blob (812 f16 values), read from the data file."""
    return np.fromfile(WEIGHTS_PATH, dtype="<u2")


def scene_frame(cfg, frame: int, clean: bool = False) -> dict:
    """One frame of a synthetic G-buffer sequence (cfg: any object with SceneConfig's fields), generated on the host
    by the oracle library's build of the generator: five (H, W, 4) float16 arrays (+ 'clean' (H, W, 3) float32)."""
    H, W = cfg.height, cfg.width
    bufs = {n: np.empty((H, W, 4), dtype=np.float16) for n in INPUTS}
    cl = np.empty((H, W, 3), dtype=np.float32) if clean else None
    d = _SceneDesc(W, H, cfg.n_objects, cfg.n_moving, cfg.sky_frac, cfg.pan_min, cfg.pan_max, cfg.yaw_deg,
                   cfg.firefly_rate, cfg.firefly_scale, cfg.cut_frame, cfg.seed & 0xFFFFFFFF)
    if lib().ho_scene_frame(C.byref(d), int(frame), *[bufs[n].ctypes.data for n in INPUTS],
                            cl.ctypes.data if clean else None) != 0:
        raise RuntimeError("scene generation failed")
    if clean:
        bufs["clean"] = cl
    return bufs


def f2h_rne(x: float) -> int:
    return int(lib().ho_f2h_rne(float(x)))


def f2h_rz(x: float) -> int:
    return int(lib().ho_f2h_rz(float(x)))


def h2f(h: int) -> float:
    return float(lib().ho_h2f(int(h)))


def qf16(x: float) -> float:
    return float(lib().ho_qf16(float(x)))


def mlp(weights: np.ndarray, features: np.ndarray, fp64=False, half=False) -> np.ndarray:
    """One MLP row: f32 (the default), f64, or half=True for the reference's f16 arithmetic (the `f16` option)."""
    w = np.ascontiguousarray(weights.astype(np.uint16))
    f = np.ascontiguousarray(features.astype(np.float32))
    o = np.zeros(12, dtype=np.float32)
    lib().ho_mlp(w.ctypes.data, w.size, f.ctypes.data, o.ctypes.data, 2 if half else (1 if fp64 else 0))
    return o


def post_level_size(width: int, height: int, level: int):
    w, h = C.c_int(), C.c_int()
    if lib().ho_post_level_size(int(width), int(height), int(level), C.byref(w), C.byref(h)) != 0:
        raise ValueError(f"no post level {level}")
    return w.value, h.value


def post(left, right, mid=None, split=0.5, split2=None, same=False, exposure=1.0, out_size=None, line=1.5,
         bloom=0.03, vignette=0.35):
    """Post.encode of src/demo/post.js on (H, W, 4) float16 arrays. Returns dict with 'hdr' (H, W, 4) float16,
    'levels' (list of six float16 arrays), 'f32' (OH, OW, 4) float32 and 'rgba8' (OH, OW, 4) uint8."""
    Hh, Ww = left.shape[:2]
    OW, OH = out_size or (Ww, Hh)
    arrs = [_as_u16(a) for a in (left, right, mid if mid is not None else right)]
    a = _PostArgs(arrs[0].ctypes.data, arrs[1].ctypes.data, arrs[2].ctypes.data if mid is not None else None,
                  Ww, Hh, OW, OH, split, split if split2 is None else split2, exposure, line, bloom, vignette,
                  1 if same else 0)
    sizes = [post_level_size(Ww, Hh, i) for i in range(1, POST_LEVELS + 1)]
    hdr = np.zeros((Hh, Ww, 4), np.uint16)
    lev = np.zeros(sum(w * h * 4 for w, h in sizes), np.uint16)
    f32 = np.zeros((OH, OW, 4), np.float32)
    u8 = np.zeros((OH, OW, 4), np.uint8)
    if lib().ho_post(C.byref(a), hdr.ctypes.data, lev.ctypes.data, f32.ctypes.data, u8.ctypes.data) != 0:
        raise ValueError("oracle post: bad arguments")
    levels, o = [], 0
    for w, h in sizes:
        levels.append(lev[o:o + w * h * 4].reshape(h, w, 4).view(np.float16))
        o += w * h * 4
    return {"hdr": hdr.view(np.float16), "levels": levels, "f32": f32, "rgba8": u8}
