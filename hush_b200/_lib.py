"""ctypes bindings of the C ABI in include/hush.h (libhush_b200.so, built in-tree by hush_b200/build.py)."""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libhush_b200.so")

HUSH_OK, HUSH_ERR_ARG, HUSH_ERR_DEVICE, HUSH_ERR_CUDA, HUSH_ERR_KERNEL = 0, 1, 2, 3, 4
MLP_FP32, MLP_BF16, MLP_F16, MLP_HALF = 0, 1, 2, 3
SCHED_FUSED, SCHED_PASSES = 0, 1
PASS_NAMES = ["temporal", "infer", "mid2", "mid3", "coarse1", "coarse2", "fine_final", "taa"]
BUF_NAMES = ["A0", "X", "BH0", "BH1", "MOM0", "MOM1", "KEY0", "KEY1", "HIST0", "HIST1", "TAA0", "TAA1",
             "PAR0_0", "PAR0_1", "PAR1", "PAR2", "F0", "F1", "F2", "F3", "C0", "C1", "CG"]
BUF = {n: i for i, n in enumerate(BUF_NAMES)}


class HushDesc(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("exposure", C.c_float),
                ("weights", C.POINTER(C.c_uint16)), ("n_weights", C.c_size_t), ("f16", C.c_int),
                ("mlp_mode", C.c_int), ("schedule", C.c_int), ("device", C.c_int)]


class HushInputs(C.Structure):
    _fields_ = [("radiance", C.c_void_p), ("normal_depth", C.c_void_p), ("motion", C.c_void_p),
                ("material", C.c_void_p), ("emission", C.c_void_p), ("width", C.c_int * 5),
                ("height", C.c_int * 5), ("pitch", C.c_size_t * 5)]


class HushTiming(C.Structure):
    _fields_ = [("label", C.c_char_p), ("ms", C.c_float)]


class SvgfOptions(C.Structure):
    _fields_ = [("iterations", C.c_int), ("sigma_l", C.c_float), ("sigma_n", C.c_float), ("sigma_z", C.c_float),
                ("alpha_color", C.c_float), ("alpha_moments", C.c_float), ("taa_alpha", C.c_float),
                ("taa", C.c_int)]


class SvgfInputs(C.Structure):
    _fields_ = [("radiance", C.c_void_p), ("normal_depth", C.c_void_p), ("motion", C.c_void_p),
                ("material", C.c_void_p), ("emission", C.c_void_p), ("prev_normal_depth", C.c_void_p),
                ("prev_motion", C.c_void_p), ("pitch", C.c_size_t * 7)]


class HushScene(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("n_objects", C.c_int), ("n_moving", C.c_int),
                ("sky_frac", C.c_float), ("pan_min", C.c_float), ("pan_max", C.c_float), ("yaw_deg", C.c_float),
                ("firefly_rate", C.c_float), ("firefly_scale", C.c_float), ("cut_frame", C.c_int),
                ("seed", C.c_uint32)]


class HushPostDesc(C.Structure):
    _fields_ = [("device", C.c_int), ("format", C.c_int), ("bloom", C.c_float), ("vignette", C.c_float)]


class HushPostInputs(C.Structure):
    _fields_ = [("left", C.c_void_p), ("right", C.c_void_p), ("mid", C.c_void_p), ("width", C.c_int),
                ("height", C.c_int), ("split", C.c_float), ("split2", C.c_float), ("exposure", C.c_float),
                ("line", C.c_float), ("same", C.c_int)]


# the training twin's passes (hush_twin_pass) and buffers (hush_trainer_buf)
TWIN_PASSES = ["mlp", "mid1", "mid2", "mid3", "fine", "taa", "loss", "temporal", "coarse1", "coarse2"]
TWIN_BUF_NAMES = ["THETA", "GRAD", "LOSS", "PAR", "DPAR", "B1", "B2", "B3", "DB1", "DB2", "DB3", "A1", "X", "DX", "OUT",
                  "OUT_PREV", "DOUT", "DA0", "DA1", "DMOM", "DHIST", "DMOM_PREV", "DAG", "AH", "DAH", "C1", "DC1", "C0",
                  "DC0"]

POST_LEVELS = 6
POST_RGBA8, POST_BGRA8, POST_RGBA32F = 0, 1, 2

_P = C.c_void_p
_SIGS = {
    "hush_hidden_of": (C.c_int, [C.c_long]),
    "hush_desc_default": (HushDesc, [C.c_int, C.c_int]),
    "hush_required_limits": (None, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_size_t)]),
    "hush_create": (C.c_int, [C.POINTER(HushDesc), C.POINTER(_P)]),
    "hush_destroy": (None, [_P]),
    "hush_resize": (C.c_int, [_P, C.c_int, C.c_int]),
    "hush_reset": (C.c_int, [_P]),
    "hush_set_exposure": (C.c_int, [_P, C.c_float]),
    "hush_get_exposure": (C.c_float, [_P]),
    "hush_set_weights": (C.c_int, [_P, C.POINTER(C.c_uint16), C.c_size_t]),
    "hush_set_mlp_mode": (C.c_int, [_P, C.c_int]),
    "hush_set_schedule": (C.c_int, [_P, C.c_int]),
    "hush_get_size": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hush_get_hidden": (C.c_int, [_P]),
    "hush_get_frame": (C.c_int, [_P]),
    "hush_denoise": (C.c_int, [_P, C.POINTER(HushInputs), _P, C.POINTER(_P)]),
    "hush_output": (_P, [_P]),
    "hush_denoise_host": (C.c_int, [_P, C.POINTER(HushInputs), _P, C.c_size_t, _P]),
    "hush_host_join": (C.c_int, [_P, _P]),
    "hush_timer_enable": (C.c_int, [_P, C.c_int]),
    "hush_timer_read": (C.c_int, [_P, C.POINTER(HushTiming), C.c_int]),
    "hush_set_graph": (C.c_int, [_P, C.c_int]),
    "hush_kernel_status": (C.c_int, [_P, C.POINTER(C.c_uint)]),
    "hush_selftest_wait": (C.c_int, [_P, C.c_uint32, _P]),
    "hush_last_error": (C.c_char_p, [_P]),
    "hush_global_error": (C.c_char_p, []),
    "hush_run_pass": (C.c_int, [_P, C.c_int, C.POINTER(HushInputs), _P]),
    "hush_end_frame": (C.c_int, [_P]),
    "hush_buffer": (C.c_int, [_P, C.c_int, C.POINTER(_P), C.POINTER(C.c_int), C.POINTER(C.c_int),
                              C.POINTER(C.c_int)]),
    "hush_trainer_create": (C.c_int, [_P, C.c_void_p, C.POINTER(_P)]),
    "hush_trainer_destroy": (None, [_P]),
    "hush_trainer_frame": (C.c_int, [_P, C.POINTER(HushInputs), C.c_void_p, C.c_void_p, C.c_float, C.c_int, _P,
                                     C.POINTER(C.c_double)]),
    "hush_trainer_end_frame": (C.c_int, [_P]),
    "hush_trainer_loss_sum": (C.c_int, [_P, _P, C.POINTER(C.c_double)]),
    "hush_trainer_reset": (C.c_int, [_P]),
    "hush_trainer_zero_grad": (C.c_int, [_P, _P]),
    "hush_trainer_grad": (C.c_int, [_P, C.c_void_p]),
    "hush_trainer_accumulators": (C.c_int, [_P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "hush_trainer_theta": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "hush_trainer_par": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "hush_trainer_output": (C.c_int, [_P, C.c_void_p]),
    "hush_trainer_step": (C.c_int, [_P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, _P,
                                    C.POINTER(C.c_double)]),
    "hush_trainer_export": (C.c_int, [_P, C.c_void_p]),
    "hush_train_step": (C.c_int, [_P, C.POINTER(HushInputs), C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_float,
                                  C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, _P, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]),
    "hush_trainer_set_mlp": (C.c_int, [_P, C.c_int]),
    "hush_trainer_windows": (C.c_int, [_P, C.POINTER(HushScene), C.POINTER(C.c_uint32), C.c_int, C.c_int,
                                       C.c_float, _P]),
    "hush_trainer_window_bptt": (C.c_int, [_P, C.POINTER(HushInputs), C.POINTER(C.c_void_p), C.c_int, C.c_float,
                                           _P]),
    "hush_trainer_windows_bptt": (C.c_int, [_P, C.POINTER(HushScene), C.POINTER(C.c_uint32), C.c_int, C.c_int,
                                            C.c_float, _P]),
    "hush_trainer_begin": (C.c_int, [_P, C.POINTER(HushInputs), C.c_void_p, C.c_void_p, C.c_float, _P]),
    "hush_trainer_zero_adjoints": (C.c_int, [_P, _P]),
    "hush_trainer_buffer": (C.c_int, [_P, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]),
    "hush_trainer_pass": (C.c_int, [_P, C.c_int, C.c_int, _P]),
    **{f"hush_{p}_{d}": (C.c_int, [_P, _P]) for p in TWIN_PASSES for d in ("fwd", "bwd")},
    "hush_mlp_grad_noalloc": (C.c_int, [C.c_void_p] * 6 + [C.c_int, C.c_int, C.c_void_p, _P]),
    "svgf_options_default": (SvgfOptions, []),
    "svgf_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(SvgfOptions), C.c_int, C.POINTER(_P)]),
    "svgf_destroy": (None, [_P]),
    "svgf_resize": (C.c_int, [_P, C.c_int, C.c_int]),
    "svgf_reset": (C.c_int, [_P]),
    "svgf_encode": (C.c_int, [_P, C.POINTER(SvgfInputs), _P, C.POINTER(_P)]),
    "svgf_output": (_P, [_P]),
    "svgf_last_error": (C.c_char_p, [_P]),
    "hush_post_desc_default": (HushPostDesc, []),
    "hush_post_inputs_default": (HushPostInputs, []),
    "hush_post_create": (C.c_int, [C.POINTER(HushPostDesc), C.POINTER(_P)]),
    "hush_post_destroy": (None, [_P]),
    "hush_post_set": (C.c_int, [_P, C.c_float, C.c_float]),
    "hush_post_encode": (C.c_int, [_P, C.POINTER(HushPostInputs), _P, C.c_int, C.c_int, C.c_size_t, _P]),
    "hush_post_buffer": (_P, [_P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hush_post_last_error": (C.c_char_p, [_P]),
    "hush_scene_frame_host": (C.c_int, [C.POINTER(HushScene), C.c_int] + [C.c_void_p] * 6),
    "hush_scene_frame_device": (C.c_int, [C.POINTER(HushScene), C.c_int] + [C.c_void_p] * 7),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libhush_b200.so (it must have been built: python -m hush_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"hush_b200: native library missing at {LIB_PATH}; run `python -m hush_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
