"""The C ABI library loads, exports every function include/hush.h declares, and its host-only entry points work
without a GPU (CPU only; no kernel is launched)."""
import ctypes as C
import os
import re

import numpy as np

from hush_b200 import _lib as L
from hush_b200 import scene

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "hush.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*([a-z][a-z0-9_]*)\s*\(", text, re.M):
        names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_surface():
    names = _declared_functions()
    for n in ("hush_create", "hush_denoise", "hush_resize", "hush_reset", "hush_set_exposure", "hush_set_weights",
              "hush_hidden_of", "hush_destroy", "hush_last_error", "svgf_create", "svgf_encode"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(L.LIB_PATH)
    missing = [n for n in _declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_every_declared_symbol():
    from hush_b200 import pt

    bound = set(L._SIGS) | set(pt._SIGS)
    assert set(_declared_functions()) <= bound, set(_declared_functions()) - bound
    pt.lib()  # every path-tracer signature resolves in the library


def test_hidden_of_through_the_abi():
    lib = L.lib()
    assert lib.hush_hidden_of(812) == 16
    assert lib.hush_hidden_of(348) == 8
    assert lib.hush_hidden_of(813) == 0


def test_desc_defaults_and_limits():
    lib = L.lib()
    d = lib.hush_desc_default(640, 360)
    assert (d.width, d.height, d.exposure, d.mlp_mode, d.schedule, d.device) == (640, 360, 1.0, 0, 0, -1)
    a, b, s = C.c_int(), C.c_int(), C.c_size_t()
    lib.hush_required_limits(C.byref(a), C.byref(b), C.byref(s))
    assert (a.value, b.value) == (10, 0)
    o = lib.svgf_options_default()
    assert (o.iterations, o.sigma_l, o.sigma_n, o.sigma_z, o.taa) == (5, 4.0, 128.0, 1.0, 1)
    assert abs(o.alpha_color - 0.2) < 1e-7 and abs(o.taa_alpha - 0.1) < 1e-7


def test_null_arguments_are_rejected_without_a_device():
    lib = L.lib()
    assert lib.hush_create(None, None) == L.HUSH_ERR_ARG
    assert b"NULL" in lib.hush_global_error()
    assert lib.hush_reset(None) == L.HUSH_ERR_ARG
    assert lib.hush_denoise(None, None, None, None) == L.HUSH_ERR_ARG
    assert lib.svgf_create(0, 0, None, -1, C.byref(C.c_void_p())) == L.HUSH_ERR_ARG
    assert b"bad size" in lib.svgf_last_error(None)


def test_scene_generator_is_deterministic_and_well_formed():
    cfg = scene.SceneConfig(160, 90, 2, seed=11)
    a = scene.frame_host(cfg, 1, clean=True)
    b = scene.frame_host(cfg, 1, clean=True)
    for k in scene.NAMES:
        assert np.array_equal(a[k].view(np.uint16), b[k].view(np.uint16))
    nd = a["normalDepth"].astype(np.float32)
    sky = nd[..., 3] < 0
    assert 0.03 < sky.mean() < 0.25
    ids = a["motion"][..., 2].astype(np.float32)[~sky]
    assert ids.min() >= 1 and ids.max() < 2048 and np.all(ids == np.round(ids))
    n = np.linalg.norm(nd[..., :3][~sky], axis=-1)
    assert np.allclose(n, 1.0, atol=2e-3)
    alb = a["material"][..., :3].astype(np.float32)[~sky]
    assert alb.min() >= 0.05 * 0.6 - 1e-3 and alb.max() <= 0.9 + 1e-3
    assert np.all(a["clean"] >= 0)


def test_node_addon_calls_only_exported_symbols():
    """node/hush_node.c cannot be compiled here (no node / node_api.h); every library function it calls must at
    least be one the library exports."""
    import re

    src = open(os.path.join(ROOT, "node", "hush_node.c")).read()
    called = set(re.findall(r"\b((?:hush|svgf)_[a-z0-9_]+)\s*\(", src))
    defined = set(re.findall(r"\b(?:static\s+)?[a-z_ ]+\*?\s*((?:hush|svgf)_[a-z0-9_]+)\s*\([^;]*\)\s*\{", src))
    lib = L.lib()
    missing = sorted(n for n in called - defined if not hasattr(lib, n))
    assert not missing, missing
    assert {"hush_create", "hush_denoise", "svgf_encode", "hush_required_limits"} <= called
