"""Known-answer tests of the CPU oracle (CPU only).

The reference has no tests or fixtures for this path, so the oracle is pinned by invariants of its WGSL
(src/denoise/hush.js) and by the byte-exact weight blob; tests/golden/oracle_seq.npz pins it against regressions.
"""
import hashlib
import os

import numpy as np
import pytest

import oracle
from hush_b200 import builtin_weights, scene
from hush_b200.hush import WEIGHTS_PATH

from .util import mismatch

HERE = os.path.dirname(os.path.abspath(__file__))


def _f32bits(x):
    return np.asarray(x, dtype=np.float32).view(np.uint32)


# ---------------------------------------------------------------------------------------------------- f16 helpers
def test_qf16_is_the_wgsl_mask():
    # qf16 (hush.js:68, 99): clamp to +-65504 then clear the low 13 mantissa bits
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.normal(0, 10, 2000), rng.uniform(-1e6, 1e6, 200), [0.0, -0.0, 65504.0, 1e9, -1e9]])
    for x in xs.astype(np.float32):
        c = np.float32(min(max(float(x), -65504.0), 65504.0))
        want = (_f32bits(c) & np.uint32(0xFFFFE000)).view(np.float32)
        assert oracle.qf16(float(x)) == float(want)


def test_f2h_rz_matches_truncation_in_the_normal_range():
    rng = np.random.default_rng(1)
    xs = rng.uniform(-60000, 60000, 5000).astype(np.float32)
    xs = xs[np.abs(xs) >= 2.0 ** -14]
    for x in xs[:2000]:
        trunc = np.float32((_f32bits(x) & np.uint32(0xFFFFE000)).view(np.float32))
        assert oracle.f2h_rz(float(x)) == int(np.float16(trunc).view(np.uint16))


def test_f2h_rz_subnormals_overflow_and_specials():
    assert oracle.f2h_rz(2.0 ** -24) == 1
    assert oracle.f2h_rz(2.0 ** -24 * 1.99) == 1  # toward zero
    assert oracle.f2h_rz(2.0 ** -25) == 0
    assert oracle.f2h_rz(3.0 * 2.0 ** -20) == 48
    assert oracle.f2h_rz(70000.0) == 0x7BFF  # round toward zero never reaches infinity
    assert oracle.f2h_rz(-70000.0) == 0xFBFF
    assert oracle.f2h_rz(float("inf")) == 0x7C00
    for h in (0, 1, 0x3C00, 0x7BFF, 0x8001, 0xC000):
        assert oracle.f2h_rz(oracle.h2f(h)) == h


# ---------------------------------------------------------------------------------------------------- weights / MLP
def test_builtin_weight_blob_is_pinned():
    blob = open(WEIGHTS_PATH, "rb").read()
    assert len(blob) == 1624
    assert hashlib.sha256(blob).hexdigest() == "728d4cb712ee4bedbf87b12b263de19a0c6318e41b27d57dfbbc6b68388bd0b5"
    w = builtin_weights().view(np.float16).astype(np.float32)
    assert w.size == 812
    assert abs(float(np.abs(w).max()) - 30.765625) < 1e-6


@pytest.mark.parametrize("h,n", [(16, 812), (8, 348), (32, 2124), (1, 47), (0, 813), (0, 0)])
def test_hidden_of(h, n):
    # n = h^2 + 34 h + 12 (hush.js:21-25)
    assert oracle.lib().ho_hidden_of(n) == h


def _np_mlp(w, f, h=16):
    W1 = w[: h * 20].reshape(h, 20)
    b1 = w[h * 20: h * 21]
    o = h * 21
    W2 = w[o: o + h * h].reshape(h, h)
    b2 = w[o + h * h: o + h * h + h]
    o = o + h * h + h
    W3 = w[o: o + 12 * h].reshape(12, h)
    b3 = w[o + 12 * h: o + 12 * h + 12]
    h1 = np.maximum(b1 + W1 @ f, 0)
    h2 = np.maximum(b2 + W2 @ h1, 0)
    return b3 + W3 @ h2


def test_mlp_against_fp64_dot_products():
    w16 = builtin_weights()
    w = w16.view(np.float16).astype(np.float64)
    rng = np.random.default_rng(2)
    for _ in range(50):
        f = rng.normal(0, 1, 20).astype(np.float16).astype(np.float32)
        ref = _np_mlp(w, f.astype(np.float64))
        o32 = oracle.mlp(w16, f, fp64=False)
        o64 = oracle.mlp(w16, f, fp64=True)
        assert np.allclose(o64, ref, rtol=1e-6, atol=1e-6)
        assert np.allclose(o32, ref, rtol=1e-4, atol=1e-4)


# ---------------------------------------------------------------------------------------------------- invariants
def _flat_inputs(W, H, illum=0.5, albedo=(0.6, 0.4, 0.2), depth=5.0, emission=(0.0, 0.0, 0.0), sky=None):
    rad = np.zeros((H, W, 4), np.float16)
    rad[..., 0] = illum * albedo[0]
    rad[..., 1] = illum * albedo[1]
    rad[..., 2] = illum * albedo[2]
    rad[..., 3] = 1
    nd = np.zeros((H, W, 4), np.float16)
    nd[..., 1] = 1.0
    nd[..., 3] = depth
    mv = np.zeros((H, W, 4), np.float16)
    mv[..., 2] = 7
    mv[..., 3] = depth
    mat = np.zeros((H, W, 4), np.float16)
    mat[..., 0], mat[..., 1], mat[..., 2], mat[..., 3] = albedo[0], albedo[1], albedo[2], 0.5
    emi = np.zeros((H, W, 4), np.float16)
    emi[..., 0], emi[..., 1], emi[..., 2] = emission
    if sky is not None:
        nd[..., 3][sky] = -1
    return {"radiance": rad, "normalDepth": nd, "motion": mv, "material": mat, "emission": emi}


def test_sky_pixels_output_their_emission():
    # sky (depth < 0): FINE_FINAL writes X = (emission, 0) (hush.js:576); a reset frame's TAA passes X through
    W, H = 24, 16
    sky = np.zeros((H, W), bool)
    sky[:, :8] = True
    inp = _flat_inputs(W, H, emission=(0.25, 0.5, 0.75), sky=sky)
    o = oracle.OracleHush(W, H, builtin_weights())
    out = o.denoise(inp).astype(np.float32)
    X = o.buffer("X").astype(np.float32)
    assert np.array_equal(X[sky][:, :3], inp["emission"][sky][:, :3].astype(np.float32))
    # itm(tm(e)) round trip within f16 storage
    assert np.allclose(out[sky][:, :3], X[sky][:, :3], rtol=4e-3)
    assert np.all(out[..., 3] == 1.0)


def test_reset_frame_has_no_history():
    # reset: TEMPORAL skips reprojection (hush.js:149), so has = false, len = 1, moments = (l, l^2, l)
    W, H = 16, 8
    inp = _flat_inputs(W, H, illum=0.5)
    o = oracle.OracleHush(W, H, builtin_weights())
    o.denoise(inp)
    mom = o.buffer("MOM0").astype(np.float32)
    l = 0.5 * (0.2126 + 0.7152 + 0.0722)
    assert np.allclose(mom[..., 0], l, rtol=2e-3)
    assert np.allclose(mom[..., 1], l * l, rtol=2e-3)
    assert np.allclose(mom[..., 2], l, rtol=2e-3)
    assert np.all(mom[..., 3] == 1.0)


@pytest.mark.parametrize("fp64", [False, True])
def test_constant_illumination_is_a_fixed_point(fp64):
    # a flat plane under constant illumination: every a-trous level normalises its weights (hush.js:473), the
    # joint-bilateral upsampling of constant levels is constant, so the output is illumination x albedo
    W, H = 37, 21
    albedo = (0.6, 0.4, 0.2)
    inp = _flat_inputs(W, H, illum=0.5, albedo=albedo)
    o = oracle.OracleHush(W, H, builtin_weights(), fp64=fp64)
    for _ in range(4):
        out = o.denoise(inp).astype(np.float32)
    want = 0.5 * np.array(albedo, np.float32)
    assert np.allclose(out[..., :3], want, rtol=5e-3)


def test_f32_oracle_tracks_the_fp64_oracle():
    cfg = scene.SceneConfig(96, 64, 4, seed=3)
    o32 = oracle.OracleHush(cfg.width, cfg.height, builtin_weights())
    o64 = oracle.OracleHush(cfg.width, cfg.height, builtin_weights(), fp64=True)
    for i in range(cfg.frames):
        f = scene.frame_host(cfg, i)
        a, b = o32.denoise(f), o64.denoise(f)
        frac, _, _ = mismatch(a, b, rel=2e-2)
        assert frac < 0.01, (i, frac)


def test_oracle_reproduces_the_committed_fixture():
    g = np.load(os.path.join(HERE, "golden", "oracle_seq.npz"))
    H, W = g["out0"].shape[:2]
    o = oracle.OracleHush(W, H, builtin_weights())
    n = sum(1 for k in g.files if k.startswith("out"))
    for i in range(n):
        inp = {k: g[f"in{i}_{k}"] for k in oracle.INPUTS}
        out = o.denoise(inp)
        assert np.array_equal(out.view(np.uint16), g[f"out{i}"].view(np.uint16)), i
    for name in ("A0", "X", "BH0", "C0", "CG", "F0", "F1", "F2", "F3"):
        assert np.array_equal(o.buffer(name).view(np.uint16), g[f"last_{name}"].view(np.uint16)), name


def test_generator_inputs_are_the_fixture_inputs():
    # the host scene generator is deterministic: the fixture's inputs regenerate bit for bit
    g = np.load(os.path.join(HERE, "golden", "oracle_seq.npz"))
    H, W = g["out0"].shape[:2]
    cfg = scene.SceneConfig(W, H, 4, n_objects=6, n_moving=2, pan_min=1.0, pan_max=3.0, seed=7)
    f = scene.frame_host(cfg, 2)
    for k in oracle.INPUTS:
        assert np.array_equal(f[k].view(np.uint16), g[f"in2_{k}"].view(np.uint16)), k


def test_svgf_oracle_runs_and_resets():
    cfg = scene.SceneConfig(48, 32, 3, seed=5)
    s = oracle.OracleSVGF(cfg.width, cfg.height)
    prev = None
    for i in range(cfg.frames):
        f = scene.frame_host(cfg, i)
        g = dict(f)
        g["prevNormalDepth"] = (prev or f)["normalDepth"]
        g["prevMotion"] = (prev or f)["motion"]
        out = s.encode(g).astype(np.float32)
        assert np.isfinite(out).all()
        assert np.all(out[..., 3] == 1.0)
        prev = f


def test_f2h_rne_matches_numpy_round_to_nearest_even():
    rng = np.random.default_rng(7)
    xs = np.concatenate([
        rng.normal(scale=s, size=2000).astype(np.float32) for s in (1e-7, 1e-5, 1e-2, 1.0, 1e3, 6e4)
    ] + [np.array([0.0, -0.0, 65504.0, 65519.99, 65520.0, 1e9, -1e9, 2.0 ** -24, 2.0 ** -25, 3 * 2.0 ** -26,
                   np.inf, -np.inf], np.float32)])
    got = np.array([oracle.f2h_rne(float(x)) for x in xs], np.uint16)
    np.testing.assert_array_equal(got, xs.astype(np.float16).view(np.uint16))


def test_oracle_scene_generator_is_the_product_generator_bit_for_bit():
    """The CPU timing arm generates its frames with the oracle library's build of scene.h; they must be the frames
    the product's generator makes (the device generator is checked against the host one in the GPU tests)."""
    from hush_b200 import scene

    for cfg, frames in ((scene.SceneConfig(96, 64, 3, n_moving=2, pan_min=0.0, pan_max=4.0, cut_frame=2, seed=3),
                         (0, 1, 2)),
                        (scene.CONFIG_1080P.with_(width=160, height=90), (0, 31, 32))):
        for i in frames:
            a = oracle.scene_frame(cfg, i, clean=True)
            b = scene.frame_host(cfg, i, clean=True)
            for k in oracle.INPUTS:
                np.testing.assert_array_equal(a[k].view(np.uint16), b[k].view(np.uint16), err_msg=f"{k} frame {i}")
            np.testing.assert_array_equal(a["clean"], b["clean"])


def _mlp_half_numpy(w16: np.ndarray, f: np.ndarray) -> np.ndarray:
    """mlpCode with f16 = true (hush.js:683-703) restated with numpy's correctly rounded float64 -> float16
    conversion: each product and each running sum rounds to f16 (ties to even) in the WGSL's order."""
    w = w16.view(np.float16).astype(np.float64)
    h = int(round((-34 + np.sqrt(34 * 34 - 4 * (12 - w.size))) / 2))
    W1, B1 = 0, 20 * h
    W2, B2 = B1 + h, B1 + h + h * h
    W3, B3 = B2 + h, B2 + h + 12 * h
    r = lambda v: float(np.float16(v))  # noqa: E731

    def layer(x, nin, wo, bo, nout, relu):
        out = []
        for j in range(nout):
            a = w[bo + j]
            for i in range(nin):
                a = r(a + r(x[i] * w[wo + j * nin + i]))
            out.append(max(a, 0.0) if relu else a)
        return out

    x = [r(v) for v in f]
    h1 = layer(x, 20, W1, B1, h, True)
    h2 = layer(h1, h, W2, B2, h, True)
    return np.array(layer(h2, h, W3, B3, 12, False), np.float32)


def test_f16_arithmetic_mlp_matches_a_numpy_restatement():
    w = builtin_weights()
    rng = np.random.default_rng(11)
    for scale in (0.5, 2.0, 8.0):
        f = (rng.normal(size=20) * scale).astype(np.float16).astype(np.float32)
        got = oracle.mlp(w, f, half=True)
        np.testing.assert_array_equal(got, _mlp_half_numpy(w, f))
        # f16 arithmetic stays near the f32 form (the hidden sums carry 11 bits)
        ref = oracle.mlp(w, f)
        assert np.max(np.abs(got - ref)) <= 2e-2 * max(1.0, np.max(np.abs(ref)))
