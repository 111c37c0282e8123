"""Known-answer checks of the display-post oracle (oracle/post_oracle.cpp, restating src/demo/post.js) on the CPU."""
import numpy as np
import pytest

import oracle


def _const(h, w, v):
    a = np.zeros((h, w, 4), np.float16)
    a[..., :3] = v
    a[..., 3] = 1
    return a


def test_level_sizes_follow_resize():
    # post.js:165-167: max(1, size >> i) for i = 1..6
    assert [oracle.post_level_size(97, 61, i) for i in range(1, 7)] == [(48, 30), (24, 15), (12, 7), (6, 3), (3, 1),
                                                                         (1, 1)]
    assert oracle.post_level_size(1, 1, 6) == (1, 1)
    with pytest.raises(ValueError):
        oracle.post_level_size(8, 8, 7)


def test_bloom_chain_of_a_constant_image():
    # DOWN and UP weights sum to 1, so every level holds c after the downsample chain; the upsample adds level i+1
    # onto level i from the coarsest up, so level i ends at (7 - i) c. c = 0.25 keeps every sum exact in f16.
    c = _const(64, 128, 0.25)
    r = oracle.post(c, c, bloom=0.0, vignette=0.0)
    for i, lev in enumerate(r["levels"]):
        np.testing.assert_array_equal(lev[..., :3].astype(np.float32), 0.25 * (6 - i))
    np.testing.assert_array_equal(r["hdr"], c)


def _agx_srgb64(c):
    """float64 restatement of agx() and srgb() of post.js:90-115 (columns of the WGSL mat3x3f constructors)."""
    to2020 = np.array([[0.6274, 0.0691, 0.0164], [0.3293, 0.9195, 0.0880], [0.0433, 0.0113, 0.8956]]).T
    to_srgb = np.array([[1.6605, -0.1246, -0.0182], [-0.5876, 1.1329, -0.1006], [-0.0728, -0.0083, 1.1187]]).T
    inset = np.array([[0.856627153315983, 0.137318972929847, 0.11189821299995],
                      [0.0951212405381588, 0.761241990602591, 0.0767994186031903],
                      [0.0482516061458583, 0.101439036467562, 0.811302368396859]]).T
    outset = np.array([[1.1271005818144368, -0.1413297634984383, -0.14132976349843826],
                       [-0.11060664309660323, 1.157823702216272, -0.11060664309660294],
                       [-0.016493938717834573, -0.016493938717834257, 1.2519364065950405]]).T
    lo, hi = -12.47393, 4.026069
    x = inset @ (to2020 @ np.asarray(c, np.float64))
    x = np.clip((np.log2(np.maximum(x, 1e-10)) - lo) / (hi - lo), 0, 1)
    x = 15.5 * x ** 6 - 40.14 * x ** 5 + 31.96 * x ** 4 - 6.868 * x ** 3 + 0.4298 * x ** 2 + 0.1191 * x - 0.00232
    lum = x @ np.array([0.2126, 0.7152, 0.0722])
    x = np.maximum(x, 0) ** 1.22
    x = lum + (x - lum) * 1.15
    x = np.maximum(outset @ x, 0) ** 2.2
    x = np.clip(to_srgb @ x, 0, 1)
    return np.where(x <= 0.0031308, x * 12.92, 1.055 * x ** (1 / 2.4) - 0.055)


@pytest.mark.parametrize("v", [0.0, 0.02, 0.18, 1.0, 6.0])
def test_tone_curve_against_a_float64_restatement(v):
    c = _const(16, 32, v)
    r = oracle.post(c, c, bloom=0.0, vignette=0.0, line=0.0)
    want = _agx_srgb64([float(np.float16(v))] * 3)
    np.testing.assert_allclose(r["f32"][..., :3], np.broadcast_to(want, (16, 32, 3)), atol=2e-5)
    assert (r["f32"][..., 3] == 1).all() and (r["rgba8"][..., 3] == 255).all()
    np.testing.assert_array_equal(r["rgba8"][..., :3], np.rint(np.clip(r["f32"][..., :3], 0, 1) * 255))


def test_composite_panels_and_exposure():
    W, H = 90, 8
    left, mid, right = _const(H, W, 1.0), _const(H, W, 2.0), _const(H, W, 3.0)
    right[0, 0, :3] = -4.0  # negative radiance is clamped to 0 before the exposure (post.js:37)
    r = oracle.post(left, right, mid, split=0.25, split2=0.6, exposure=0.5)
    u = (np.arange(W) + 0.5) / W
    want = np.where(u < 0.25, 1.0, np.where(u < 0.6, 2.0, 3.0)) * 0.5
    got = r["hdr"][..., 0].astype(np.float32)
    np.testing.assert_array_equal(got[1], want)
    assert got[0, 0] == 0.5 and r["hdr"][0, W - 1, 0] == 1.5
    r2 = oracle.post(left, right, mid, split=0.25, split2=0.6, exposure=0.5)
    assert r2["hdr"][0, 0, 0] == 0.5  # deterministic


def test_same_mode_shows_the_middle_third_in_every_panel():
    W, H = 99, 4
    ramp = np.zeros((H, W, 4), np.float16)
    ramp[..., 0] = np.arange(W, dtype=np.float16)[None, :]
    r = oracle.post(ramp, ramp, ramp, split=1 / 3, split2=2 / 3, same=True)
    x = np.arange(W)
    src = x - (np.minimum(x * 3 // W, 2) - 1) * (W // 3)
    np.testing.assert_array_equal(r["hdr"][0, :, 0].astype(np.float32), src.astype(np.float32))
    assert src.min() >= W // 3 and src.max() < 2 * W // 3 + 1


def test_divider_line_is_drawn_at_the_split():
    c = _const(8, 200, 0.05)
    r = oracle.post(c, c, split=0.5, line=1.5, vignette=0.0, bloom=0.0)
    row = r["f32"][4, :, 0]
    assert row[99] > 0.85 and row[100] > 0.85       # |u - 0.5| * 200 = 0.5 < 1.5
    assert row[97] < 0.5 and row[102] < 0.5          # 2.5 and 2.5 px away
