"""The display post (src/demo/post.js) on a B200 against the oracle: composited HDR image bit-exact, bloom levels and
the final colour within the fast-math / rounding-flip tolerance, 8-bit targets within one step."""
import numpy as np
import pytest

import oracle
from hush_b200 import HushError, Post

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _hdr(h, w, seed):
    rng = np.random.default_rng(seed)
    a = rng.exponential(0.4, (h, w, 4)).astype(np.float32)
    a[rng.random((h, w)) < 0.01, :3] *= 60.0      # fireflies for the Karis average
    a[rng.random((h, w)) < 0.01, :3] *= -1.0      # negative values are clamped by COMPOSITE
    a[..., 3] = 1.0
    return a.astype(np.float16)


def _check(post, want, got, out_fmt):
    np.testing.assert_array_equal(post.buffer(0).cpu().numpy().view(np.uint16), want["hdr"].view(np.uint16))
    for i, lev in enumerate(want["levels"]):
        g = post.buffer(i + 1).cpu().numpy()[..., :3].astype(np.float32)
        w = lev[..., :3].astype(np.float32)
        # f32 sums in another order, then a round-toward-zero f16 store: a 1-ulp flip is 2^-10 relative
        assert np.abs(g - w).max() <= 4e-3 * max(1.0, np.abs(w).max()), (i, np.abs(g - w).max())
    if out_fmt == "rgba32float":
        np.testing.assert_allclose(got, want["f32"], atol=2e-3, rtol=0)
    else:
        g = got.astype(np.int16)
        if out_fmt == "bgra8unorm":
            g = g[..., [2, 1, 0, 3]]
        d = np.abs(g - want["rgba8"].astype(np.int16))
        assert d.max() <= 1 and (d > 0).mean() < 0.01, (d.max(), (d > 0).mean())


@pytest.mark.parametrize("fmt", ["rgba8unorm", "bgra8unorm", "rgba32float"])
def test_two_panels_match_the_oracle(fmt):
    H, W = 61, 97
    left, right = _hdr(H, W, 1), _hdr(H, W, 2)
    post = Post(0, fmt)
    got = post.encode(torch.from_numpy(left).cuda(), torch.from_numpy(right).cuda(), split=0.4, exposure=1.5)
    torch.cuda.synchronize()
    want = oracle.post(left, right, split=0.4, exposure=1.5)
    _check(post, want, got.cpu().numpy(), fmt)


def test_three_panels_same_region_scaled_target():
    H, W = 90, 160
    imgs = [_hdr(H, W, s) for s in (3, 4, 5)]
    post = Post(0, "rgba32float", bloom=0.2, vignette=0.6)
    t = [torch.from_numpy(a).cuda() for a in imgs]
    got = post.encode(t[0], t[2], mid=t[1], split=1 / 3, split2=2 / 3, same=True, width=211, height=117, line=2.0)
    torch.cuda.synchronize()
    want = oracle.post(imgs[0], imgs[2], imgs[1], split=1 / 3, split2=2 / 3, same=True, out_size=(211, 117),
                       line=2.0, bloom=0.2, vignette=0.6)
    _check(post, want, got.cpu().numpy(), "rgba32float")


def test_strength_setters_and_resize():
    post = Post(0, "rgba32float")
    for (H, W) in ((40, 64), (33, 17), (40, 64)):
        a = _hdr(H, W, H + W)
        post.bloom, post.vignette = 0.5, 0.1
        got = post.encode(torch.from_numpy(a).cuda(), torch.from_numpy(a).cuda())
        torch.cuda.synchronize()
        want = oracle.post(a, a, bloom=0.5, vignette=0.1)
        _check(post, want, got.cpu().numpy(), "rgba32float")


def test_errors():
    post = Post(0)
    a = torch.zeros((8, 8, 4), dtype=torch.float16, device="cuda")
    b = torch.zeros((8, 9, 4), dtype=torch.float16, device="cuda")
    with pytest.raises(HushError, match="'right' is 9x8, expected 8x8"):
        post.encode(a, b)
    with pytest.raises(HushError, match="must be a contiguous CUDA"):
        post.encode(a, a.float())
    with pytest.raises(HushError, match="unknown target format"):
        Post(0, "rgb565")
    with pytest.raises(HushError, match="target must be"):
        post.encode(a, a, target=torch.zeros((8, 8, 4), dtype=torch.float32, device="cuda"))


@pytest.mark.parametrize("fmt", ["rgba8unorm", "rgba32float"])
def test_even_size_takes_the_separable_bloom_path(fmt):
    # target = HDR size = twice the first bloom level: FINAL reads the HDR texel directly and the bloom through the
    # 4 x 4 separable form of its nine bilinear taps
    H, W = 96, 160
    left, right = _hdr(H, W, 7), _hdr(H, W, 8)
    post = Post(0, fmt, bloom=0.4)
    got = post.encode(torch.from_numpy(left).cuda(), torch.from_numpy(right).cuda(), split=0.3)
    torch.cuda.synchronize()
    want = oracle.post(left, right, split=0.3, bloom=0.4)
    _check(post, want, got.cpu().numpy(), fmt)
