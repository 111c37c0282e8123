"""Path tracer host logic on the CPU: the product's BVH builder and environment-map preparation against the oracle
(bit for bit), and known-answer checks of the oracle's traversal, refit, alias table, texture LOD and jitter."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle.pt as opt
from hush_b200 import pt


def _soup(n, seed, spread=10.0, size=0.5):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 1, 3))
    return (c + rng.normal(0, size, (n, 3, 3))).astype(np.float32).reshape(n, 9)


@pytest.mark.parametrize("n,seed", [(1, 0), (3, 1), (4, 2), (5, 3), (17, 4), (100, 5), (3000, 6)])
def test_bvh_builder_matches_the_oracle_bit_for_bit(n, seed):
    pos = _soup(n, seed)
    a_nodes, a_order, a_depth = pt.bvh_build(pos)
    b_nodes, b_order, b_depth = opt.bvh_build(pos)
    assert a_depth == b_depth
    np.testing.assert_array_equal(a_order, b_order)
    np.testing.assert_array_equal(a_nodes.view(np.uint32), b_nodes.view(np.uint32))


def test_bvh_builder_degenerate_inputs():
    # all centroids coincide: median splits by index (bvh.js:116-118); a flat grid: one axis without extent
    same = np.tile(np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float32), (40, 1))
    xs, zs = np.meshgrid(np.arange(12, dtype=np.float32), np.arange(12, dtype=np.float32))
    flat = np.stack([xs, 0 * xs, zs, xs + 1, 0 * xs, zs, xs, 0 * xs, zs + 1], -1).reshape(-1, 9)
    for pos in (same, flat):
        a, ao, ad = pt.bvh_build(pos)
        b, bo, bd = opt.bvh_build(pos)
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
        np.testing.assert_array_equal(ao, bo)
        assert ad == bd


def _check_tree(nodes, pos, order):
    u = nodes.view(np.uint32)
    tri = pos[order].reshape(-1, 3, 3)
    seen = np.zeros(len(order), int)
    for i in range(len(nodes)):
        lo, hi, cnt, ref = nodes[i, 0:3], nodes[i, 4:7], u[i, 7], u[i, 3]
        if cnt:
            t = tri[ref:ref + cnt]
            assert (t.min(axis=(0, 1)) >= lo).all() and (t.max(axis=(0, 1)) <= hi).all()
            seen[ref:ref + cnt] += 1
            assert cnt <= 16
        else:
            assert ref > i  # children after the parent (reverse walk = bottom-up)
            for c in (ref, ref + 1):
                assert (nodes[c, 0:3] >= lo).all() and (nodes[c, 4:7] <= hi).all()
    assert (seen == 1).all()


def test_bvh_invariants_and_refit():
    pos = _soup(500, 9)
    nodes, order, _ = opt.bvh_build(pos)
    _check_tree(nodes, pos, order)
    moved = pos + np.random.default_rng(1).normal(0, 2.0, pos.shape).astype(np.float32)
    opt.bvh_refit(nodes, moved[order])
    _check_tree(nodes, moved, order)


def _brute_force(pos, o, d):
    tri = pos.reshape(-1, 3, 3).astype(np.float64)
    best = (1e30, -1)
    for i, (v0, v1, v2) in enumerate(tri):
        e1, e2 = v1 - v0, v2 - v0
        p = np.cross(d, e2)
        det = e1 @ p
        if abs(det) < 1e-12:
            continue
        s = o - v0
        u = (s @ p) / det
        q = np.cross(s, e1)
        v = (d @ q) / det
        t = (e2 @ q) / det
        if u >= 0 and v >= 0 and u + v <= 1 and 1e-4 < t < best[0]:
            best = (t, i)
    return best


def _frame_bytes(blas, lights=()):
    f = pt.PtFrame()
    f.size[:] = [4, 4]
    f.counts[:] = [len(blas), len(lights), 0, 0]
    for i, b in enumerate(blas):
        f.blas[i].node_offset, f.blas[i].tri_offset, f.blas[i].node_count, f.blas[i].flags = b
    return bytes(f)


def _mats(n=1):
    m = np.zeros((n, 20), np.float32)
    m[:, 0:3] = 0.5
    m[:, 8:12] = [1.0, 0.0, 0.0, 1.5]
    m.view(np.int32)[:, 12:15] = -1
    m[:, 16:18] = 1
    return m


def test_oracle_closest_hit_matches_brute_force():
    pos = _soup(300, 11, spread=4.0)
    idx = np.arange(900, dtype=np.uint32).reshape(-1, 3)
    sc = opt.Scene([{"pos": pos.reshape(-1, 3), "idx": idx, "mat": np.zeros(300, np.uint32)}], _mats())
    fb = _frame_bytes(sc.blas)
    rng = np.random.default_rng(3)
    hits = 0
    for _ in range(200):
        o = rng.uniform(-8, 8, 3)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        got = sc.trace(fb, o.astype(np.float32), d.astype(np.float32))
        t, i = _brute_force(pos, o.astype(np.float32).astype(np.float64), d.astype(np.float32).astype(np.float64))
        if i < 0:
            assert got[1] < 0
            continue
        hits += 1
        assert got[1] >= 0
        assert abs(got[0] - t) <= 1e-4 * max(1.0, t)
    assert hits > 20


def test_tri_lod_known_answer():
    # unit right triangle whose uv spans the unit square's half: texel density 1024 per unit -> log2(1024) = 10
    a = np.array([0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0], np.float32)
    b = np.array([1, 0, 0, 1, 1, 0, 0, 0, 0, 0, 0, 0], np.float32)
    c = np.array([0, 1, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1], np.float32)
    assert opt.lib().ho_tri_lod(a.ctypes.data, b.ctypes.data, c.ctypes.data, 1024) == 0x4900  # f16 10.0


def _env_image(seed=0, sun=True):
    rng = np.random.default_rng(seed)
    H, W = 64, 128
    y = (np.arange(H) + 0.5) / H
    img = np.zeros((H, W, 4), np.float32)
    img[..., 0] = (0.2 + 0.8 * (1 - y))[:, None] + rng.uniform(0, 0.05, (H, W))
    img[..., 1] = 0.4 + rng.uniform(0, 0.05, (H, W))
    img[..., 2] = (0.3 + 0.7 * (1 - y))[:, None]
    img[..., 3] = 1
    if sun:
        img[12, 40, :3] = 5000.0
        img[12, 41, :3] = 3000.0
    return img


@pytest.mark.parametrize("sun", [True, False])
def test_env_prepare_matches_the_oracle(sun):
    img = _env_image(sun=sun)
    a = pt.prepare_env_map(img, sun=True)
    b = opt.env_prepare(img, sun=True)
    np.testing.assert_array_equal(a.half, b["half"])
    np.testing.assert_array_equal(a.table.view(np.uint32), b["table"].view(np.uint32))
    if sun:
        assert a.sun is not None and b["sun"] is not None
        np.testing.assert_allclose(a.sun["dir"], b["sun"][0], rtol=0, atol=1e-12)
        np.testing.assert_allclose(a.sun["irradiance"], b["sun"][1], rtol=1e-12)
        # the sun sits at row 12 / 64 of the map: polar angle (12.5 / 64) pi from +y
        assert abs(math.acos(a.sun["dir"][1]) - 12.5 / 64 * math.pi) < 0.05
    else:
        assert a.sun is None and b["sun"] is None


def test_alias_table_reproduces_the_pmf():
    t = pt.prepare_env_map(_env_image(), sun=True).table.reshape(-1, 4)
    N = len(t)
    thr, alias, pmf = t[:, 0].astype(np.float64), t[:, 1].view(np.uint32), t[:, 2].astype(np.float64)
    p = thr / N
    np.add.at(p, alias, (1 - thr) / N)
    np.testing.assert_allclose(p, pmf, atol=1e-6)
    assert abs(pmf.sum() - 1) < 1e-5


def test_env_sun_light():
    m = pt.prepare_env_map(_env_image(), sun=True)
    L = pt.env_sun_light(m, rotation=0.5, scale=2.0)
    assert L["kind"] == 0 and abs(np.linalg.norm(L["dir"]) - 1) < 1e-9
    omega = 2 * math.pi * (1 - L["cosMax"])
    np.testing.assert_allclose(np.array(L["radiance"]) * omega, 2 * np.array(m.sun["irradiance"]))
    assert pt.env_sun_light(pt.prepare_env_map(_env_image(sun=False))) is None


def test_jitter_is_halton_2_3():
    out = (C.c_float * 32)()
    pt.lib().hush_pt_jitter(out)
    prod = np.array(list(out)).reshape(16, 2)
    np.testing.assert_array_equal(prod, opt.jitter())
    np.testing.assert_allclose(prod, np.array(pt.JITTER, np.float32))
    assert tuple(prod[0]) == (0.0, np.float32(1 / 3 - 0.5)) and tuple(prod[1]) == (-0.25, np.float32(2 / 3 - 0.5))


def test_camera_matches_three_js_conventions():
    cam = pt.Camera(position=(0, 2, 10), target=(0, 2, 0), fov=60, aspect=2.0, near=0.1, far=100)
    vp = cam.view_proj().reshape(4, 4).T  # back to row-major
    c = vp @ np.array([0, 2, 0, 1.0])
    assert abs(c[0] / c[3]) < 1e-6 and abs(c[1] / c[3]) < 1e-6 and abs(c[3] - 10) < 1e-5
    # a point at the top edge of the frustum maps to ndc y = 1
    c = vp @ np.array([0, 2 + 5 * math.tan(math.radians(30)), 5, 1.0])
    assert abs(c[1] / c[3] - 1) < 1e-5
    e = cam.elements
    np.testing.assert_allclose(-e[8:11], [0, 0, -1], atol=1e-12)  # forward = -z column
