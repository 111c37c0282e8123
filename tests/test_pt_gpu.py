"""The path tracer on a B200 against the oracle (oracle/pt_oracle.cpp restating pathtracer.wgsl.js):

* the scene buffers the product uploads equal the oracle's own assembly (BVH nodes, triangles, indices bit for bit);
* mode 0 (1 spp + G-buffer): geometry planes (normal, depth, motion, object id, albedo, roughness, primary emission)
  match per pixel; radiance matches per pixel wherever the random path did not branch differently (FMA contraction
  on the GPU moves a few decisions that sit within an ulp of their threshold), and on average;
* mode 1 (accumulated paths), the environment map, textures (albedo, alpha cut-out, normal and ARM maps) and a
  dynamic group re-posed between frames (exact motion vectors) are all covered;
* the G-buffer feeds Hush.denoise end to end.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle.pt as opt
from hush_b200 import Hush, HushError
from hush_b200 import pt

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

W, H = 96, 64


def _download(ptr, nbytes):
    class V:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (int(ptr), False), "version": 3,
                                    "strides": None}
    return torch.as_tensor(V(), device="cuda").cpu().numpy().copy()


def _oracle_scene(sc):
    info = sc.info()
    dev = sc.device_buffers()
    mats = sc.materials_array()
    tex_layers = int(mats.view(np.int32)[:, 12:15].max()) + 1 if mats.size else 0
    tex = _download(dev["tex"], max(1, tex_layers) * _layer_bytes()) if tex_layers > 0 else None
    del info
    return opt.Scene(sc.group_arrays(), mats, tex, tex_layers)


def _layer_bytes():
    return sum(max(1, 1024 >> m) ** 2 * 4 for m in range(11))


def _camera():
    return pt.Camera(position=(1.0, 4.0, 13.0), target=(0.0, 0.8, 0.0), fov=50, aspect=W / H)


def _check_buffers(sc, osc):
    dev = sc.device_buffers()
    info = sc.info()
    nodes = _download(dev["nodes"], info["node_total"] * 64).view(np.uint32)
    np.testing.assert_array_equal(nodes, osc.nodes.view(np.uint32).ravel())
    tris = _download(dev["tris"], info["tri_total"] * 48).view(np.uint32)
    np.testing.assert_array_equal(tris, osc.tris.view(np.uint32).ravel())
    ti = _download(dev["tri_idx"], info["tri_total"] * 16).view(np.uint32)
    np.testing.assert_array_equal(ti, osc.tri_idx.ravel())
    verts = _download(dev["verts"], info["vert_total"] * 48).view(np.float32)
    np.testing.assert_allclose(verts, osc.verts.ravel(), rtol=0, atol=1e-7)


def _gbuf_host(p, slot):
    return [p.gbuf[slot][n].cpu().numpy() for n in pt.GBUF_NAMES]


def _compare_mode0(got, want, rad_frac=0.9):
    g = [a.astype(np.float32) for a in got]
    w = [a.astype(np.float32) for a in want]
    n = g[0].shape[0] * g[0].shape[1]
    # geometry: normal + depth, motion + object id + previous depth, albedo + roughness
    for k, tol in ((1, 2e-3), (2, 2e-2), (3, 2e-3)):
        d = np.abs(g[k] - w[k]) / np.maximum(1.0, np.abs(w[k]))
        bad = (d > tol).any(axis=2).sum()
        assert bad <= max(2, 0.005 * n), (pt.GBUF_NAMES[k], bad, d.max())
    # primary emission (sky colour on sky pixels)
    d = np.abs(g[4] - w[4]) / np.maximum(1.0, np.abs(w[4]))
    assert (d > 2e-3).any(axis=2).sum() <= max(2, 0.005 * n)
    # radiance: per pixel where the path took the same branches, and on average
    r = np.abs(g[0][..., :3] - w[0][..., :3]) / np.maximum(0.05, np.abs(w[0][..., :3]))
    close = (r <= 1e-2).all(axis=2).mean()
    assert close >= rad_frac, close
    assert np.isfinite(g[0]).all()
    mg, mw = g[0][..., :3].mean(), w[0][..., :3].mean()
    assert abs(mg - mw) <= 0.05 * mw + 1e-3, (mg, mw)


@pytest.fixture(scope="module")
def demo():
    sc, env, mover = pt.demo_scene(0, seed=2)
    return sc, env, mover


def test_scene_buffers_match_the_oracle_assembly(demo):
    sc, _, _ = demo
    _check_buffers(sc, _oracle_scene(sc))


def test_mode0_gbuffer_matches_the_oracle(demo):
    sc, env, _ = demo
    p = pt.PathTracer(0, sc, W, H)
    cam = _camera()
    for frame in (0, 5):
        p.write_uniforms(camera=cam, frame=frame, mode=0, jitter=pt.JITTER[frame % 16], env=env)
        p.encode(frame & 1)
        torch.cuda.synchronize()
        want = _oracle_scene(sc).render(bytes(p._frame), W, H, 0)
        _compare_mode0(_gbuf_host(p, frame & 1), want)
    p.destroy()


def test_mode1_accumulation_matches_the_oracle(demo):
    sc, env, _ = demo
    p = pt.PathTracer(0, sc, W, H)
    p.clear_accum()
    p.write_uniforms(camera=_camera(), frame=3, mode=1, spp=2, sample_offset=4, env=env)
    p.encode(0)
    p.encode(0)  # accumulates twice
    torch.cuda.synchronize()
    got = p.accum.cpu().numpy()
    osc = _oracle_scene(sc)
    want = osc.render(bytes(p._frame), W, H, 1)
    want = osc.render(bytes(p._frame), W, H, 1, accum=want)
    assert (got[..., 3] == 4).all() and (want[..., 3] == 4).all()
    r = np.abs(got[..., :3] - want[..., :3]) / np.maximum(0.05, np.abs(want[..., :3]))
    assert (r <= 1e-2).all(axis=2).mean() >= 0.85
    assert abs(got[..., :3].mean() - want[..., :3].mean()) <= 0.05 * want[..., :3].mean()
    p.destroy()


def _env_image():
    Hh, Ww = 64, 128
    y = (np.arange(Hh) + 0.5) / Hh
    img = np.zeros((Hh, Ww, 4), np.float32)
    img[..., 0] = (0.3 + 0.7 * (1 - y))[:, None]
    img[..., 1] = (0.35 + 0.5 * (1 - y))[:, None]
    img[..., 2] = (0.5 + 0.5 * (1 - y))[:, None]
    img[..., 3] = 1
    img[10, 20, :3] = 8000.0
    return img


def test_environment_map_matches_the_oracle(demo):
    sc, env, _ = demo
    m = pt.prepare_env_map(_env_image(), sun=True)
    e = dict(env, map=m, mapRotation=0.7, mapIntensity=1.3, lights=[pt.env_sun_light(m, 0.7, scale=1.3)])
    p = pt.PathTracer(0, sc, W, H)
    p.write_uniforms(camera=_camera(), frame=1, mode=0, jitter=pt.JITTER[1], env=e)
    p.encode(1)
    torch.cuda.synchronize()
    osc = _oracle_scene(sc)
    osc.set_env(m.half, m.table)
    _compare_mode0(_gbuf_host(p, 1), osc.render(bytes(p._frame), W, H, 0))
    p.destroy()


def test_dynamic_group_motion_vectors_and_refit():
    sc, env, mover = pt.demo_scene(0, seed=5, n_objects=4)
    p = pt.PathTracer(0, sc, W, H)
    cam = _camera()
    vp0 = p.write_uniforms(camera=cam, frame=0, mode=0, jitter=(0.0, 0.0), env=env)
    p.encode(0)
    pos_prev, _ = mover(20)
    pos, nrm = mover(21)  # previous = the frame-20 pose (in front of the other objects), current = frame 21
    cam.look_at((1.3, 4.0, 12.8), (0.0, 0.8, 0.0))
    p.write_uniforms(camera=cam, prev_view_proj=vp0, frame=1, mode=0, jitter=(0.0, 0.0), env=env)
    p.encode(1)
    torch.cuda.synchronize()
    # the oracle scene at the frame-1 pose with the frame-0 pose as previous positions
    groups = sc.group_arrays()
    groups[-1]["pos"], groups[-1]["nrm"] = pos, nrm
    mats = sc.materials_array()
    n_layers = int(mats.view(np.int32)[:, 12:15].max()) + 1
    osc = opt.Scene(groups, mats, _download(sc.device_buffers()["tex"], n_layers * _layer_bytes()), n_layers)
    nv = len(pos)
    osc.verts[-nv:, 4:7] = pos_prev
    got, want = _gbuf_host(p, 1), osc.render(bytes(p._frame), W, H, 0)
    _compare_mode0(got, want)
    # the refitted BVH of the dynamic group bounds the moved box: boxes hold every triangle of their leaves
    info = sc.info()
    nodes = _download(sc.device_buffers()["nodes"], info["node_total"] * 64).view(np.float32).reshape(-1, 16)
    b = sc.blas_table()[-1]
    grp = nodes[b.node_offset:b.node_offset + b.node_count]
    lo = np.minimum(grp[:, 0:3], grp[:, 8:11]).min(axis=0)
    hi = np.maximum(grp[:, 4:7], grp[:, 12:15]).max(axis=0)
    assert (pos.min(axis=0) >= lo - 1e-6).all() and (pos.max(axis=0) <= hi + 1e-6).all()
    # pixels on the mover carry its object id and a non-zero motion
    mv = got[2].astype(np.float32)
    mover_id = len(mats) - 1
    on = mv[..., 2] == mover_id
    assert on.sum() > 20 and (np.hypot(mv[on, 0], mv[on, 1]) > 0.01).mean() > 0.9
    p.destroy()


def test_errors(demo):
    sc, env, _ = demo
    p = pt.PathTracer(0, sc, W, H)
    p.write_uniforms(camera=_camera(), env=env)
    p._frame.size[0] = W + 1
    with pytest.raises(HushError, match="differs from the tracer"):
        p.encode(0)
    p.write_uniforms(camera=_camera(), env=env)
    p._frame.blas[0].node_offset += 1
    with pytest.raises(HushError, match="is not one of the scene's"):
        p.encode(0)
    p.write_uniforms(camera=_camera(), env=env)
    p._frame.env[3] = 1.0
    with pytest.raises(HushError, match="no environment map"):
        p.encode(0)
    with pytest.raises(HushError, match="slot must be 0 or 1"):
        p.write_uniforms(camera=_camera(), env=env) is not None and p.encode(2)
    with pytest.raises(HushError, match="not dynamic"):
        sc.update(0, np.zeros((sc._groups[0].n_verts, 3), np.float32))
    p.destroy()


def test_gbuffer_feeds_hush_end_to_end():
    sc, env, mover = pt.demo_scene(0, seed=7, n_objects=8)
    w, h = 160, 96
    p = pt.PathTracer(0, sc, w, h)
    den = Hush(0, {"width": w, "height": h})
    cam = pt.Camera(position=(0.0, 3.5, 12.0), target=(0.0, 0.8, 0.0), fov=50, aspect=w / h)
    vp = None
    outs = []
    for t in range(6):
        mover(t)
        cam.look_at((0.2 * t, 3.5, 12.0), (0.0, 0.8, 0.0))
        vp = p.write_uniforms(camera=cam, prev_view_proj=vp, frame=t, mode=0, jitter=pt.JITTER[t % 16], env=env)
        g = p.encode(t & 1)
        outs.append(den.denoise(g).float().clone())
    torch.cuda.synchronize()
    o = torch.stack(outs)
    assert torch.isfinite(o).all()
    noisy = p.gbuf[1]["radiance"].float()
    assert o[-1][..., :3].mean() > 0
    den.destroy()
    p.destroy()
    del noisy
