"""Path-tracer oracle helpers (TEST INFRASTRUCTURE ONLY): ctypes bindings of oracle/pt_oracle.cpp and a numpy
restatement of SceneGPU.build (src/pt/scene.js:64-176, 178-222) that turns world-space meshes into the reference's
scene buffers with the oracle's own BVH builder. Only the tests import this module."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as _olib

P = C.c_void_p
ENV_GW, ENV_GH = 256, 128
TEX_SIZE = 1024


class PtScene(C.Structure):
    _fields_ = [("nodes", P), ("tris", P), ("verts", P), ("mats", P), ("tri_idx", P), ("tex", P),
                ("tex_layers", C.c_int), ("env", P), ("env_w", C.c_int), ("env_h", C.c_int), ("env_table", P)]


_bound = False


def lib():
    global _bound
    L = _olib()
    if not _bound:
        sig = {
            "ho_pt_render": (C.c_int, [C.POINTER(PtScene), P, C.POINTER(P), P]),
            "ho_pt_pixel": (None, [C.POINTER(PtScene), P, C.c_int, C.c_int, P]),
            "ho_pt_trace": (None, [C.POINTER(PtScene), P, P, P, P]),
            "ho_bvh_build": (C.c_int, [P, C.c_int, P, P, C.POINTER(C.c_int)]),
            "ho_bvh_refit": (None, [P, C.c_int, P]),
            "ho_bvh_packed_count": (C.c_int, [P, C.c_int]),
            "ho_bvh_pack": (None, [P, C.c_int, P]),
            "ho_tri_lod": (C.c_uint16, [P, P, P, C.c_int]),
            "ho_env_prepare": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_double, P, P, P, P]),
            "ho_pt_jitter": (None, [P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _bound = True
    return L


def bvh_build(pos: np.ndarray):
    """buildBVH: (nodes (n, 8) float32, order, max depth)."""
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 9)
    n = len(p)
    nodes = np.zeros((max(1, 2 * n), 8), np.float32)
    order = np.zeros(max(1, n), np.uint32)
    d = C.c_int()
    used = lib().ho_bvh_build(p.ctypes.data, n, nodes.ctypes.data, order.ctypes.data, C.byref(d))
    return nodes[:used].copy(), order[:n].copy(), d.value


def bvh_refit(nodes: np.ndarray, tri_pos: np.ndarray):
    tp = np.ascontiguousarray(tri_pos, np.float32)
    lib().ho_bvh_refit(nodes.ctypes.data, len(nodes), tp.ctypes.data)


def bvh_pack(nodes: np.ndarray) -> np.ndarray:
    k = lib().ho_bvh_packed_count(nodes.ctypes.data, len(nodes))
    out = np.zeros((k, 16), np.float32)
    lib().ho_bvh_pack(nodes.ctypes.data, len(nodes), out.ctypes.data)
    return out


def env_prepare(rgba: np.ndarray, sun=True, cone_deg=3.0):
    img = np.ascontiguousarray(rgba, np.float32).copy()
    H, W = img.shape[:2]
    half = np.zeros((H, W, 4), np.uint16)
    table = np.zeros((ENV_GH, ENV_GW, 4), np.float32)
    d, e = (C.c_double * 3)(), (C.c_double * 3)()
    has = lib().ho_env_prepare(img.ctypes.data, W, H, 1 if sun else 0, cone_deg, half.ctypes.data, table.ctypes.data,
                               d, e)
    return {"rgba": img, "half": half, "table": table, "sun": (list(d), list(e)) if has else None}


def jitter():
    out = (C.c_float * 32)()
    lib().ho_pt_jitter(out)
    return np.array(list(out), np.float32).reshape(16, 2)


class Scene:
    """Scene buffers assembled like SceneGPU.build from groups of world-space meshes.

    groups: list of dicts {flags, pos (V, 3), nrm (V, 3) or None, uv (V, 2) or None, idx (T, 3), mat (T,)};
    mats: (M, 20) float32 records (int32 texture layers stored bitwise); tex: uint8 texture array or None."""

    def __init__(self, groups, mats: np.ndarray, tex: np.ndarray | None = None, tex_layers: int = 0):
        verts, gpos, gidx = [], [], []
        voff = 0
        for g in groups:
            p = np.asarray(g["pos"], np.float32).reshape(-1, 3)
            V = len(p)
            nrm = g.get("nrm")
            if nrm is None:
                n = np.tile(np.array([0, 1, 0], np.float32), (V, 1))
            else:
                n64 = np.asarray(nrm, np.float32).astype(np.float64)
                ln = np.sqrt((n64 ** 2).sum(axis=1, keepdims=True))
                n = np.where(ln > 0, n64 / np.where(ln > 0, ln, 1), 0).astype(np.float32)
            uv = np.zeros((V, 2), np.float32) if g.get("uv") is None else np.asarray(g["uv"], np.float32)
            v = np.zeros((V, 12), np.float32)
            v[:, 0:3], v[:, 3], v[:, 4:7], v[:, 8:11], v[:, 11] = p, uv[:, 0], p, n, uv[:, 1]
            verts.append(v)
            idx = np.asarray(g["idx"], np.uint32).reshape(-1, 3) + voff
            gidx.append(np.column_stack([idx, np.asarray(g["mat"], np.uint32)]))
            gpos.append(p[idx - voff].reshape(-1, 9))
            voff += V
        self.verts = np.ascontiguousarray(np.concatenate(verts))
        mats = np.ascontiguousarray(mats, np.float32).reshape(-1, 20)
        self.mats = mats
        tri_idx, tri_pos, nodes, blas = [], [], [], []
        toff = noff = 0
        self.max_depth = 0
        for g, ix, pos in zip(groups, gidx, gpos):
            nb, order, depth = bvh_build(pos)
            self.max_depth = max(self.max_depth, depth)
            packed = bvh_pack(nb)
            tri_idx.append(ix[order])
            tri_pos.append(pos[order])
            nodes.append(packed)
            blas.append((noff, toff, len(packed), g.get("flags", 0)))
            noff += len(packed)
            toff += len(ix)
        self.tri_idx = np.ascontiguousarray(np.concatenate(tri_idx), np.uint32)
        self.tri_pos = np.ascontiguousarray(np.concatenate(tri_pos), np.float32)
        self.nodes = np.ascontiguousarray(np.concatenate(nodes), np.float32)
        self.blas = blas
        for t in range(len(self.tri_idx)):  # computeTriLod
            a, b, c = (self.verts[self.tri_idx[t, k]] for k in range(3))
            lod = lib().ho_tri_lod(a.ctypes.data, b.ctypes.data, c.ctypes.data, TEX_SIZE)
            self.tri_idx[t, 3] = (int(self.tri_idx[t, 3]) & 0xffff) | (int(lod) << 16)
        tex_of = mats.view(np.int32)[:, 12]
        base_w = mats[:, 3]
        tris = np.zeros((len(self.tri_pos), 12), np.float32)  # packTris
        tp = self.tri_pos.reshape(-1, 3, 3)
        m = self.tri_idx[:, 3] & 0xffff
        tris[:, 0:3] = tp[:, 0]
        tris[:, 3] = ((base_w[m] > 0) & (tex_of[m] >= 0)).astype(np.float32)
        tris[:, 4:7] = tp[:, 1] - tp[:, 0]
        tris[:, 8:11] = tp[:, 2] - tp[:, 0]
        self.tris = tris
        self.tex = np.zeros(16, np.uint8) if tex is None else np.ascontiguousarray(tex, np.uint8)
        self.tex_layers = tex_layers
        self.env = None
        self.env_table = None
        self.env_w = self.env_h = 0

    def set_env(self, half: np.ndarray | None, table: np.ndarray | None):
        if half is None:
            self.env = self.env_table = None
            self.env_w = self.env_h = 0
        else:
            self.env = np.ascontiguousarray(half, np.uint16)
            self.env_table = np.ascontiguousarray(table, np.float32)
            self.env_h, self.env_w = self.env.shape[:2]

    def _struct(self):
        e = self.env.ctypes.data if self.env is not None else None
        t = self.env_table.ctypes.data if self.env_table is not None else None
        return PtScene(self.nodes.ctypes.data, self.tris.ctypes.data, self.verts.ctypes.data, self.mats.ctypes.data,
                       self.tri_idx.ctypes.data, self.tex.ctypes.data, self.tex_layers, e, self.env_w, self.env_h, t)

    def render(self, frame_bytes: bytes, width: int, height: int, mode: int = 0, accum: np.ndarray | None = None):
        """main() over the image: mode 0 returns the five G-buffer images as float16 (H, W, 4); mode 1 adds to and
        returns accum (H, W, 4) float32."""
        s = self._struct()
        fb = C.create_string_buffer(bytes(frame_bytes), len(frame_bytes))
        if mode == 0:
            imgs = [np.zeros((height, width, 4), np.uint16) for _ in range(5)]
            ptrs = (P * 5)(*[a.ctypes.data for a in imgs])
            lib().ho_pt_render(C.byref(s), fb, ptrs, None)
            return [a.view(np.float16) for a in imgs]
        acc = np.zeros((height, width, 4), np.float32) if accum is None else accum
        ptrs = (P * 5)()
        lib().ho_pt_render(C.byref(s), fb, ptrs, acc.ctypes.data)
        return acc

    def trace(self, frame_bytes: bytes, o, d):
        s = self._struct()
        fb = C.create_string_buffer(bytes(frame_bytes), len(frame_bytes))
        oo, dd = np.asarray(o, np.float32), np.asarray(d, np.float32)
        out = np.zeros(5, np.float32)
        lib().ho_pt_trace(C.byref(s), fb, oo.ctypes.data, dd.ctypes.data, out.ctypes.data)
        return out
