"""hush_mlp_grad_noalloc: the MLP weight gradient for callers that cannot allocate device memory.

Render or training loops with a fixed device-memory budget (where an allocation mid-frame would synchronise the
device or fail) and hosts that only lend the library buffers they own cannot call cudaMalloc; this entry point keeps
its scratch in a fixed device array instead. It must give the same gradient as the trainer's own weight-gradient
path, call after call (the array keeps the previous call's partial sums, which must not leak into the next result).
This file is collected last so that a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from hush_b200 import Hush, scene
from hush_b200 import _lib as L
from hush_b200.train import Trainer, xavier_init

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(f):
    return {k: torch.from_numpy(np.ascontiguousarray(f[k])).cuda() for k in oracle.INPUTS}


def _noalloc(g, dpar, theta, out):
    ptrs = [g.buffer(n).data_ptr() for n in ("F0", "F1", "F2", "F3")]
    W2, H2 = (g.width + 1) // 2, (g.height + 1) // 2
    rc = L.lib().hush_mlp_grad_noalloc(*ptrs, dpar.data_ptr(), theta.data_ptr(), W2, H2, out.data_ptr(),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == L.HUSH_OK, L.lib().hush_global_error()
    torch.cuda.synchronize()
    return out.cpu().numpy().copy()


def test_noalloc_weight_gradient_matches_the_trainer():
    W, H = 96, 64
    cfg = scene.SceneConfig(W, H, 3, n_moving=2, pan_min=1.0, pan_max=3.0, seed=21)
    host = [scene.frame_host(cfg, i, clean=True) for i in range(3)]
    cleans = [torch.from_numpy(h["clean"]).cuda() for h in host]
    g = Hush(0, {"width": W, "height": H, "schedule": "passes"})
    tr = Trainer(g, xavier_init(21))
    for t in range(2):
        tr.frame(_dev(host[t]), cleans[t], cleans[t - 1] if t else None, 0.5, backward=False)
        tr.end_frame()
    tr.zero_grad()
    tr.frame(_dev(host[2]), cleans[2], cleans[1], 0.5, backward=True)
    torch.cuda.synchronize()
    ref = tr.grad()  # the trainer's weight gradient (per-CTA scratch owned by the trainer)
    _, dpar = tr.par()
    dpar_d = torch.from_numpy(dpar).cuda()
    theta_d = torch.from_numpy(tr.theta).cuda()
    out = torch.full((812,), float("nan"), dtype=torch.float64, device="cuda")
    scale = np.abs(ref).max()
    assert scale > 0
    for _ in range(2):  # two calls in a row on the shared scratch
        got = _noalloc(g, dpar_d, theta_d, out)
        assert np.isfinite(got).all()
        # same tolerance as the adjoint tests: 1e-3 of the largest component
        assert np.abs(got - ref).max() <= 1e-3 * scale, np.abs(got - ref).max() / scale


def test_noalloc_matches_the_mlp_adjoint_on_all_seeds_and_many_chunks():
    """At 640 x 360 (320 x 180 = 57,600 half-res rows: 900 chunks of 64 on 512 CTAs, so CTAs sum two chunks) with a
    random dL/dpar on all 12 channels, alpha and gamma included, against hush_mlp_bwd's weight gradient; then a
    smaller call on the same scratch (the first 60 half-res rows) against the adjoint of the seed cut to those rows,
    so partial sums left by the larger call cannot leak into it. The smaller call takes the first 60 rows (300
    chunks): the top rows of the scenes are sky, which carries no gradient."""
    W, H = 640, 360
    cfg = scene.SceneConfig(W, H, 3, n_moving=2, pan_min=1.0, pan_max=3.0, seed=5)
    host = [scene.frame_host(cfg, i, clean=True) for i in range(3)]
    cleans = [torch.from_numpy(h["clean"]).cuda() for h in host]
    g = Hush(0, {"width": W, "height": H, "schedule": "passes"})
    tr = Trainer(g, xavier_init(5))
    for t in range(2):
        tr.frame(_dev(host[t]), cleans[t], cleans[t - 1] if t else None, 0.5, backward=False)
        tr.end_frame()
    inputs = _dev(host[2])
    tr.begin(inputs, cleans[2], cleans[1], 0.5)
    tr.fwd("mlp")
    dpar = tr.buffer("DPAR")
    H2, W2 = dpar.shape[0], dpar.shape[1]
    assert H2 * W2 > 512 * 64
    seed = torch.randn(dpar.shape, generator=torch.Generator().manual_seed(9), dtype=torch.float64).float().cuda()
    theta = tr.buffer("THETA")

    def adjoint(sd):
        tr.zero_adjoints()
        tr.zero_grad()
        dpar.copy_(sd)
        tr.bwd("mlp")
        torch.cuda.synchronize()
        return tr.grad()

    ref = adjoint(seed)
    b3 = 16 * 20 + 16 + 16 * 16 + 16 + 12 * 16  # offset of b3 in the blob
    assert ref[b3] != 0.0 and ref[b3 + 1] != 0.0, "the alpha / gamma seeds must reach their biases"
    out = torch.full((812,), float("nan"), dtype=torch.float64, device="cuda")
    scale = np.abs(ref).max()
    for _ in range(2):
        got = _noalloc(g, seed, theta, out)
        assert np.isfinite(got).all()
        assert np.abs(got - ref).max() <= 1e-3 * scale, np.abs(got - ref).max() / scale
    # a smaller call after the larger one: the first 60 half-res rows
    n_small = 60
    cut = seed.clone()
    cut[n_small:] = 0.0
    ref_small = adjoint(cut)
    ptrs = [g.buffer(n).data_ptr() for n in ("F0", "F1", "F2", "F3")]
    rc = L.lib().hush_mlp_grad_noalloc(*ptrs, seed.data_ptr(), theta.data_ptr(), W2, n_small, out.data_ptr(),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == L.HUSH_OK, L.lib().hush_global_error()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    s_small = np.abs(ref_small).max()
    assert s_small > 0
    assert np.abs(got - ref_small).max() <= 1e-3 * s_small, np.abs(got - ref_small).max() / s_small
    tr.destroy()
    g.destroy()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    t = torch.zeros(16, dtype=torch.float32, device="cuda")
    d = torch.zeros(812, dtype=torch.float64, device="cuda")
    p = t.data_ptr()
    rc = L.lib().hush_mlp_grad_noalloc(p, p, p, p, p, p, 8192, 4096, d.data_ptr(), None)
    assert rc == L.HUSH_ERR_ARG
    assert b"exceed the maximum of 16777216" in L.lib().hush_global_error()
    rc = L.lib().hush_mlp_grad_noalloc(None, p, p, p, p, p, 8, 8, d.data_ptr(), None)
    assert rc == L.HUSH_ERR_ARG
