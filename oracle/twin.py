"""FP64 restatement of the training twin (torch autograd): TEST INFRASTRUCTURE ONLY.

The twin is the frame after TEMPORAL without f16 storage rounding: the MLP on FP32 master weights and its heads
(src/denoise/hush.js:683-704, 357-362), the mid levels mid1-mid3 (hush.js:366, 753-754 via atrousFn 431-476), the
fine level and recombination (hush.js:578-620) and TAA (hush.js:649-676), followed by the training loss (relative L1 per value, clipped at 1). Its inputs
are the frame's state as the CUDA trainer leaves it (features F0..F3, A0, key, coarse level, history, G-buffer). The
autograd gradient of this float64 graph is the reference the hand-written CUDA adjoint is checked against.
"""
from __future__ import annotations

import math

import numpy as np
import torch

LUM = (0.2126, 0.7152, 0.0722)
W1o, B1o = 0, 320
W2o, B2o = 336, 592
W3o, B3o = 608, 800


def _t(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64))


def lum(c):
    return c[..., 0] * LUM[0] + c[..., 1] * LUM[1] + c[..., 2] * LUM[2]


def oct_dec(ex, ey):
    vz = 1.0 - ex.abs() - ey.abs()
    t = torch.clamp(-vz, min=0.0)
    vx = ex + torch.where(ex >= 0, -t, t)
    vy = ey + torch.where(ey >= 0, -t, t)
    n = torch.stack([vx, vy, vz], -1)
    return n / torch.clamp(n.norm(dim=-1, keepdim=True), min=1e-20)


def pow128(x):
    for _ in range(7):
        x = x * x
    return x


def gather(img, yy, xx):
    return img[yy.clamp(0, img.shape[0] - 1), xx.clamp(0, img.shape[1] - 1)]


H3, H5 = (0.25, 0.5, 0.25), (1 / 16, 1 / 4, 3 / 8, 1 / 4, 1 / 16)  # the B-spline tap weights of atrousFn (R = 1, 2)


def filt(A, G, s, c, step, pref, R=1):
    """atrousFn (hush.js:431-476) with radius R at every pixel of a (H, W) level; A (H, W, 4) colour + variance, G
    (H, W, 4) normal + depth, s / c (H, W) or scalars. Clamp-to-edge tiles, taps outside the image or on sky
    skipped."""
    H, W = A.shape[:2]
    ys, xs = torch.meshgrid(torch.arange(H), torch.arange(W), indexing="ij")
    gp, cen = G, A
    if pref:
        def a(dx, dy):
            return gather(A, ys + dy, xs + dx)[..., 3]
        gv = 0.0625 * (a(-1, -1) + a(1, -1) + a(-1, 1) + a(1, 1)) + 0.125 * (a(0, -1) + a(-1, 0) + a(1, 0) + a(0, 1)) \
            + 0.25 * cen[..., 3]
    else:
        gv = cen[..., 3]
    lc = lum(cen)
    sl = s / (torch.sqrt(torch.clamp(gv, min=1e-12)) + 1e-6)
    zl, zr = gather(G, ys, xs - 1)[..., 3], gather(G, ys, xs + 1)[..., 3]
    zu, zd = gather(G, ys - 1, xs)[..., 3], gather(G, ys + 1, xs)[..., 3]
    big = torch.full_like(zl, 1e9)
    gx = torch.minimum(torch.where(zr > 0, (zr - gp[..., 3]).abs(), big), torch.where(zl > 0, (zl - gp[..., 3]).abs(), big))
    gy = torch.minimum(torch.where(zd > 0, (zd - gp[..., 3]).abs(), big), torch.where(zu > 0, (zu - gp[..., 3]).abs(), big))
    zg = torch.minimum(torch.maximum(gx, gy), gp[..., 3])
    # sky centres are discarded by the caller; a positive depth keeps their weights finite (an infinite weight in a
    # discarded torch.where branch still turns the zero gradient into NaN)
    zg = torch.where(gp[..., 3] >= 0, zg, torch.ones_like(zg))
    hw = H3 if R == 1 else H5
    cw = (hw[R] * hw[R]) * torch.as_tensor(c, dtype=torch.float64) * torch.ones_like(lc)
    Wt = cw
    S = cen[..., :3] * cw[..., None]
    V = cen[..., 3] * cw * cw
    for dy in range(-R, R + 1):
        for dx in range(-R, R + 1):
            if dx == 0 and dy == 0:
                continue
            hh = hw[dx + R] * hw[dy + R]
            tx, ty = xs + dx * step, ys + dy * step
            gq, cq = gather(G, ty, tx), gather(A, ty, tx)
            ok = (tx >= 0) & (ty >= 0) & (tx < W) & (ty < H) & (gq[..., 3] >= 0)
            iz = 1.0 / (zg * (math.sqrt(dx * dx + dy * dy) * step) + 1e-3)
            wq = hh * pow128(torch.clamp((gq[..., :3] * gp[..., :3]).sum(-1), min=0.0)) * torch.exp(
                -(gq[..., 3] - gp[..., 3]).abs() * iz - sl * (lum(cq) - lc).abs())
            wq = torch.where(ok, wq, torch.zeros_like(wq))
            Wt = Wt + wq
            S = S + wq[..., None] * cq[..., :3]
            V = V + wq * wq * cq[..., 3]
    return torch.cat([S / Wt[..., None], (V / (Wt * Wt))[..., None]], -1)


COARSE_S = 0.25  # hush.js:26


def coarse_guide(CG):
    """The coarse guide as the coarse passes read it: (qh, qw, 4) rgba16float (oct normal, depth) -> decoded normal +
    depth."""
    g = _t(np.asarray(CG, np.float16).astype(np.float64))
    return torch.cat([oct_dec(g[..., 0], g[..., 1]), g[..., 2:3]], -1)


def down(Ah, cnt):
    """down() of hush.js:385-402 over the whole quarter-res grid without the f16 rounding: the block means Ah
    (h, w, 4) weighted by the blocks' pixel counts cnt (h, w) over each 2x2 group -> (col / N, var / N / N), zeros
    where no block has a surface."""
    h, w = Ah.shape[:2]
    qh, qw = (h + 1) // 2, (w + 1) // 2
    pad_h, pad_w = 2 * qh - h, 2 * qw - w
    A = torch.nn.functional.pad(Ah.permute(2, 0, 1), (0, pad_w, 0, pad_h)).permute(1, 2, 0)
    n = torch.nn.functional.pad(torch.clamp(cnt, min=0.0), (0, pad_w, 0, pad_h))
    A = A.reshape(qh, 2, qw, 2, 4)
    n = n.reshape(qh, 2, qw, 2)
    N = n.sum((1, 3))
    col = (n[..., None] * A[..., :3]).sum((1, 3))
    vr = (n * A[..., 3]).sum((1, 3))
    Ns = torch.where(N > 0, N, torch.ones_like(N))
    out = torch.cat([col / Ns[..., None], (vr / Ns / Ns)[..., None]], -1)
    return torch.where((N > 0)[..., None], out, torch.zeros_like(out))


def coarse1(Ah, cnt, Gq):
    """COARSE1 (hush.js:372-421): the 5x5 a-trous (step 1, variance prefilter, s = COARSE_S, c = 1) of down(Ah);
    zeros where the coarse guide has no surface."""
    sky = Gq[..., 3] < 0
    y = filt(down(Ah, cnt), Gq, COARSE_S, 1.0, 1, True, R=2)
    return torch.where(sky[..., None], torch.zeros_like(y), y)


def coarse2(C1, Gq):
    """coarse2 (hush.js:752): the 5x5 a-trous (step 2, variance prefilter, s = COARSE_S, c = 1) of C1."""
    sky = Gq[..., 3] < 0
    y = filt(C1, Gq, COARSE_S, 1.0, 2, True, R=2)
    return torch.where(sky[..., None], torch.zeros_like(y), y)


def jbw(frx, fry, j, nq, zq, n, z):
    wb = (frx if (j & 1) else 1.0 - frx) * (fry if (j >> 1) else 1.0 - fry)
    dn = torch.clamp((nq * n).sum(-1), min=0.0)
    dn4 = (dn * dn) * (dn * dn)
    return wb * torch.exp(-(zq - z).abs() / (0.05 * z + 1e-3)) * dn4 * dn4


def tm(c):
    return c / (1.0 + lum(c))[..., None]


def to_ycocg(c):
    r, g, b = c[..., 0], c[..., 1], c[..., 2]
    return torch.stack([r * 0.25 + g * 0.5 + b * 0.25, r * 0.5 - b * 0.5, -r * 0.25 + g * 0.5 - b * 0.25], -1)


def from_ycocg(c):
    x, y, z = c[..., 0], c[..., 1], c[..., 2]
    return torch.stack([x + y - z, x + z, x - y - z], -1)


def unpack_half(a):
    """(h, w, 8) float16 array -> float64 tensor."""
    return _t(np.asarray(a, np.float16).astype(np.float64))


def half_inputs(st: dict):
    """Half-resolution inputs of the twin from the packed features: (features (h, w, 20), guide (h, w, 4) = oct-decoded
    normal + depth, sky mask (h, w), block means (h, w, 4))."""
    F0, F1, F2, F3 = (unpack_half(st[k]) for k in ("F0", "F1", "F2", "F3"))
    feats = torch.cat([F0, F1, F2[..., :4]], -1)[..., :20]
    guide_n = oct_dec(F3[..., 0], F3[..., 1])
    Gh = torch.cat([guide_n, F3[..., 2:3]], -1)
    sky_h = F3[..., 2] < 0
    Ah = F2[..., 4:8]
    return feats, Gh, sky_h, Ah


def mlp(feats, theta, sky_h):
    """The MLP and its heads (hush.js:683-704, 357-362): (par_raw, par) with par zero on sky rows, (h, w, 12)."""
    w = theta
    M1, b1 = w[W1o:B1o].view(16, 20), w[B1o:W2o]
    M2, b2 = w[W2o:B2o].view(16, 16), w[B2o:W3o]
    M3, b3 = w[W3o:B3o].view(12, 16), w[B3o:B3o + 12]
    h1 = torch.relu(feats @ M1.T + b1)
    h2 = torch.relu(h1 @ M2.T + b2)
    o = h2 @ M3.T + b3
    sig = torch.sigmoid
    par = torch.stack([1 / 32 + (31 / 32) * sig(o[..., 0]), 0.5 + 7.5 * sig(o[..., 1]), sig(o[..., 2]), sig(o[..., 3])]
                      + [0.25 * torch.exp(torch.clamp(o[..., 4 + k], -5, 5)) for k in range(4)]
                      + [torch.exp(torch.clamp(o[..., 8 + k], -4, 4)) for k in range(4)], -1)
    return par, torch.where(sky_h[..., None], torch.zeros_like(par), par)


def _par_f(par, sky_h):
    # rows of sky blocks carry zeros; the levels see c = 1 there so that the masked-out branches stay finite (a 0/0
    # in an unselected torch.where branch would turn its zero gradient into NaN)
    return torch.where(sky_h[..., None], torch.ones_like(par), par)


def mid(k: int, src, Gh, sky_h, par):
    """Mid level k = 1, 2, 3 (hush.js:366, 753-754): B_k = filt(src; s_k, c_k) with step 1, 2, 4; level 1 reads the
    block means with the variance prefilter. Zero on sky rows."""
    pf = _par_f(par, sky_h)
    step = (1, 2, 4)[k - 1]
    z4 = torch.zeros(*src.shape[:2], 4, dtype=torch.float64)
    return torch.where(sky_h[..., None], z4, filt(src, Gh, pf[..., 4 + k], pf[..., 8 + k], step, k == 1))


def fine(st: dict, par, B3, Gh, sky_h, Ah, A0=None, C0=None):
    """Fine level and recombination (hush.js:578-620): (A1, X), (H, W, 4) and (H, W, 3). A0: TEMPORAL's colour +
    variance as a tensor (to differentiate through it), else st["A0"]; C0 likewise for the coarse level."""
    par_f = _par_f(par, sky_h)
    A0 = _t(st["A0"]) if A0 is None else A0
    key = _t(st["key"])
    H, W = A0.shape[:2]
    G = torch.cat([oct_dec(key[..., 0], key[..., 1]), key[..., 2:3]], -1)
    ys, xs = torch.meshgrid(torch.arange(H), torch.arange(W), indexing="ij")
    hp_y, hp_x = ys >> 1, xs >> 1
    p_full = par[hp_y, hp_x]
    pf_full = par_f[hp_y, hp_x]
    A1 = filt(A0, G, pf_full[..., 4], pf_full[..., 8], 1, True)
    sky = G[..., 3] < 0
    f = A1[..., :3]
    n, z = G[..., :3], torch.where(G[..., 3] >= 0, G[..., 3], torch.ones_like(G[..., 3]))  # sky: see filt()
    hposx, hposy = (xs.double() + 0.5) / 2.0 - 0.5, (ys.double() + 0.5) / 2.0 - 0.5
    hbx, hby = torch.floor(hposx), torch.floor(hposy)
    uB = torch.zeros(H, W, 3, dtype=torch.float64)
    uA = torch.zeros(H, W, 3, dtype=torch.float64)
    swh = torch.zeros(H, W, dtype=torch.float64)
    hsx, hsy = (W + 1) // 2, (H + 1) // 2
    for j in range(4):
        qx, qy = hbx.long() + (j & 1), hby.long() + (j >> 1)
        ok = (qx >= 0) & (qy >= 0) & (qx < hsx) & (qy < hsy)
        g = gather(Gh, qy, qx)
        ok = ok & (g[..., 3] >= 0)
        wj = jbw(hposx - hbx, hposy - hby, j, g[..., :3], g[..., 3], n, z)
        wj = torch.where(ok, wj, torch.zeros_like(wj))
        swh = swh + wj
        uB = uB + wj[..., None] * gather(B3, qy, qx)[..., :3]
        uA = uA + wj[..., None] * gather(Ah, qy, qx)[..., :3]
    mid_ok = swh > 1e-4
    kappa, beta = p_full[..., 3], p_full[..., 2]
    swh_s = torch.where(mid_ok, swh, torch.ones_like(swh))
    ill = torch.where(mid_ok[..., None], uB / swh_s[..., None] + kappa[..., None] * (f - uA / swh_s[..., None]), f)
    C0, CG = (_t(st["C0"]) if C0 is None else C0), _t(st["CG"])
    CGd = torch.cat([oct_dec(CG[..., 0], CG[..., 1]), CG[..., 2:3]], -1)
    cposx, cposy = (xs.double() + 0.5) / 4.0 - 0.5, (ys.double() + 0.5) / 4.0 - 0.5
    cbx, cby = torch.floor(cposx), torch.floor(cposy)
    uC = torch.zeros(H, W, 3, dtype=torch.float64)
    swq = torch.zeros(H, W, dtype=torch.float64)
    qsx, qsy = (W + 3) // 4, (H + 3) // 4
    for j in range(4):
        qx, qy = cbx.long() + (j & 1), cby.long() + (j >> 1)
        ok = (qx >= 0) & (qy >= 0) & (qx < qsx) & (qy < qsy)
        g = gather(CGd, qy, qx)
        ok = ok & (g[..., 3] >= 0)
        wj = jbw(cposx - cbx, cposy - cby, j, g[..., :3], g[..., 3], n, z)
        wj = torch.where(ok, wj, torch.zeros_like(wj))
        swq = swq + wj
        uC = uC + wj[..., None] * gather(C0, qy, qx)[..., :3]
    coarse = swq > 1e-4
    up = torch.where(coarse[..., None], uC / torch.where(coarse, swq, torch.ones_like(swq))[..., None], ill)
    ill2 = ill + (up - ill) * beta[..., None]
    alb, emi = _t(st["material"])[..., :3], _t(st["emission"])[..., :3]
    X = torch.where(sky[..., None], emi, ill2 * alb + emi)
    return A1, X


def taa(st: dict, X):
    """TAA (hush.js:649-676) on the recombined colour X (H, W, 3): the output (H, W, 3)."""
    H, W = X.shape[:2]
    ys, xs = torch.meshgrid(torch.arange(H), torch.arange(W), indexing="ij")
    cur = tm(X)
    if st.get("reset", False):
        res = cur
    else:
        Y = to_ycocg(tm(X))
        win = [gather(Y, ys + dy, xs + dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
        m1 = sum(win) / 9.0
        v3 = sum((q - m1) ** 2 for q in win) / 9.0
        sd = torch.sqrt(torch.clamp(v3, min=1e-12))
        mv = _t(st["motion"])
        uvx, uvy = (xs.double() + 0.5 + mv[..., 0]) / W, (ys.double() + 0.5 + mv[..., 1]) / H
        inside = (uvx >= 0) & (uvy >= 0) & (uvx <= 1) & (uvy <= 1)
        ppx, ppy = uvx * W - 0.5, uvy * H - 0.5
        bx, by = torch.floor(ppx), torch.floor(ppy)
        fx, fy = ppx - bx, ppy - by
        prev = _t(st["taa_prev"])[..., :3]
        hist = 0
        for j in range(4):
            ox, oy = j & 1, j >> 1
            wb = (fx if ox else 1 - fx) * (fy if oy else 1 - fy)
            hist = hist + wb[..., None] * gather(prev, by.long() + oy, bx.long() + ox)
        hh = to_ycocg(tm(hist))
        hh = torch.minimum(torch.maximum(hh, m1 - 1.25 * sd), m1 + 1.25 * sd)
        hr = from_ycocg(hh)
        res = torch.where(inside[..., None], hr + (cur - hr) * 0.1, cur)
    return res / torch.clamp(1.0 - lum(res), min=1e-4)[..., None]


def loss_of(st: dict, out, lambda_t=0.0):
    """The training loss of a TAA output (H, W, 3): clipped relative L1 against st["clean"] plus lambda_t times the
    same on the difference to the previous frame (st["out_prev"], st["clean_prev"])."""
    H, W = out.shape[:2]
    clean = _t(st["clean"])
    den = clean.abs() + 1e-2
    N = 3.0 * H * W
    loss = torch.clamp((out - clean).abs() / den, max=1.0).sum() / N
    if st.get("out_prev") is not None and lambda_t > 0 and not st.get("reset", False):
        op = _t(st["out_prev"])[..., :3]
        cp = _t(st["clean_prev"])
        loss = loss + lambda_t * torch.clamp(((out - op) - (clean - cp)).abs() / den, max=1.0).sum() / N
    return loss


def _nb(img, dy, dx, fill=0.0):
    """img shifted so that out[y, x] = img[y + dy, x + dx], `fill` outside the image."""
    H, W = img.shape[:2]
    out = torch.full_like(img, fill)
    ys0, ys1 = max(0, -dy), min(H, H - dy)
    xs0, xs1 = max(0, -dx), min(W, W - dx)
    if ys0 < ys1 and xs0 < xs1:
        out[ys0:ys1, xs0:xs1] = img[ys0 + dy:ys1 + dy, xs0 + dx:xs1 + dx]
    return out


def _check_key(k, nd, z_prev, obj):
    """The history key test (hush.js:103-105) on gathered keys k (..., 4) against the pixel's normal / depth."""
    n = oct_dec(k[..., 0], k[..., 1])
    return ((k[..., 2] >= 0) & (k[..., 3] == obj) & ((k[..., 2] - z_prev).abs() <= 0.05 * z_prev + 0.01)
            & ((n * nd[..., :3]).sum(-1) >= 0.9))


def temporal(st: dict, hist_prev, mom_prev, par0_prev):
    """TEMPORAL's pixel() (hush.js:111-223) in float64 for the gradient through the history: (A0 (H, W, 4) colour +
    variance, mom (H, W, 4) = m1, m2, fast mean, history length), differentiable in hist_prev (H, W, 4; rgb used),
    mom_prev (H, W, 4) and par0_prev (h, w, 4; alpha = .x, gamma = .y). The G-buffer (st: radiance, normalDepth,
    motion, material) and the previous keys (st["key_prev"]) fix the statistics, the reprojection taps and their
    weights. For frames with history (st["reset"] false)."""
    rad, nd, mv, mat = (_t(np.asarray(st[k], np.float32)) for k in ("radiance", "normalDepth", "motion", "material"))
    keyp = _t(np.asarray(st["key_prev"], np.float32))
    H, W = rad.shape[:2]
    ys, xs = torch.meshgrid(torch.arange(H), torch.arange(W), indexing="ij")
    valid = nd[..., 3] >= 0
    illum = torch.where(valid[..., None], rad[..., :3] / torch.clamp(mat[..., :3], min=1e-3), torch.zeros(H, W, 3,
                        dtype=torch.float64))
    vf = valid.double()
    win = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    cnt = torch.clamp(sum(_nb(vf, dy, dx) for dy, dx in win), min=1.0)
    mu = sum(_nb(illum, dy, dx) * _nb(vf, dy, dx)[..., None] for dy, dx in win) / cnt[..., None]
    slm = lum(mu)
    sv = sum(_nb(vf, dy, dx)[..., None] * (_nb(illum, dy, dx) - mu) ** 2 for dy, dx in win)
    svar = sum(_nb(vf, dy, dx) * (lum(_nb(illum, dy, dx)) - slm) ** 2 for dy, dx in win) / cnt
    sd = torch.sqrt(torch.clamp(sv / cnt[..., None], min=1e-12))
    l = lum(illum)
    ppx, ppy = xs.double() + mv[..., 0], ys.double() + mv[..., 1]
    bxf, byf = torch.floor(ppx), torch.floor(ppy)
    fx, fy = ppx - bxf, ppy - byf
    bix, biy = bxf.long(), byf.long()
    wts = [(1 - fx) * (1 - fy), fx * (1 - fy), (1 - fx) * fy, fx * fy]
    sumW = torch.zeros(H, W, dtype=torch.float64)
    hc = torch.zeros(H, W, 3, dtype=torch.float64)
    hm = torch.zeros(H, W, 4, dtype=torch.float64)
    for i in range(4):
        qx, qy = bix + (i & 1), biy + (i >> 1)
        ok = (wts[i] > 0) & (qx >= 0) & (qy >= 0) & (qx < W) & (qy < H)
        ok = ok & _check_key(gather(keyp, qy, qx), nd, mv[..., 3], mv[..., 2])
        w = torch.where(ok, wts[i], torch.zeros_like(wts[i]))
        sumW = sumW + w
        hc = hc + w[..., None] * gather(hist_prev, qy, qx)[..., :3]
        hm = hm + w[..., None] * gather(mom_prev, qy, qx)
    bil = sumW >= 0.01
    cx, cy = torch.floor(ppx + 0.5).long(), torch.floor(ppy + 0.5).long()
    n3 = torch.zeros(H, W, dtype=torch.float64)
    hc3 = torch.zeros(H, W, 3, dtype=torch.float64)
    hm3 = torch.zeros(H, W, 4, dtype=torch.float64)
    for j in range(9):
        qx, qy = cx + j % 3 - 1, cy + j // 3 - 1
        ok = (qx >= 0) & (qy >= 0) & (qx < W) & (qy < H) & _check_key(gather(keyp, qy, qx), nd, mv[..., 3], mv[..., 2])
        okd = ok.double()
        n3 = n3 + okd
        hc3 = hc3 + okd[..., None] * gather(hist_prev, qy, qx)[..., :3]
        hm3 = hm3 + okd[..., None] * gather(mom_prev, qy, qx)
    one = torch.ones_like(sumW)
    hc = torch.where(bil[..., None], hc / torch.where(bil, sumW, one)[..., None],
                     hc3 / torch.where(n3 > 0, n3, one)[..., None])
    hm = torch.where(bil[..., None], hm / torch.where(bil, sumW, one)[..., None],
                     hm3 / torch.where(n3 > 0, n3, one)[..., None])
    has = (bil | (n3 > 0)) & (hm[..., 3] > 0) & valid
    hq = gather(par0_prev, torch.clamp(cy, 0, H - 1) >> 1, torch.clamp(cx, 0, W - 1) >> 1)
    alpha, gamma = hq[..., 0], hq[..., 1]
    hcl = torch.minimum(torch.maximum(hc, mu - gamma[..., None] * sd), mu + gamma[..., None] * sd)
    len1 = torch.clamp(torch.where(has, hm[..., 3], one) + 1.0, max=32.0)
    a = torch.maximum(alpha, 1.0 / len1)
    col = hcl + (illum - hcl) * a[..., None]
    nmx = hm[..., 0] + (l - hm[..., 0]) * a
    nmy = hm[..., 1] + (l * l - hm[..., 1]) * a
    nfast = hm[..., 2] + (l - hm[..., 2]) * torch.clamp(1.0 / len1, min=1.0 / 6.0)
    col = torch.where(has[..., None], col, illum)
    nmx, nmy = torch.where(has, nmx, l), torch.where(has, nmy, l * l)
    nfast, len1 = torch.where(has, nfast, l), torch.where(has, len1, one)
    tvar = torch.clamp(nmy - nmx * nmx, min=0.0)
    Aw = svar + (tvar - svar) * torch.clamp(len1 / 4.0, max=1.0)
    A0 = torch.cat([col, Aw[..., None]], -1)
    mom = torch.stack([nmx, nmy, nfast, len1], -1)
    z = torch.zeros_like(A0)
    return torch.where(valid[..., None], A0, z), torch.where(valid[..., None], mom, z)


def _st_value(x64, stored):
    """x64 in the backward, the stored f16 value in the forward (the straight-through gradient of the storage)."""
    return x64 + (_t(np.asarray(stored, np.float32)) - x64).detach()


def block_means(A0, surf):
    """block()'s mean of A0 (H, W, 4) over each 2x2 block's surface pixels surf (H, W) (hush.js:241-244): (h, w, 4),
    zeros for blocks without a surface."""
    H, W = A0.shape[:2]
    h, w = (H + 1) // 2, (W + 1) // 2
    A = torch.nn.functional.pad(A0.permute(2, 0, 1), (0, 2 * w - W, 0, 2 * h - H)).permute(1, 2, 0)
    m = torch.nn.functional.pad(surf.double(), (0, 2 * w - W, 0, 2 * h - H))
    A = A.reshape(h, 2, w, 2, 4)
    m = m.reshape(h, 2, w, 2)
    nv = m.sum((1, 3))
    s = (m[..., None] * A).sum((1, 3))
    return torch.where((nv > 0)[..., None], s / torch.clamp(nv, min=1.0)[..., None], torch.zeros_like(s))


def window_loss(states, theta, lambda_t=0.0):
    """The summed loss of a window with the gradient through time of hush_trainer_window_bptt: states[i] is frame i's
    st (twin_loss's keys, plus the frame's stored mom / hist / par0 and the G-buffer, and key_prev), frame 0 a reset.
    TEMPORAL runs in float64 on the previous frame's history, each stored value (A0, moments, colour history, par0)
    entering with the straight-through gradient; from the second frame on A0 also reaches the loss through the block
    means (block(), then mid1, the recombination and the coarse levels COARSE1 / coarse2, the stored block means,
    C1 and C0 entering straight through; states[i] then also holds C1). The features and the TAA history are
    constants."""
    total = 0.0
    hist_prev = mom_prev = par0_prev = None
    for i, st in enumerate(states):
        if i == 0:
            A0 = _t(np.asarray(st["A0"], np.float32))
            mom = _t(np.asarray(st["mom"], np.float32))
        else:
            A0_64, mom_64 = temporal(st, hist_prev, mom_prev, par0_prev)
            A0, mom = _st_value(A0_64, st["A0"]), _st_value(mom_64, st["mom"])
        feats, Gh, sky_h, Ah = half_inputs(st)
        C0 = None
        if i > 0:
            surf = _t(np.asarray(st["key"], np.float32))[..., 2] >= 0
            Ah = _st_value(block_means(A0, surf), Ah.numpy())
            Gq = coarse_guide(st["CG"])
            C1 = _st_value(coarse1(Ah, unpack_half(st["F3"])[..., 3], Gq), st["C1"])
            C0 = _st_value(coarse2(C1, Gq), st["C0"])
        _, par = mlp(feats, theta, sky_h)
        B1 = mid(1, Ah, Gh, sky_h, par)
        B2 = mid(2, B1, Gh, sky_h, par)
        B3 = mid(3, B2, Gh, sky_h, par)
        A1, X = fine(st, par, B3, Gh, sky_h, Ah, A0=A0, C0=C0)
        total = total + loss_of(st, taa(st, X), lambda_t)
        sky = _t(np.asarray(st["key"], np.float32))[..., 2] < 0
        A1 = torch.where(sky[..., None], torch.zeros_like(A1), A1)  # sky pixels store no history
        hist_prev, mom_prev = _st_value(A1, st["hist"]), mom
        par0_prev = _st_value(par[..., :4], st["par0"])
    return total


def twin_loss(st: dict, theta, lambda_t=0.0, return_all=False):
    """Loss of one frame. st: numpy arrays F0..F3 (h, w, 8) f16, A0 / key / material / emission / motion / taa_prev
    (H, W, 4), C0 / CG (qh, qw, 4), clean / clean_prev (H, W, 3) f32, out_prev (H, W, 4) f32 or None, reset (bool).
    theta: float64 tensor (812,) (may require grad)."""
    feats, Gh, sky_h, Ah = half_inputs(st)
    par_raw, par = mlp(feats, theta, sky_h)
    B1 = mid(1, Ah, Gh, sky_h, par)
    B2 = mid(2, B1, Gh, sky_h, par)
    B3 = mid(3, B2, Gh, sky_h, par)
    A1, X = fine(st, par, B3, Gh, sky_h, Ah)
    out = taa(st, X)
    loss = loss_of(st, out, lambda_t)
    if return_all:
        return loss, {"par": par, "par_raw": par_raw, "out": out, "X": X, "A1": A1, "B3": B3}
    return loss
