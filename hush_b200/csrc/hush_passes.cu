// One kernel per reference dispatch (src/denoise/hush.js:858-870), with the reference's 16 x 8 tiles. This is the
// pass-by-pass form used by the pass-level parity tests and by the per-pass C ABI; the frame's hot path is the fused
// form in hush_fused.cu.
#include "hush_device.cuh"
#include "hush_internal.h"

namespace hush {

constexpr int TW = 16, TH = 8;

// ------------------------------------------------------------------------------------------------ TEMPORAL
// hush.js:284-307: illumination tile (apron 1, zero outside the image or on sky), pixel() per thread, block() for
// the 32 2x2 blocks of the tile.
__global__ void __launch_bounds__(TW *TH) k_temporal(const __grid_constant__ HushFrame f) {
  constexpr int SW = TW + 2, SH = TH + 2;
  __shared__ float4 sI[SW * SH];
  __shared__ PixP sP[TW * TH];
  const int li = threadIdx.y * TW + threadIdx.x;
  const int ox = blockIdx.x * TW - 1, oy = blockIdx.y * TH - 1;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const int qx = ox + i % SW, qy = oy + i / SW;
    float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
    if (qx >= 0 && qy >= 0 && qx < f.W && qy < f.H && ldh(f.nd, qy * f.p_nd + qx).w >= 0.0f) {
      const float4 r = ldh(f.rad, qy * f.p_rad + qx), m = ldh(f.mat, qy * f.p_mat + qx);
      e = make_float4(r.x / fmaxf(m.x, 1e-3f), r.y / fmaxf(m.y, 1e-3f), r.z / fmaxf(m.z, 1e-3f), 1.0f);
    }
    sI[i] = e;
  }
  __syncthreads();
  const int px = blockIdx.x * TW + threadIdx.x, py = blockIdx.y * TH + threadIdx.y;
  PixP P = pixp_default();
  if (px < f.W && py < f.H) P = temporal_pixel<SW>(f, px, py, sI, threadIdx.x + 1, threadIdx.y + 1);
  sP[li] = P;
  __syncthreads();
  if (li < (TW / 2) * (TH / 2)) {
    const int lbx = li % (TW / 2), lby = li / (TW / 2);
    const int X = blockIdx.x * (TW / 2) + lbx, Y = blockIdx.y * (TH / 2) + lby;
    if (X < f.W2 && Y < f.H2) {
      PixP Pj[4];
#pragma unroll
      for (int j = 0; j < 4; j++) Pj[j] = sP[(lby * 2 + (j >> 1)) * TW + lbx * 2 + (j & 1)];
      float fe[20];
      float4 AC, G;
      const int o = Y * f.W2 + X;
      // 4x4 neighbourhood starts at block*2 - 1 in tile coordinates, i.e. tile index (2 lby) * SW + 2 lbx
      if (!block_features<SW>(Pj, sI, (2 * lby) * SW + 2 * lbx, f.exposure, fe, AC, G)) {
        f.F0[o] = make_uint4(0, 0, 0, 0);
        f.F1[o] = make_uint4(0, 0, 0, 0);
        f.F2[o] = make_uint4(0, 0, 0, 0);
        f.F3[o] = make_uint4(pk(0.f, 0.f), pk(-1.0f, 0.f), 0, 0);
      } else {
        f.F0[o] = make_uint4(pk(fe[0], fe[1]), pk(fe[2], fe[3]), pk(fe[4], fe[5]), pk(fe[6], fe[7]));
        f.F1[o] = make_uint4(pk(fe[8], fe[9]), pk(fe[10], fe[11]), pk(fe[12], fe[13]), pk(fe[14], fe[15]));
        f.F2[o] = make_uint4(pk(fe[16], fe[17]), pk(fe[18], fe[19]), pk(AC.x, AC.y), pk(AC.z, AC.w));
        f.F3[o] = make_uint4(pk(G.x, G.y), pk(G.z, G.w), 0, 0);
      }
    }
  }
}

// Tile loaders for the half-res passes: block mean (F2.zw) and decoded guide (F3.xy) at a clamped position.
HD_INL float4 f2_ac(const uint4 *F2, int i) {
  const uint4 t = __ldg(F2 + i);
  const float2 a = unpack2(t.z), b = unpack2(t.w);
  return make_float4(a.x, a.y, b.x, b.y);
}
HD_INL float4 f3_guide(const uint4 *F3, int i) {
  const uint4 t = __ldg(F3 + i);
  const float2 o = unpack2(t.x), z = unpack2(t.y);
  float4 g = oct_dec(o.x, o.y);
  g.w = z.x;
  return g;
}

// ------------------------------------------------------------------------------------------------ INFER + mid1
// hush.js:329-367. HD > 0: weights of width HD by value; HD == 0: any width from global memory.
template <int HD>
__global__ void __launch_bounds__(TW *TH) k_infer(const __grid_constant__ HushFrame f, const __grid_constant__ MlpW16 w) {
  constexpr int AP = 1, SW = TW + 2, SH = TH + 2;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const int li = threadIdx.y * TW + threadIdx.x;
  const int bx = blockIdx.x * TW, by = blockIdx.y * TH;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const int q = clampi(by - AP + i / SW, 0, f.H2 - 1) * f.W2 + clampi(bx - AP + i % SW, 0, f.W2 - 1);
    sA[i] = f2_ac(f.F2, q);
    sG[i] = f3_guide(f.F3, q);
  }
  __syncthreads();
  const int X = bx + threadIdx.x, Y = by + threadIdx.y;
  if (X >= f.W2 || Y >= f.H2) return;
  const int o = Y * f.W2 + X;
  const int lx = threadIdx.x + AP, ly = threadIdx.y + AP;
  if (sG[ly * SW + lx].w < 0.0f) {
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    sth(f.par0, o, z); sth(f.par1, o, z); sth(f.par2, o, z); sth(f.Bh0, o, z);
    return;
  }
  float fe[N_FEAT], out[N_OUT];
  {
    const uint4 a = __ldg(f.F0 + o), b = __ldg(f.F1 + o), c = __ldg(f.F2 + o);
    const uint32_t u[10] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y};
#pragma unroll
    for (int i = 0; i < 10; i++) {
      const float2 t = unpack2(u[i]);
      fe[2 * i] = t.x;
      fe[2 * i + 1] = t.y;
    }
  }
  if (f.mlp_half) mlp_fwd_half(HD > 0 ? w.w : f.w_glob, f.hidden, fe, out);
  else if constexpr (HD > 0) mlp_fwd<HD>(w.w, fe, out);
  else mlp_fwd_dyn(f.w_glob, f.hidden, fe, out);
  float4 p0, p1, p2;
  mlp_heads(out, p0, p1, p2);
  sth(f.par0, o, p0);
  sth(f.par1, o, p1);
  sth(f.par2, o, p2);
  sth(f.Bh0, o, filt<1, 1, true, SW>(sA, sG, lx, ly, X, Y, f.W2, f.H2, qf16(p1.y), qf16(p2.y)));
}

// ------------------------------------------------------------------------------------------------ mid2 / mid3
// atrousShader kinds mid2 / mid3 (hush.js:482-525, 753-754). COMP selects the learned s / c component.
template <int STEP, int COMP>
__global__ void __launch_bounds__(TW *TH) k_mid(const __grid_constant__ HushFrame f, const uint2 *src, uint2 *dst) {
  constexpr int AP = STEP, SW = TW + 2 * AP, SH = TH + 2 * AP;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const int li = threadIdx.y * TW + threadIdx.x;
  const int bx = blockIdx.x * TW, by = blockIdx.y * TH;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const int q = clampi(by - AP + i / SW, 0, f.H2 - 1) * f.W2 + clampi(bx - AP + i % SW, 0, f.W2 - 1);
    sA[i] = ldh(src, q);
    sG[i] = f3_guide(f.F3, q);
  }
  __syncthreads();
  const int X = bx + threadIdx.x, Y = by + threadIdx.y;
  if (X >= f.W2 || Y >= f.H2) return;
  const int o = Y * f.W2 + X;
  const int lx = threadIdx.x + AP, ly = threadIdx.y + AP;
  if (sG[ly * SW + lx].w < 0.0f) { sth(dst, o, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  const float4 a = ldh(f.par1, o), b = ldh(f.par2, o);
  const float s = COMP == 2 ? a.z : a.w, c = COMP == 2 ? b.z : b.w;
  sth(dst, o, filt<1, STEP, false, SW>(sA, sG, lx, ly, X, Y, f.W2, f.H2, s, c));
}

// ------------------------------------------------------------------------------------------------ COARSE1
// hush.js:385-421: down() of the half-res block means into the quarter-res tile (apron 2), the coarse guide, then
// the 5x5 step-1 a-trous with s = COARSE_S.
HD_INL void coarse_down(const HushFrame &f, int Qx, int Qy, float4 &c, float4 &g) {
  float N = 0.f, vr = 0.f, z = 0.f, cx = 0.f, cy = 0.f, cz = 0.f, nx = 0.f, ny = 0.f, nz = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int hx = Qx * 2 + (j & 1), hy = Qy * 2 + (j >> 1);
    if (hx >= f.W2 || hy >= f.H2) continue;
    const uint4 g3 = __ldg(f.F3 + hy * f.W2 + hx);
    const float2 oz = unpack2(g3.y);
    if (oz.y <= 0.0f) continue;
    const float4 a = f2_ac(f.F2, hy * f.W2 + hx);
    const float w = oz.y;
    N += w;
    cx += w * a.x; cy += w * a.y; cz += w * a.z;
    vr += w * a.w;
    const float2 oe = unpack2(g3.x);
    const float4 n = oct_dec(oe.x, oe.y);
    nx += w * n.x; ny += w * n.y; nz += w * n.z;
    z += w * oz.x;
  }
  if (N == 0.0f) {
    c = make_float4(0.f, 0.f, 0.f, 0.f);
    g = make_float4(0.f, 0.f, -1.0f, 0.f);
    return;
  }
  const float nl = fmaxf(sqrtf(nx * nx + ny * ny + nz * nz), 1e-6f);
  const float2 o = oct_enc(nx / nl, ny / nl, nz / nl);
  c = make_float4(qf16(cx / N), qf16(cy / N), qf16(cz / N), qf16(vr / N / N));
  g = make_float4(qf16(o.x), qf16(o.y), qf16(z / N), 0.0f);
}

__global__ void __launch_bounds__(TW *TH) k_coarse1(const __grid_constant__ HushFrame f) {
  constexpr int AP = 2, SW = TW + 2 * AP, SH = TH + 2 * AP;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const int li = threadIdx.y * TW + threadIdx.x;
  const int bx = blockIdx.x * TW, by = blockIdx.y * TH;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const int lqx = bx - AP + i % SW, lqy = by - AP + i / SW;
    const int qx = clampi(lqx, 0, f.W4 - 1), qy = clampi(lqy, 0, f.H4 - 1);
    float4 c, g;
    coarse_down(f, qx, qy, c, g);
    sA[i] = c;
    float4 gd = oct_dec(g.x, g.y);
    gd.w = g.z;
    sG[i] = gd;
    if (lqx == qx && lqy == qy && lqx >= bx && lqy >= by && lqx < bx + TW && lqy < by + TH)
      sth(f.CG, qy * f.W4 + qx, g);
  }
  __syncthreads();
  const int X = bx + threadIdx.x, Y = by + threadIdx.y;
  if (X >= f.W4 || Y >= f.H4) return;
  const int lx = threadIdx.x + AP, ly = threadIdx.y + AP;
  if (sG[ly * SW + lx].w < 0.0f) { sth(f.C1, Y * f.W4 + X, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  sth(f.C1, Y * f.W4 + X, filt<2, 1, true, SW>(sA, sG, lx, ly, X, Y, f.W4, f.H4, COARSE_S, 1.0f));
}

// atrousShader kind coarse (hush.js:752): C1 -> C0, 5x5, step 2, prefilter, guide CG.
__global__ void __launch_bounds__(TW *TH) k_coarse2(const __grid_constant__ HushFrame f) {
  constexpr int AP = 4, SW = TW + 2 * AP, SH = TH + 2 * AP;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const int li = threadIdx.y * TW + threadIdx.x;
  const int bx = blockIdx.x * TW, by = blockIdx.y * TH;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const int q = clampi(by - AP + i / SW, 0, f.H4 - 1) * f.W4 + clampi(bx - AP + i % SW, 0, f.W4 - 1);
    sA[i] = ldh(f.C1, q);
    const float4 g = ldh(f.CG, q);
    float4 gd = oct_dec(g.x, g.y);
    gd.w = g.z;
    sG[i] = gd;
  }
  __syncthreads();
  const int X = bx + threadIdx.x, Y = by + threadIdx.y;
  if (X >= f.W4 || Y >= f.H4) return;
  const int lx = threadIdx.x + AP, ly = threadIdx.y + AP;
  if (sG[ly * SW + lx].w < 0.0f) { sth(f.C0, Y * f.W4 + X, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  sth(f.C0, Y * f.W4 + X, filt<2, 2, true, SW>(sA, sG, lx, ly, X, Y, f.W4, f.H4, COARSE_S, 1.0f));
}

// ------------------------------------------------------------------------------------------------ FINE_FINAL
// Fine level + recombination + remodulation at one pixel (hush.js:573-620), given the fine a-trous result A1.
// Reads the half-res par0, block means / guide (Ah, Gh as decoded float4 loaders), the mid level and the coarse
// level. Returns X.
template <class LoadAh, class LoadGh>
HD_INL float4 fine_recombine(const HushFrame &f, int px, int py, float4 A1, float4 gp, float4 alb, float4 emi,
                             const uint2 *mid, LoadAh loadAh, LoadGh loadGh) {
  const float fx = qf16(A1.x), fy = qf16(A1.y), fz = qf16(A1.z);
  const float z = gp.w;
  const int hp = (py >> 1) * f.W2 + (px >> 1);
  const float4 pr = ldh(f.par0, hp);
  const int hsx = (f.W + 1) / 2, hsy = (f.H + 1) / 2;
  const float hposx = ((float)px + 0.5f) / 2.0f - 0.5f, hposy = ((float)py + 0.5f) / 2.0f - 0.5f;
  const float hbx = floorf(hposx), hby = floorf(hposy);
  float uBx = 0.f, uBy = 0.f, uBz = 0.f, uAx = 0.f, uAy = 0.f, uAz = 0.f, swh = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int qx = (int)hbx + (j & 1), qy = (int)hby + (j >> 1);
    if (qx < 0 || qy < 0 || qx >= hsx || qy >= hsy) continue;
    const int q = qy * f.W2 + qx;
    const float4 g = loadGh(q);  // decoded normal, depth
    if (g.w < 0.0f) continue;
    const float w = jbw(hposx - hbx, hposy - hby, j, g, g.w, gp, z);
    const float4 a = loadAh(q);
    const float4 m = ldh(mid, q);
    swh += w;
    uBx += w * m.x; uBy += w * m.y; uBz += w * m.z;
    uAx += w * a.x; uAy += w * a.y; uAz += w * a.z;
  }
  float ix = fx, iy = fy, iz = fz;
  if (swh > 1e-4f) {
    ix = uBx / swh + pr.w * (fx - uAx / swh);
    iy = uBy / swh + pr.w * (fy - uAy / swh);
    iz = uBz / swh + pr.w * (fz - uAz / swh);
  }
  const int qsx = (f.W + 3) / 4, qsy = (f.H + 3) / 4;
  const float cposx = ((float)px + 0.5f) / 4.0f - 0.5f, cposy = ((float)py + 0.5f) / 4.0f - 0.5f;
  const float cbx = floorf(cposx), cby = floorf(cposy);
  float uCx = 0.f, uCy = 0.f, uCz = 0.f, swq = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int qx = (int)cbx + (j & 1), qy = (int)cby + (j >> 1);
    if (qx < 0 || qy < 0 || qx >= qsx || qy >= qsy) continue;
    const int q = qy * f.W4 + qx;
    const float4 cg = ldh(f.CG, q);
    if (cg.z < 0.0f) continue;
    const float w = jbw(cposx - cbx, cposy - cby, j, oct_dec(cg.x, cg.y), cg.z, gp, z);
    const float4 c = ldh(f.C0, q);
    swq += w;
    uCx += w * c.x; uCy += w * c.y; uCz += w * c.z;
  }
  float upx = ix, upy = iy, upz = iz;
  if (swq > 1e-4f) { upx = uCx / swq; upy = uCy / swq; upz = uCz / swq; }
  ix = ix + (upx - ix) * pr.z;
  iy = iy + (upy - iy) * pr.z;
  iz = iz + (upz - iz) * pr.z;
  return make_float4(ix * alb.x + emi.x, iy * alb.y + emi.y, iz * alb.z + emi.z, 0.0f);
}

__global__ void __launch_bounds__(TW *TH) k_fine_final(const __grid_constant__ HushFrame f) {
  constexpr int AP = 1, SW = TW + 2, SH = TH + 2;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const int li = threadIdx.y * TW + threadIdx.x;
  const int bx = blockIdx.x * TW, by = blockIdx.y * TH;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const int q = clampi(by - AP + i / SW, 0, f.H - 1) * f.W + clampi(bx - AP + i % SW, 0, f.W - 1);
    sA[i] = ldh(f.A0, q);
    const float4 k = ldh(f.key, q);
    float4 g = oct_dec(k.x, k.y);
    g.w = k.z;
    sG[i] = g;
  }
  __syncthreads();
  const int px = bx + threadIdx.x, py = by + threadIdx.y;
  if (px >= f.W || py >= f.H) return;
  const int lx = threadIdx.x + AP, ly = threadIdx.y + AP;
  const float4 alb = ldh(f.mat, py * f.p_mat + px), emi = ldh(f.emi, py * f.p_emi + px);
  const float4 gp = sG[ly * SW + lx];
  const int o = py * f.W + px;
  if (gp.w < 0.0f) {
    sth(f.hist, o, make_float4(0.f, 0.f, 0.f, 0.f));
    sth(f.X, o, make_float4(emi.x, emi.y, emi.z, 0.f));
    return;
  }
  const int hp = (py >> 1) * f.W2 + (px >> 1);
  const float4 A1 = filt<1, 1, true, SW>(sA, sG, lx, ly, px, py, f.W, f.H, ldh(f.par1, hp).x, ldh(f.par2, hp).x);
  sth(f.hist, o, A1);
  const uint4 *F2 = f.F2, *F3 = f.F3;
  sth(f.X, o,
      fine_recombine(f, px, py, A1, gp, alb, emi, f.Bh0, [&](int q) { return f2_ac(F2, q); },
                     [&](int q) { return f3_guide(F3, q); }));
}

// ------------------------------------------------------------------------------------------------ TAA
// hush.js:639-677. sX holds YCoCg(tm(X)) of a clamp-to-edge tile.
HD_INL float3 taa_resolve(const HushFrame &f, int px, int py, float3 cur, const float3 *sX, int ti, int SW) {
  float3 m1 = make_float3(0.f, 0.f, 0.f);
#pragma unroll
  for (int j = 0; j < 9; j++) {
    const float3 c = sX[ti + (j / 3 - 1) * SW + (j % 3 - 1)];
    m1.x += c.x; m1.y += c.y; m1.z += c.z;
  }
  m1.x /= 9.0f; m1.y /= 9.0f; m1.z /= 9.0f;
  float3 v3 = make_float3(0.f, 0.f, 0.f);
#pragma unroll
  for (int j = 0; j < 9; j++) {
    const float3 c = sX[ti + (j / 3 - 1) * SW + (j % 3 - 1)];
    const float dx = c.x - m1.x, dy = c.y - m1.y, dz = c.z - m1.z;
    v3.x += dx * dx; v3.y += dy * dy; v3.z += dz * dz;
  }
  const float sdx = sqrtf(fmaxf(v3.x / 9.0f, 1e-12f)), sdy = sqrtf(fmaxf(v3.y / 9.0f, 1e-12f)),
              sdz = sqrtf(fmaxf(v3.z / 9.0f, 1e-12f));
  const float4 mv = ldh(f.mv, py * f.p_mv + px);
  const float szx = (float)f.W, szy = (float)f.H;
  const float uvx = ((float)px + 0.5f + mv.x) / szx, uvy = ((float)py + 0.5f + mv.y) / szy;
  float3 res = cur;
  if (uvx >= 0.0f && uvy >= 0.0f && uvx <= 1.0f && uvy <= 1.0f) {
    const float ppx = uvx * szx - 0.5f, ppy = uvy * szy - 0.5f;
    const float bx = floorf(ppx), by = floorf(ppy);
    const float fx = ppx - bx, fy = ppy - by;
    const int ibx = (int)bx, iby = (int)by;
    float3 hist = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int ox = j & 1, oy = j >> 1;
      const float wb = (ox == 1 ? fx : 1.0f - fx) * (oy == 1 ? fy : 1.0f - fy);
      const float4 t = ldh(f.taa_prev, clampi(iby + oy, 0, f.H - 1) * f.W + clampi(ibx + ox, 0, f.W - 1));
      hist.x += wb * t.x; hist.y += wb * t.y; hist.z += wb * t.z;
    }
    float3 hh = to_ycocg(tmap(hist));
    hh.x = fminf(fmaxf(hh.x, m1.x - 1.25f * sdx), m1.x + 1.25f * sdx);
    hh.y = fminf(fmaxf(hh.y, m1.y - 1.25f * sdy), m1.y + 1.25f * sdy);
    hh.z = fminf(fmaxf(hh.z, m1.z - 1.25f * sdz), m1.z + 1.25f * sdz);
    const float3 hr = from_ycocg(hh);
    res = make_float3(hr.x + (cur.x - hr.x) * 0.1f, hr.y + (cur.y - hr.y) * 0.1f, hr.z + (cur.z - hr.z) * 0.1f);
  }
  return itmap(res);
}

__global__ void __launch_bounds__(TW *TH) k_taa(const __grid_constant__ HushFrame f) {
  constexpr int SW = TW + 2, SH = TH + 2;
  __shared__ float3 sX[SW * SH];
  const int li = threadIdx.y * TW + threadIdx.x;
  const int ox = blockIdx.x * TW - 1, oy = blockIdx.y * TH - 1;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const float4 x = ldh(f.X, clampi(oy + i / SW, 0, f.H - 1) * f.W + clampi(ox + i % SW, 0, f.W - 1));
    sX[i] = to_ycocg(tmap(make_float3(x.x, x.y, x.z)));
  }
  __syncthreads();
  const int px = blockIdx.x * TW + threadIdx.x, py = blockIdx.y * TH + threadIdx.y;
  if (px >= f.W || py >= f.H) return;
  const int o = py * f.W + px;
  const float4 x = ldh(f.X, o);
  const float3 cur = tmap(make_float3(x.x, x.y, x.z));
  float3 r;
  if (f.reset) r = itmap(cur);
  else r = taa_resolve(f, px, py, cur, sX, (threadIdx.y + 1) * SW + threadIdx.x + 1, SW);
  sth(f.taa, o, make_float4(r.x, r.y, r.z, 1.0f));
}

// ------------------------------------------------------------------------------------------------ launchers
static dim3 tiles(int w, int h) { return dim3((w + TW - 1) / TW, (h + TH - 1) / TH); }

cudaError_t launch_pass(int pass, const HushFrame &f, const MlpW16 &w16, cudaStream_t st) {
  const dim3 blk(TW, TH);
  switch (pass) {
    case PASS_TEMPORAL: k_temporal<<<tiles(f.W, f.H), blk, 0, st>>>(f); break;
    case PASS_INFER:
      if (f.hidden == 16) k_infer<16><<<tiles(f.W2, f.H2), blk, 0, st>>>(f, w16);
      else k_infer<0><<<tiles(f.W2, f.H2), blk, 0, st>>>(f, w16);
      break;
    case PASS_MID2: k_mid<2, 2><<<tiles(f.W2, f.H2), blk, 0, st>>>(f, f.Bh0, f.Bh1); break;
    case PASS_MID3: k_mid<4, 3><<<tiles(f.W2, f.H2), blk, 0, st>>>(f, f.Bh1, f.Bh0); break;
    case PASS_COARSE1: k_coarse1<<<tiles(f.W4, f.H4), blk, 0, st>>>(f); break;
    case PASS_COARSE2: k_coarse2<<<tiles(f.W4, f.H4), blk, 0, st>>>(f); break;
    case PASS_FINE_FINAL: k_fine_final<<<tiles(f.W, f.H), blk, 0, st>>>(f); break;
    case PASS_TAA: k_taa<<<tiles(f.W, f.H), blk, 0, st>>>(f); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace hush
