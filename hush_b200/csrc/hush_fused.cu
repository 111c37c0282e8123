// The fused B200 frame. Same arithmetic as the per-pass kernels (hush_passes.cu); different kernel boundaries:
//
//   stage 0  temporal   TEMPORAL + block features + the MLP heads (hush.js:79-308, 312-365) in one kernel: the 2x2
//                       blocks align with the tile, so the 20 features never leave the SM (the reference writes
//                       F0/F1 and reads them back in INFER). Writes A0, mom, key, par0..2 and the half-res block
//                       means Ah (= F2.zw) and guide Gh (= F3.xy).
//   stage 1  mid1|c1    mid1 (INFER's a-trous, hush.js:366) and COARSE1 (hush.js:404-421) in one launch
//   stage 2  mid2|c2    mid2 (hush.js:753) and coarse2 (hush.js:752) in one launch
//   stage 3  mid3       hush.js:754
//   stage 4  fine+final hush.js:560-621
//   stage 5  taa        hush.js:639-677
//
// Levels with a neighbourhood (the a-trous levels, TAA) stay separate launches: fusing them needs recomputed halos,
// and on B200 these passes are bound by instruction issue rather than HBM, so recomputation costs more than the
// L2-resident round trip of a half-res image.
#include "hush_device.cuh"
#include "hush_internal.h"

namespace hush {

// ------------------------------------------------------------------------------------------------ loaders
HD_INL float4 gh_decode(float4 g) {  // (oct normal, depth, count) -> (normal, depth)
  float4 n = oct_dec(g.x, g.y);
  n.w = g.z;
  return n;
}

// ------------------------------------------------------------------------------------------------ stage 0
// Tile 32 x 8 pixels = 16 x 4 blocks, 256 threads; the illumination tile carries an apron of 1.
constexpr int K1_TW = 32, K1_TH = 8;

template <bool TC>
__global__ void __launch_bounds__(K1_TW *K1_TH, 3)
    k_temporal_fused(const __grid_constant__ HushFrame f, const __grid_constant__ MlpW16 w) {
  constexpr int SW = K1_TW + 2, SH = K1_TH + 2, NT = K1_TW * K1_TH, NB = (K1_TW / 2) * (K1_TH / 2);
  __shared__ float4 sI[SW * SH];
  __shared__ PixP sP[NT];
  const int li = threadIdx.x;
  const int tx = li % K1_TW, ty = li / K1_TW;
  const int ox = blockIdx.x * K1_TW - 1, oy = blockIdx.y * K1_TH - 1;
  for (int i = li; i < SW * SH; i += NT) {
    const int qx = ox + i % SW, qy = oy + i / SW;
    float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
    if (qx >= 0 && qy >= 0 && qx < f.W && qy < f.H && ldh(f.nd, qy * f.p_nd + qx).w >= 0.0f) {
      const float4 r = ldh(f.rad, qy * f.p_rad + qx), m = ldh(f.mat, qy * f.p_mat + qx);
      e = make_float4(r.x / fmaxf(m.x, 1e-3f), r.y / fmaxf(m.y, 1e-3f), r.z / fmaxf(m.z, 1e-3f), 1.0f);
    }
    sI[i] = e;
  }
  __syncthreads();
  const int px = blockIdx.x * K1_TW + tx, py = blockIdx.y * K1_TH + ty;
  PixP P = pixp_default();
  if (px < f.W && py < f.H) P = temporal_pixel<SW>(f, px, py, sI, tx + 1, ty + 1);
  sP[li] = P;
  __syncthreads();
  if (li >= NB) return;
  const int lbx = li % (K1_TW / 2), lby = li / (K1_TW / 2);
  const int X = blockIdx.x * (K1_TW / 2) + lbx, Y = blockIdx.y * (K1_TH / 2) + lby;
  if (X >= f.W2 || Y >= f.H2) return;
  PixP Pj[4];
#pragma unroll
  for (int j = 0; j < 4; j++) Pj[j] = sP[(lby * 2 + (j >> 1)) * K1_TW + lbx * 2 + (j & 1)];
  float fe[N_FEAT];
  float4 AC, G;
  const int o = Y * f.W2 + X;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  if (!block_features<SW>(Pj, sI, (2 * lby) * SW + 2 * lbx, f.exposure, fe, AC, G)) {
    // INFER on a block without valid pixels (hush.js:343-346) and its packed F2/F3 (hush.js:241-244)
    f.Ah[o] = make_uint2(0, 0);
    f.Gh[o] = make_uint2(pk(0.f, 0.f), pk(-1.0f, 0.f));
    sth(f.par0, o, z4); sth(f.par1, o, z4); sth(f.par2, o, z4);
    return;
  }
  f.Ah[o] = make_uint2(pk(AC.x, AC.y), pk(AC.z, AC.w));
  f.Gh[o] = make_uint2(pk(G.x, G.y), pk(G.z, G.w));
  // the MLP sees the features as stored (packed f16, hush.js:278-280, 348-353)
#pragma unroll
  for (int i = 0; i < N_FEAT; i++) fe[i] = __half2float(__ushort_as_half(f2h(qf16(fe[i]))));
  float out[N_OUT];
  mlp_fwd<16>(w.w, fe, out);
  float4 p0, p1, p2;
  mlp_heads(out, p0, p1, p2);
  sth(f.par0, o, p0);
  sth(f.par1, o, p1);
  sth(f.par2, o, p2);
}

// ------------------------------------------------------------------------------------------------ half / quarter
// 16 x 8 tiles like the reference. One launch runs two kinds of tiles: blockIdx.x < nA runs kind A, the rest kind B.
constexpr int HT_W = 16, HT_H = 8;

// mid1 (hush.js:326, 366): 3x3 step 1 with prefilter on the block means, learned s_1 / c_1 (stored par1.y / par2.y
// are the qf16 values INFER passes).
HD_INL void tile_mid1(const HushFrame &f, int tileX, int tileY, float4 *sA, float4 *sG) {
  constexpr int AP = 1, SW = HT_W + 2, SH = HT_H + 2;
  const int li = threadIdx.x;
  const int bx = tileX * HT_W, by = tileY * HT_H;
  for (int i = li; i < SW * SH; i += HT_W * HT_H) {
    const int q = clampi(by - AP + i / SW, 0, f.H2 - 1) * f.W2 + clampi(bx - AP + i % SW, 0, f.W2 - 1);
    sA[i] = ldh(f.Ah, q);
    sG[i] = gh_decode(ldh(f.Gh, q));
  }
  __syncthreads();
  const int X = bx + li % HT_W, Y = by + li / HT_W;
  if (X >= f.W2 || Y >= f.H2) return;
  const int lx = li % HT_W + AP, ly = li / HT_W + AP;
  const int o = Y * f.W2 + X;
  if (sG[ly * SW + lx].w < 0.0f) { sth(f.Bh0, o, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  const float s = ldh(f.par1, o).y, c = ldh(f.par2, o).y;
  sth(f.Bh0, o, filt<1, 1, true, SW>(sA, sG, lx, ly, X, Y, f.W2, f.H2, s, c));
}

template <int STEP, int COMP>
HD_INL void tile_mid(const HushFrame &f, int tileX, int tileY, const uint2 *src, uint2 *dst, float4 *sA, float4 *sG) {
  constexpr int AP = STEP, SW = HT_W + 2 * AP, SH = HT_H + 2 * AP;
  const int li = threadIdx.x;
  const int bx = tileX * HT_W, by = tileY * HT_H;
  for (int i = li; i < SW * SH; i += HT_W * HT_H) {
    const int q = clampi(by - AP + i / SW, 0, f.H2 - 1) * f.W2 + clampi(bx - AP + i % SW, 0, f.W2 - 1);
    sA[i] = ldh(src, q);
    sG[i] = gh_decode(ldh(f.Gh, q));
  }
  __syncthreads();
  const int X = bx + li % HT_W, Y = by + li / HT_W;
  if (X >= f.W2 || Y >= f.H2) return;
  const int lx = li % HT_W + AP, ly = li / HT_W + AP;
  const int o = Y * f.W2 + X;
  if (sG[ly * SW + lx].w < 0.0f) { sth(dst, o, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  const float4 a = ldh(f.par1, o), b = ldh(f.par2, o);
  const float s = COMP == 2 ? a.z : a.w, c = COMP == 2 ? b.z : b.w;
  sth(dst, o, filt<1, STEP, false, SW>(sA, sG, lx, ly, X, Y, f.W2, f.H2, s, c));
}

// down() (hush.js:385-402) from the half-res planes.
HD_INL void down_h(const HushFrame &f, int Qx, int Qy, float4 &c, float4 &g) {
  float N = 0.f, vr = 0.f, z = 0.f, cx = 0.f, cy = 0.f, cz = 0.f, nx = 0.f, ny = 0.f, nz = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int hx = Qx * 2 + (j & 1), hy = Qy * 2 + (j >> 1);
    if (hx >= f.W2 || hy >= f.H2) continue;
    const float4 gq = ldh(f.Gh, hy * f.W2 + hx);
    if (gq.w <= 0.0f) continue;
    const float4 a = ldh(f.Ah, hy * f.W2 + hx);
    const float w = gq.w;
    N += w;
    cx += w * a.x; cy += w * a.y; cz += w * a.z;
    vr += w * a.w;
    const float4 n = oct_dec(gq.x, gq.y);
    nx += w * n.x; ny += w * n.y; nz += w * n.z;
    z += w * gq.z;
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

HD_INL void tile_coarse1(const HushFrame &f, int tileX, int tileY, float4 *sA, float4 *sG) {
  constexpr int AP = 2, SW = HT_W + 2 * AP, SH = HT_H + 2 * AP;
  const int li = threadIdx.x;
  const int bx = tileX * HT_W, by = tileY * HT_H;
  for (int i = li; i < SW * SH; i += HT_W * HT_H) {
    const int lqx = bx - AP + i % SW, lqy = by - AP + i / SW;
    const int qx = clampi(lqx, 0, f.W4 - 1), qy = clampi(lqy, 0, f.H4 - 1);
    float4 c, g;
    down_h(f, qx, qy, c, g);
    sA[i] = c;
    sG[i] = gh_decode(g);
    if (lqx == qx && lqy == qy && lqx >= bx && lqy >= by && lqx < bx + HT_W && lqy < by + HT_H)
      sth(f.CG, qy * f.W4 + qx, g);
  }
  __syncthreads();
  const int X = bx + li % HT_W, Y = by + li / HT_W;
  if (X >= f.W4 || Y >= f.H4) return;
  const int lx = li % HT_W + AP, ly = li / HT_W + AP;
  if (sG[ly * SW + lx].w < 0.0f) { sth(f.C1, Y * f.W4 + X, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  sth(f.C1, Y * f.W4 + X, filt<2, 1, true, SW>(sA, sG, lx, ly, X, Y, f.W4, f.H4, COARSE_S, 1.0f));
}

HD_INL void tile_coarse2(const HushFrame &f, int tileX, int tileY, float4 *sA, float4 *sG) {
  constexpr int AP = 4, SW = HT_W + 2 * AP, SH = HT_H + 2 * AP;
  const int li = threadIdx.x;
  const int bx = tileX * HT_W, by = tileY * HT_H;
  for (int i = li; i < SW * SH; i += HT_W * HT_H) {
    const int q = clampi(by - AP + i / SW, 0, f.H4 - 1) * f.W4 + clampi(bx - AP + i % SW, 0, f.W4 - 1);
    sA[i] = ldh(f.C1, q);
    sG[i] = gh_decode(ldh(f.CG, q));
  }
  __syncthreads();
  const int X = bx + li % HT_W, Y = by + li / HT_W;
  if (X >= f.W4 || Y >= f.H4) return;
  const int lx = li % HT_W + AP, ly = li / HT_W + AP;
  if (sG[ly * SW + lx].w < 0.0f) { sth(f.C0, Y * f.W4 + X, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  sth(f.C0, Y * f.W4 + X, filt<2, 2, true, SW>(sA, sG, lx, ly, X, Y, f.W4, f.H4, COARSE_S, 1.0f));
}

// stage 1: mid1 tiles then coarse1 tiles; stage 2: mid2 tiles then coarse2 tiles; stage 3: mid3 tiles.
template <int STAGE>
__global__ void __launch_bounds__(HT_W *HT_H) k_half_stage(const __grid_constant__ HushFrame f, int nAx, int nA,
                                                           int nBx) {
  constexpr int SMAX = (HT_W + 8) * (HT_H + 8);
  __shared__ float4 sA[SMAX], sG[SMAX];
  const int b = blockIdx.x;
  if (b < nA) {
    const int tX = b % nAx, tY = b / nAx;
    if (STAGE == 1) tile_mid1(f, tX, tY, sA, sG);
    else if (STAGE == 2) tile_mid<2, 2>(f, tX, tY, f.Bh0, f.Bh1, sA, sG);
    else tile_mid<4, 3>(f, tX, tY, f.Bh1, f.Bh0, sA, sG);
  } else {
    const int t = b - nA, tX = t % nBx, tY = t / nBx;
    if (STAGE == 1) tile_coarse1(f, tX, tY, sA, sG);
    else if (STAGE == 2) tile_coarse2(f, tX, tY, sA, sG);
  }
}

// ------------------------------------------------------------------------------------------------ stage 4 / 5
constexpr int FT_W = 32, FT_H = 8;

__global__ void __launch_bounds__(FT_W *FT_H) k_fine_final_fused(const __grid_constant__ HushFrame f) {
  constexpr int AP = 1, SW = FT_W + 2, SH = FT_H + 2;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const int li = threadIdx.x;
  const int bx = blockIdx.x * FT_W, by = blockIdx.y * FT_H;
  for (int i = li; i < SW * SH; i += FT_W * FT_H) {
    const int q = clampi(by - AP + i / SW, 0, f.H - 1) * f.W + clampi(bx - AP + i % SW, 0, f.W - 1);
    sA[i] = ldh(f.A0, q);
    const float4 k = ldh(f.key, q);
    float4 g = oct_dec(k.x, k.y);
    g.w = k.z;
    sG[i] = g;
  }
  __syncthreads();
  const int px = bx + li % FT_W, py = by + li / FT_W;
  if (px >= f.W || py >= f.H) return;
  const int lx = li % FT_W + AP, ly = li / FT_W + AP;
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
  // recombination (hush.js:580-620) with the half-res block means / guide from Ah / Gh
  const float fx = qf16(A1.x), fy = qf16(A1.y), fz = qf16(A1.z);
  const float z = gp.w;
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
    const float4 g = ldh(f.Gh, q);
    if (g.z < 0.0f) continue;
    const float w = jbw(hposx - hbx, hposy - hby, j, oct_dec(g.x, g.y), g.z, gp, z);
    const float4 a = ldh(f.Ah, q);
    const float4 m = ldh(f.Bh0, q);
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
  sth(f.X, o, make_float4(ix * alb.x + emi.x, iy * alb.y + emi.y, iz * alb.z + emi.z, 0.0f));
}

// TAA (hush.js:639-677) with a 32 x 8 tile.
__global__ void __launch_bounds__(FT_W *FT_H) k_taa_fused(const __grid_constant__ HushFrame f) {
  constexpr int SW = FT_W + 2, SH = FT_H + 2;
  __shared__ float3 sX[SW * SH];
  const int li = threadIdx.x;
  const int ox = blockIdx.x * FT_W - 1, oy = blockIdx.y * FT_H - 1;
  for (int i = li; i < SW * SH; i += FT_W * FT_H) {
    const float4 x = ldh(f.X, clampi(oy + i / SW, 0, f.H - 1) * f.W + clampi(ox + i % SW, 0, f.W - 1));
    sX[i] = to_ycocg(tmap(make_float3(x.x, x.y, x.z)));
  }
  __syncthreads();
  const int tx = li % FT_W, ty = li / FT_W;
  const int px = blockIdx.x * FT_W + tx, py = blockIdx.y * FT_H + ty;
  if (px >= f.W || py >= f.H) return;
  const int o = py * f.W + px;
  const float4 x = ldh(f.X, o);
  const float3 cur = tmap(make_float3(x.x, x.y, x.z));
  float3 r;
  if (f.reset) {
    r = itmap(cur);
  } else {
    const int ti = (ty + 1) * SW + tx + 1;
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
      const float bxf = floorf(ppx), byf = floorf(ppy);
      const float fx = ppx - bxf, fy = ppy - byf;
      const int ibx = (int)bxf, iby = (int)byf;
      float3 hist = make_float3(0.f, 0.f, 0.f);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int oxj = j & 1, oyj = j >> 1;
        const float wb = (oxj == 1 ? fx : 1.0f - fx) * (oyj == 1 ? fy : 1.0f - fy);
        const float4 t = ldh(f.taa_prev, clampi(iby + oyj, 0, f.H - 1) * f.W + clampi(ibx + oxj, 0, f.W - 1));
        hist.x += wb * t.x; hist.y += wb * t.y; hist.z += wb * t.z;
      }
      float3 hh = to_ycocg(tmap(hist));
      hh.x = fminf(fmaxf(hh.x, m1.x - 1.25f * sdx), m1.x + 1.25f * sdx);
      hh.y = fminf(fmaxf(hh.y, m1.y - 1.25f * sdy), m1.y + 1.25f * sdy);
      hh.z = fminf(fmaxf(hh.z, m1.z - 1.25f * sdz), m1.z + 1.25f * sdz);
      const float3 hr = from_ycocg(hh);
      res = make_float3(hr.x + (cur.x - hr.x) * 0.1f, hr.y + (cur.y - hr.y) * 0.1f, hr.z + (cur.z - hr.z) * 0.1f);
    }
    r = itmap(res);
  }
  sth(f.taa, o, make_float4(r.x, r.y, r.z, 1.0f));
}

// ------------------------------------------------------------------------------------------------ launchers
static const char *STAGE_LABELS[6] = {"temporal+mlp", "mid1+coarse1", "mid2+coarse2", "mid3", "fine+final", "taa"};
int fused_stage_count() { return 6; }
const char *fused_stage_label(int s) { return (s >= 0 && s < 6) ? STAGE_LABELS[s] : "?"; }

cudaError_t launch_fused_stage(int stage, const HushFrame &f, const MlpW16 &w16, int mlp_mode, const void *mlp_tc,
                               cudaStream_t st) {
  (void)mlp_mode;
  (void)mlp_tc;
  const int hx = (f.W2 + HT_W - 1) / HT_W, hy = (f.H2 + HT_H - 1) / HT_H;
  const int qx = (f.W4 + HT_W - 1) / HT_W, qy = (f.H4 + HT_H - 1) / HT_H;
  switch (stage) {
    case 0:
      k_temporal_fused<false><<<dim3((f.W + K1_TW - 1) / K1_TW, (f.H + K1_TH - 1) / K1_TH), K1_TW * K1_TH, 0, st>>>(
          f, w16);
      break;
    case 1: k_half_stage<1><<<hx * hy + qx * qy, HT_W * HT_H, 0, st>>>(f, hx, hx * hy, qx); break;
    case 2: k_half_stage<2><<<hx * hy + qx * qy, HT_W * HT_H, 0, st>>>(f, hx, hx * hy, qx); break;
    case 3: k_half_stage<3><<<hx * hy, HT_W * HT_H, 0, st>>>(f, hx, hx * hy, qx); break;
    case 4: k_fine_final_fused<<<dim3((f.W + FT_W - 1) / FT_W, (f.H + FT_H - 1) / FT_H), FT_W * FT_H, 0, st>>>(f); break;
    case 5: k_taa_fused<<<dim3((f.W + FT_W - 1) / FT_W, (f.H + FT_H - 1) / FT_H), FT_W * FT_H, 0, st>>>(f); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

size_t fused_scratch_bytes(int, int) { return 0; }

}  // namespace hush
