// Training twin of the Hush frame: hand-written forward / adjoint kernels for on-device training of the parameter MLP.
//
// The twin runs the frame after TEMPORAL in FP32 without the f16 storage rounding (so finite differences see a
// smooth function): the MLP on FP32 master weights (hush.js:683-704 / 357-362), the mid levels mid1-mid3 (hush.js:366,
// 753-754), the fine level + recombination (hush.js:578-620) and TAA (hush.js:649-676). TEMPORAL and the coarse levels
// run as the reference passes in the frame (their outputs do not depend on the weights within a frame); each also has
// its own forward / adjoint pair in the per-pass API, and TEMPORAL's adjoint drives the window sweep through time. The
// loss is the relative L1 of the TAA output against the noise-free image (clipped at 1 per value) plus a
// temporal-gradient term.
//
// Gradients are exact for one frame with the temporal history held fixed (the history buffers are inputs of the
// frame); over a window the per-frame gradients are summed (truncated backpropagation through time: the alpha / gamma
// heads, which only act on the next frame's temporal blend, receive no gradient). The backward recomputes every
// a-trous weight from the level's input instead of storing the weights, accumulates input gradients of the levels with
// atomics, reduces the weight gradient per CTA in FP32 and across CTAs in FP64, and updates FP32 master weights with
// Adam.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "hush.h"
#include "hush_device.cuh"
#include "hush_instance.h"
#include "hush_internal.h"
#include "umma.cuh"

namespace hush {
namespace twin {

constexpr int NW = H16_COUNT;  // 812 weights of the h = 16 network
constexpr int TW = 16, TH = 8;
constexpr int W1o = 0, B1o = 16 * 20, W2o = B1o + 16, B2o = W2o + 256, W3o = B2o + 16, B3o = W3o + 12 * 16;

struct TwinFrame {
  HushFrame f;            // instance buffers of the frame (inputs, A0, key, F0..F3, C0, CG, history)
  const float *theta;     // FP32 master weights
  float4 *par;            // half: 3 float4 per row (alpha gamma beta kappa | s0..s3 | c0..c3)
  float4 *B1, *B2, *B3;   // half: mid levels
  float4 *A1, *X, *out;   // full: fine level, pre-TAA colour, TAA output
  const float4 *out_prev; // full: previous frame's TAA output (temporal loss term)
  const float *clean, *clean_prev;  // full: noise-free rgb (f32, dense), previous frame's
  float4 *gT;             // full: gradient w.r.t. the tone-mapped colour tm(X)
  float4 *dB1, *dB2, *dB3;  // half: level gradients
  const float4 *gA1;        // full: dL/d fine level through the colour history (the next frame's TEMPORAL), or NULL
  float4 *dA0;              // full: dL/d TEMPORAL's colour + variance A0 (the fine level's input), or NULL
  float4 *dAh;              // half: dL/d block means (F2.zw) from mid1 and the recombination, or NULL
  float4 *dC0;              // quarter: dL/d coarse level C0 from the recombination, or NULL
  float4 *dpar;           // half: 3 float4 per row
  float *partials;        // per-CTA weight-gradient partials (NW floats each)
  double *loss_partials;  // per-CTA loss partials
  float lambda_t;         // weight of the temporal term
  int has_prev;
  float inv_n;            // 1 / (3 * pixels)
  int zero_adj;           // forward kernels clear the adjoint accumulators (dpar, dB1..dB3) they precede
};

HD_INL float4 f3_guide_tw(const uint4 *F3, int i) {
  const uint4 t = __ldg(F3 + i);
  const float2 o = unpack2(t.x), z = unpack2(t.y);
  float4 g = oct_dec(o.x, o.y);
  g.w = z.x;
  return g;
}
HD_INL float4 f2_ac_tw(const uint4 *F2, int i) {
  const uint4 t = __ldg(F2 + i);
  const float2 a = unpack2(t.z), b = unpack2(t.w);
  return make_float4(a.x, a.y, b.x, b.y);
}
HD_INL void atomic_add4(float4 *p, float4 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
  atomicAdd(&p->z, v.z);
  atomicAdd(&p->w, v.w);
}
HD_INL float sgn(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

// ------------------------------------------------------------------------------------------------ MLP
HD_INL void mlp_full(const float *th, const float *fe, float *h1, float *h2, float *o) {
  for (int j = 0; j < 16; j++) {
    float a = th[B1o + j];
    for (int i = 0; i < 20; i++) a = a + fe[i] * th[W1o + j * 20 + i];
    h1[j] = fmaxf(a, 0.0f);
  }
  for (int j = 0; j < 16; j++) {
    float a = th[B2o + j];
    for (int i = 0; i < 16; i++) a = a + h1[i] * th[W2o + j * 16 + i];
    h2[j] = fmaxf(a, 0.0f);
  }
  for (int j = 0; j < 12; j++) {
    float a = th[B3o + j];
    for (int i = 0; i < 16; i++) a = a + h2[i] * th[W3o + j * 16 + i];
    o[j] = a;
  }
}

HD_INL void load_features(const HushFrame &f, int o, float *fe) {
  const uint4 a = __ldg(f.F0 + o), b = __ldg(f.F1 + o), c = __ldg(f.F2 + o);
  const uint32_t u[10] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y};
  for (int i = 0; i < 10; i++) {
    const float2 t = unpack2(u[i]);
    fe[2 * i] = t.x;
    fe[2 * i + 1] = t.y;
  }
}

// MLP forward and heads per half-res pixel; also writes the instance's f16 par0..2 (the next frame's history).
__global__ void k_mlp_fwd(const TwinFrame T) {
  __shared__ float th[NW];
  for (int i = threadIdx.x; i < NW; i += blockDim.x) th[i] = T.theta[i];
  __syncthreads();
  const HushFrame &f = T.f;
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= f.W2 * f.H2) return;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  if (T.zero_adj) { T.dpar[3 * o] = z4; T.dpar[3 * o + 1] = z4; T.dpar[3 * o + 2] = z4; }
  if (f3_guide_tw(f.F3, o).w < 0.0f) {
    T.par[3 * o] = z4; T.par[3 * o + 1] = z4; T.par[3 * o + 2] = z4;
    sth(f.par0, o, z4); sth(f.par1, o, z4); sth(f.par2, o, z4);
    return;
  }
  float fe[20], h1[16], h2[16], out[12];
  load_features(f, o, fe);
  mlp_full(th, fe, h1, h2, out);
  float4 p0, p1, p2;
  mlp_heads(out, p0, p1, p2);
  T.par[3 * o] = p0; T.par[3 * o + 1] = p1; T.par[3 * o + 2] = p2;
  sth(f.par0, o, p0); sth(f.par1, o, p1); sth(f.par2, o, p2);
}

// ------------------------------------------------------------------------------------------------ a-trous (R = 1)
// Forward of atrousFn with R = 1 over float4 tiles (see hush_device.cuh filt); the weight gradient helper below
// recomputes exactly these weights.
template <int STEP, bool PREF, int SW>
struct Filt1 {
  float4 gp, center;
  float gv, lc, den, sl, cw, W;
  float wq[8], lq[8];
  bool ok[8];
  float3 S;
  float V;
  HD_INL void run(const float4 *sA, const float4 *sG, int ti, int qx, int qy, int w, int h, float s, float c) {
    gp = sG[ti];
    center = sA[ti];
    if (PREF) {
      gv = 0.0625f * (sA[ti - SW - 1].w + sA[ti - SW + 1].w + sA[ti + SW - 1].w + sA[ti + SW + 1].w) +
           0.125f * (sA[ti - SW].w + sA[ti - 1].w + sA[ti + 1].w + sA[ti + SW].w) + 0.25f * center.w;
    } else {
      gv = center.w;
    }
    lc = lum(center);
    den = sqrtf(fmaxf(gv, 1e-12f)) + 1e-6f;
    sl = s / den;
    const float zl = sG[ti - 1].w, zr = sG[ti + 1].w, zu = sG[ti - SW].w, zd = sG[ti + SW].w;
    const float gx = fminf(zr > 0.0f ? fabsf(zr - gp.w) : 1e9f, zl > 0.0f ? fabsf(zl - gp.w) : 1e9f);
    const float gy = fminf(zd > 0.0f ? fabsf(zd - gp.w) : 1e9f, zu > 0.0f ? fabsf(zu - gp.w) : 1e9f);
    const float zg = fminf(fmaxf(gx, gy), gp.w);
    const float iz1 = 1.0f / (zg * (1.0f * STEP) + 1e-3f), iz2 = 1.0f / (zg * (1.41421356237309515f * STEP) + 1e-3f);
    cw = 0.25f * c;
    W = cw;
    S = make_float3(center.x * cw, center.y * cw, center.z * cw);
    V = center.w * cw * cw;
    int t = 0;
#pragma unroll
    for (int dy = -1; dy <= 1; dy++) {
#pragma unroll
      for (int dx = -1; dx <= 1; dx++) {
        if (dx == 0 && dy == 0) continue;
        const float hh = (dx == 0 ? 0.5f : 0.25f) * (dy == 0 ? 0.5f : 0.25f);
        const int off = dy * STEP * SW + dx * STEP;
        const float4 gq = sG[ti + off];
        const int tx = qx + dx * STEP, ty = qy + dy * STEP;
        ok[t] = tx >= 0 && ty >= 0 && tx < w && ty < h && gq.w >= 0.0f;
        wq[t] = 0.0f;
        lq[t] = 0.0f;
        if (ok[t]) {
          const float4 cq = sA[ti + off];
          lq[t] = lum(cq);
          const float iz = (dx == 0 || dy == 0) ? iz1 : iz2;
          wq[t] = hh * pow128(fmaxf(dot3(gq, gp), 0.0f)) * expf(-fabsf(gq.w - gp.w) * iz - sl * fabsf(lq[t] - lc));
          W += wq[t];
          S.x += wq[t] * cq.x; S.y += wq[t] * cq.y; S.z += wq[t] * cq.z;
          V += wq[t] * wq[t] * cq.w;
        }
        t++;
      }
    }
  }
  HD_INL float4 out() const { return make_float4(S.x / W, S.y / W, S.z / W, V / (W * W)); }

  // Adjoint for output gradient (g_rgb, g_v): parameter gradients ds, dc and, if dIn != nullptr, the input-level
  // gradient scattered to the taps (image index of the tile centre pix, tap offsets STEP on a row pitch of `pitch`).
  HD_INL void adjoint(const float4 *sA, int ti, float3 g, float g_v, float s, float &ds, float &dc, float4 *dIn,
                      int pix, int pitch, float *dgv_out = nullptr) const {
    const float o_r = S.x / W, o_g = S.y / W, o_b = S.z / W, ov = V / (W * W);
    const float3 gS = make_float3(g.x / W, g.y / W, g.z / W);
    const float gV = g_v / (W * W);
    const float gW = -(g.x * o_r + g.y * o_g + g.z * o_b) / W - 2.0f * g_v * ov / W;
    const float dcw = gS.x * center.x + gS.y * center.y + gS.z * center.z + gV * 2.0f * cw * center.w + gW;
    dc = dcw * 0.25f;
    float dsl = 0.0f, dlp = 0.0f;
    int t = 0;
#pragma unroll
    for (int dy = -1; dy <= 1; dy++) {
#pragma unroll
      for (int dx = -1; dx <= 1; dx++) {
        if (dx == 0 && dy == 0) continue;
        if (ok[t]) {
          const float4 cq = sA[ti + dy * STEP * SW + dx * STEP];
          const float dw = gS.x * cq.x + gS.y * cq.y + gS.z * cq.z + gV * 2.0f * wq[t] * cq.w + gW;
          const float de = dw * wq[t];
          const float sg = sgn(lq[t] - lc);
          dsl += de * (-fabsf(lq[t] - lc));
          dlp += de * sl * sg;
          if (dIn) {
            const float dlq = -de * sl * sg;
            atomic_add4(dIn + pix + dy * STEP * pitch + dx * STEP,
                        make_float4(gS.x * wq[t] + dlq * 0.2126f, gS.y * wq[t] + dlq * 0.7152f,
                                    gS.z * wq[t] + dlq * 0.0722f, gV * wq[t] * wq[t]));
          }
        }
        t++;
      }
    }
    ds = dsl / den;
    const float dgv = gv > 1e-12f ? dsl * (-s / (den * den)) * (0.5f / sqrtf(gv)) : 0.0f;
    if (dgv_out) *dgv_out = dgv;  // with the prefilter, the caller spreads it over the 3x3 variances
    if (dIn) {
      // centre: direct terms, luminance through every tap's weight, variance through sl (no prefilter here)
      atomic_add4(dIn + pix, make_float4(gS.x * cw + dlp * 0.2126f, gS.y * cw + dlp * 0.7152f, gS.z * cw + dlp * 0.0722f,
                                         gV * cw * cw + (PREF ? 0.0f : dgv)));
    }
  }
};

// Mid level k (1, 2, 3): B_k = filt(src; s_k, c_k). Level 1 reads the block means from F2.zw (with prefilter).
template <int K>
__global__ void __launch_bounds__(TW *TH) k_mid_fwd(const TwinFrame T) {
  constexpr int STEP = K == 1 ? 1 : (K == 2 ? 2 : 4), AP = STEP, SW = TW + 2 * AP, SH = TH + 2 * AP;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const HushFrame &f = T.f;
  const float4 *src = K == 2 ? T.B1 : T.B2;
  float4 *dst = K == 1 ? T.B1 : (K == 2 ? T.B2 : T.B3);
  const int li = threadIdx.y * TW + threadIdx.x;
  const int bx = blockIdx.x * TW, by = blockIdx.y * TH;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const int q = clampi(by - AP + i / SW, 0, f.H2 - 1) * f.W2 + clampi(bx - AP + i % SW, 0, f.W2 - 1);
    sA[i] = K == 1 ? f2_ac_tw(f.F2, q) : src[q];
    sG[i] = f3_guide_tw(f.F3, q);
  }
  __syncthreads();
  const int X = bx + threadIdx.x, Y = by + threadIdx.y;
  if (X >= f.W2 || Y >= f.H2) return;
  const int o = Y * f.W2 + X, ti = (threadIdx.y + AP) * SW + threadIdx.x + AP;
  if (T.zero_adj) (K == 1 ? T.dB1 : (K == 2 ? T.dB2 : T.dB3))[o] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (sG[ti].w < 0.0f) { dst[o] = make_float4(0.f, 0.f, 0.f, 0.f); return; }
  const float4 p1 = T.par[3 * o + 1], p2 = T.par[3 * o + 2];
  const float s = K == 1 ? p1.y : (K == 2 ? p1.z : p1.w), c = K == 1 ? p2.y : (K == 2 ? p2.z : p2.w);
  Filt1<STEP, K == 1, SW> F;
  F.run(sA, sG, ti, X, Y, f.W2, f.H2, s, c);
  dst[o] = F.out();
}

template <int K>
__global__ void __launch_bounds__(TW *TH) k_mid_bwd(const TwinFrame T) {
  constexpr int STEP = K == 1 ? 1 : (K == 2 ? 2 : 4), AP = STEP, SW = TW + 2 * AP, SH = TH + 2 * AP;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const HushFrame &f = T.f;
  const float4 *src = K == 2 ? T.B1 : T.B2;
  const float4 *gout = K == 1 ? T.dB1 : (K == 2 ? T.dB2 : T.dB3);
  float4 *gin = K == 1 ? T.dAh : (K == 2 ? T.dB1 : T.dB2);  // level 1 reads the block means
  const int li = threadIdx.y * TW + threadIdx.x;
  const int bx = blockIdx.x * TW, by = blockIdx.y * TH;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const int q = clampi(by - AP + i / SW, 0, f.H2 - 1) * f.W2 + clampi(bx - AP + i % SW, 0, f.W2 - 1);
    sA[i] = K == 1 ? f2_ac_tw(f.F2, q) : src[q];
    sG[i] = f3_guide_tw(f.F3, q);
  }
  __syncthreads();
  const int X = bx + threadIdx.x, Y = by + threadIdx.y;
  if (X >= f.W2 || Y >= f.H2) return;
  const int o = Y * f.W2 + X, ti = (threadIdx.y + AP) * SW + threadIdx.x + AP;
  if (sG[ti].w < 0.0f) return;
  const float4 p1 = T.par[3 * o + 1], p2 = T.par[3 * o + 2];
  const float s = K == 1 ? p1.y : (K == 2 ? p1.z : p1.w), c = K == 1 ? p2.y : (K == 2 ? p2.z : p2.w);
  Filt1<STEP, K == 1, SW> F;
  F.run(sA, sG, ti, X, Y, f.W2, f.H2, s, c);
  const float4 g = gout[o];
  float ds, dc, dgv = 0.0f;
  F.adjoint(sA, ti, make_float3(g.x, g.y, g.z), g.w, s, ds, dc, gin, o, f.W2, K == 1 ? &dgv : nullptr);
  if (K == 1 && gin && dgv != 0.0f) {  // level 1's 3x3 variance prefilter (clamp-to-edge taps)
#pragma unroll
    for (int j = 0; j < 9; j++) {
      const int dx = j % 3 - 1, dy = j / 3 - 1;
      const float k = (dx == 0 && dy == 0) ? 0.25f : ((dx == 0 || dy == 0) ? 0.125f : 0.0625f);
      atomicAdd(&gin[clampi(Y + dy, 0, f.H2 - 1) * f.W2 + clampi(X + dx, 0, f.W2 - 1)].w, k * dgv);
    }
  }
  // s_k / c_k live in components k of par1 / par2
  float *dp1 = &T.dpar[3 * o + 1].x, *dp2 = &T.dpar[3 * o + 2].x;
  atomicAdd(dp1 + K, ds);
  atomicAdd(dp2 + K, dc);
}

// ------------------------------------------------------------------------------------------------ coarse levels
// COARSE1 (hush.js:372-421: down() of the half-res block means, then the 5x5 a-trous with step 1) and coarse2
// (hush.js:752: the 5x5 a-trous with step 2), both with the variance prefilter, s = COARSE_S and c = 1, in FP32
// without the f16 storage rounding. Their only differentiable input is the colour + variance level they filter (the
// guide is geometry), so each adjoint takes dL/d(output level) to dL/d(input level): the direct taps, the luminance
// edge-stopping terms of every tap and of the centre, and the prefiltered variance through s / sd.
template <int STEP, int SW>
struct Filt2 {
  static constexpr int NT = 24;
  float4 gp, center;
  float gv, lc, den, sl, cw, W;
  float wq[NT], lq[NT];
  bool ok[NT];
  float3 S;
  float V;
  HD_INL static float hw(int d) { return d == 0 ? 0.375f : (d == 1 || d == -1) ? 0.25f : 0.0625f; }
  HD_INL static int dx_of(int t) { const int k = t < NT / 2 ? t : t + 1; return k % 5 - 2; }
  HD_INL static int dy_of(int t) { const int k = t < NT / 2 ? t : t + 1; return k / 5 - 2; }
  HD_INL void run(const float4 *sA, const float4 *sG, int ti, int qx, int qy, int w, int h, float s, float c) {
    gp = sG[ti];
    center = sA[ti];
    gv = 0.0625f * (sA[ti - SW - 1].w + sA[ti - SW + 1].w + sA[ti + SW - 1].w + sA[ti + SW + 1].w) +
         0.125f * (sA[ti - SW].w + sA[ti - 1].w + sA[ti + 1].w + sA[ti + SW].w) + 0.25f * center.w;
    lc = lum(center);
    den = sqrtf(fmaxf(gv, 1e-12f)) + 1e-6f;
    sl = s / den;
    const float zl = sG[ti - 1].w, zr = sG[ti + 1].w, zu = sG[ti - SW].w, zd = sG[ti + SW].w;
    const float gx = fminf(zr > 0.0f ? fabsf(zr - gp.w) : 1e9f, zl > 0.0f ? fabsf(zl - gp.w) : 1e9f);
    const float gy = fminf(zd > 0.0f ? fabsf(zd - gp.w) : 1e9f, zu > 0.0f ? fabsf(zu - gp.w) : 1e9f);
    const float zg = fminf(fmaxf(gx, gy), gp.w);
    cw = (0.375f * 0.375f) * c;
    W = cw;
    S = make_float3(center.x * cw, center.y * cw, center.z * cw);
    V = center.w * cw * cw;
#pragma unroll
    for (int t = 0; t < NT; t++) {
      const int dx = dx_of(t), dy = dy_of(t);
      const int off = dy * STEP * SW + dx * STEP;
      const float4 gq = sG[ti + off];
      const int tx = qx + dx * STEP, ty = qy + dy * STEP;
      ok[t] = tx >= 0 && ty >= 0 && tx < w && ty < h && gq.w >= 0.0f;
      wq[t] = 0.0f;
      lq[t] = 0.0f;
      if (ok[t]) {
        const float4 cq = sA[ti + off];
        lq[t] = lum(cq);
        const float iz = 1.0f / (zg * (sqrtf((float)(dx * dx + dy * dy)) * STEP) + 1e-3f);
        wq[t] = hw(dx) * hw(dy) * pow128(fmaxf(dot3(gq, gp), 0.0f)) *
                expf(-fabsf(gq.w - gp.w) * iz - sl * fabsf(lq[t] - lc));
        W += wq[t];
        S.x += wq[t] * cq.x; S.y += wq[t] * cq.y; S.z += wq[t] * cq.z;
        V += wq[t] * wq[t] * cq.w;
      }
    }
  }
  HD_INL float4 out() const { return make_float4(S.x / W, S.y / W, S.z / W, V / (W * W)); }

  // Adjoint for the output gradient (g_rgb, g_v), added into dIn (image of row pitch `pitch`, size w x h): every
  // tap at its image position; the centre and its 3x3 prefilter neighbours at their clamp-to-edge positions (qx, qy)
  // is the centre's image position.
  HD_INL void adjoint(const float4 *sA, int ti, float3 g, float g_v, float s, float4 *dIn, int qx, int qy, int w,
                      int h) const {
    const float o_r = S.x / W, o_g = S.y / W, o_b = S.z / W, ov = V / (W * W);
    const float3 gS = make_float3(g.x / W, g.y / W, g.z / W);
    const float gV = g_v / (W * W);
    const float gW = -(g.x * o_r + g.y * o_g + g.z * o_b) / W - 2.0f * g_v * ov / W;
    float dsl = 0.0f, dlp = 0.0f;
#pragma unroll
    for (int t = 0; t < NT; t++) {
      if (!ok[t]) continue;
      const int dx = dx_of(t), dy = dy_of(t);
      const float4 cq = sA[ti + dy * STEP * SW + dx * STEP];
      const float dw = gS.x * cq.x + gS.y * cq.y + gS.z * cq.z + gV * 2.0f * wq[t] * cq.w + gW;
      const float de = dw * wq[t];
      const float sg = sgn(lq[t] - lc);
      dsl += de * (-fabsf(lq[t] - lc));
      dlp += de * sl * sg;
      const float dlq = -de * sl * sg;
      atomic_add4(dIn + (qy + dy * STEP) * w + qx + dx * STEP,
                  make_float4(gS.x * wq[t] + dlq * 0.2126f, gS.y * wq[t] + dlq * 0.7152f, gS.z * wq[t] + dlq * 0.0722f,
                              gV * wq[t] * wq[t]));
    }
    const float dgv = gv > 1e-12f ? dsl * (-s / (den * den)) * (0.5f / sqrtf(gv)) : 0.0f;
#pragma unroll
    for (int dy = -1; dy <= 1; dy++) {
#pragma unroll
      for (int dx = -1; dx <= 1; dx++) {
        const float k = (dx == 0 && dy == 0) ? 0.25f : (dx == 0 || dy == 0) ? 0.125f : 0.0625f;
        const int o = clampi(qy + dy, 0, h - 1) * w + clampi(qx + dx, 0, w - 1);
        if (dx == 0 && dy == 0)
          atomic_add4(dIn + o, make_float4(gS.x * cw + dlp * 0.2126f, gS.y * cw + dlp * 0.7152f,
                                           gS.z * cw + dlp * 0.0722f, gV * cw * cw + k * dgv));
        else
          atomicAdd(&dIn[o].w, k * dgv);
      }
    }
  }
};

// down() (hush.js:385-402) of the twin's FP32 block means ah at quarter-res texel Q, without the f16 rounding; the
// weights are the blocks' pixel counts (F3), N their sum (0: the texel has no surface and holds zeros).
HD_INL float4 down_tw(const HushFrame &f, const float4 *ah, int Qx, int Qy, float *Nout) {
  float N = 0.f, vr = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int hx = Qx * 2 + (j & 1), hy = Qy * 2 + (j >> 1);
    if (hx >= f.W2 || hy >= f.H2) continue;
    const float w = unpack2(__ldg(f.F3 + hy * f.W2 + hx).y).y;
    if (w <= 0.0f) continue;
    const float4 a = ah[hy * f.W2 + hx];
    N += w;
    cx += w * a.x; cy += w * a.y; cz += w * a.z;
    vr += w * a.w;
  }
  if (Nout) *Nout = N;
  if (N == 0.0f) return make_float4(0.f, 0.f, 0.f, 0.f);
  return make_float4(cx / N, cy / N, cz / N, vr / N / N);
}

// ah = the block means F2.zw as FP32 (COARSE1's input level in the per-pass pair)
__global__ void k_ah_fill(const TwinFrame T, float4 *ah) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o < T.f.W2 * T.f.H2) ah[o] = f2_ac_tw(T.f.F2, o);
}

// LEVEL 1: src = down(ah), output c1; LEVEL 2: src = c1, output c0. The guide is the stored coarse guide CG.
template <int LEVEL>
__global__ void __launch_bounds__(TW *TH) k_coarse_tw(const TwinFrame T, const float4 *src, float4 *dst,
                                                        const float4 *gout, float4 *gin) {
  constexpr int STEP = LEVEL, AP = 2 * STEP, SW = TW + 2 * AP, SH = TH + 2 * AP;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const HushFrame &f = T.f;
  const int li = threadIdx.y * TW + threadIdx.x;
  const int bx = blockIdx.x * TW, by = blockIdx.y * TH;
  for (int i = li; i < SW * SH; i += TW * TH) {
    const int qx = clampi(bx - AP + i % SW, 0, f.W4 - 1), qy = clampi(by - AP + i / SW, 0, f.H4 - 1);
    const int q = qy * f.W4 + qx;
    sA[i] = LEVEL == 1 ? down_tw(f, src, qx, qy, nullptr) : src[q];
    float4 g = ldh(f.CG, q);
    float4 n = oct_dec(g.x, g.y);
    n.w = g.z;
    sG[i] = n;
  }
  __syncthreads();
  const int X = bx + threadIdx.x, Y = by + threadIdx.y;
  if (X >= f.W4 || Y >= f.H4) return;
  const int o = Y * f.W4 + X, ti = (threadIdx.y + AP) * SW + threadIdx.x + AP;
  if (sG[ti].w < 0.0f) {  // no surface: the level holds zeros (and passes no gradient)
    if (!gout) dst[o] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  Filt2<STEP, SW> F;
  F.run(sA, sG, ti, X, Y, f.W4, f.H4, COARSE_S, 1.0f);
  if (!gout) {
    dst[o] = F.out();
    return;
  }
  const float4 g = gout[o];
  F.adjoint(sA, ti, make_float3(g.x, g.y, g.z), g.w, COARSE_S, gin, X, Y, f.W4, f.H4);
}

// down()'s adjoint: dah (half-res) += the gradient of its quarter-res texel spread over the blocks by their weights
// (colour: w / N; variance: w / N^2). A gather: every half-res texel reads its one quarter-res texel.
__global__ void k_down_bwd(const TwinFrame T, const float4 *ah, const float4 *ddown, float4 *dah) {
  const HushFrame &f = T.f;
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= f.W2 * f.H2) return;
  const int hx = o % f.W2, hy = o / f.W2;
  const float w = unpack2(__ldg(f.F3 + o).y).y;
  if (w <= 0.0f) return;
  float N = 0.0f;
  down_tw(f, ah, hx >> 1, hy >> 1, &N);
  const float4 g = ddown[(hy >> 1) * f.W4 + (hx >> 1)];
  const float k = w / N;
  float4 d = dah[o];
  d.x += g.x * k; d.y += g.y * k; d.z += g.z * k;
  d.w += g.w * k / N;
  dah[o] = d;
}

// c1 = the stored coarse level C1 as FP32 (coarse2's input in the window sweep, straight through the f16 storage)
__global__ void k_c1_fill(const TwinFrame T, float4 *c1) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o < T.f.W4 * T.f.H4) c1[o] = ldh(T.f.C1, o);
}

// The block means' adjoint into TEMPORAL's output: block() forms Ah as the mean of the f16-quantised A0 over the
// block's surface pixels (hush.js:241-244, 280), so every surface pixel gets dL/dAh / nv (the quantisation counts as
// the identity).
__global__ void k_ah_to_a0(const TwinFrame T, const float4 *dah, float4 *dA0) {
  const HushFrame &f = T.f;
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= f.W * f.H) return;
  const int px = o % f.W, py = o / f.W;
  if (ldh(f.key, o).z < 0.0f) return;  // sky: not in the block's mean
  const int hp = (py >> 1) * f.W2 + (px >> 1);
  const float nv = unpack2(__ldg(f.F3 + hp).y).y;
  if (nv <= 0.0f) return;
  const float4 g = dah[hp];
  const float k = 1.0f / nv;
  float4 d = dA0[o];
  d.x += g.x * k; d.y += g.y * k; d.z += g.z * k; d.w += g.w * k;
  dA0[o] = d;
}

// ------------------------------------------------------------------------------------------------ fine + final
struct Recomb {
  float fx, fy, fz, swh, swq, uBx, uBy, uBz, uAx, uAy, uAz, uCx, uCy, uCz;
  float wh[4], wqq[4];
  int qh[4];
  bool vh[4], vq[4];
};

HD_INL void recomb_fwd(const TwinFrame &T, int px, int py, float4 A1, float4 gp, Recomb &R) {
  const HushFrame &f = T.f;
  R.fx = A1.x; R.fy = A1.y; R.fz = A1.z;
  const float z = gp.w;
  const int hsx = (f.W + 1) / 2, hsy = (f.H + 1) / 2;
  const float hposx = ((float)px + 0.5f) / 2.0f - 0.5f, hposy = ((float)py + 0.5f) / 2.0f - 0.5f;
  const float hbx = floorf(hposx), hby = floorf(hposy);
  R.uBx = R.uBy = R.uBz = R.uAx = R.uAy = R.uAz = R.swh = 0.f;
  for (int j = 0; j < 4; j++) {
    const int qx = (int)hbx + (j & 1), qy = (int)hby + (j >> 1);
    R.vh[j] = false;
    R.wh[j] = 0.f;
    R.qh[j] = 0;
    if (qx < 0 || qy < 0 || qx >= hsx || qy >= hsy) continue;
    const int q = qy * f.W2 + qx;
    const float4 g = f3_guide_tw(f.F3, q);
    if (g.w < 0.0f) continue;
    const float w = jbw(hposx - hbx, hposy - hby, j, g, g.w, gp, z);
    const float4 a = f2_ac_tw(f.F2, q), m = T.B3[q];
    R.vh[j] = true;
    R.wh[j] = w;
    R.qh[j] = q;
    R.swh += w;
    R.uBx += w * m.x; R.uBy += w * m.y; R.uBz += w * m.z;
    R.uAx += w * a.x; R.uAy += w * a.y; R.uAz += w * a.z;
  }
  const int qsx = (f.W + 3) / 4, qsy = (f.H + 3) / 4;
  const float cposx = ((float)px + 0.5f) / 4.0f - 0.5f, cposy = ((float)py + 0.5f) / 4.0f - 0.5f;
  const float cbx = floorf(cposx), cby = floorf(cposy);
  R.uCx = R.uCy = R.uCz = R.swq = 0.f;
  for (int j = 0; j < 4; j++) {
    const int qx = (int)cbx + (j & 1), qy = (int)cby + (j >> 1);
    if (qx < 0 || qy < 0 || qx >= qsx || qy >= qsy) continue;
    const int q = qy * f.W4 + qx;
    const float4 cg = ldh(f.CG, q);
    if (cg.z < 0.0f) continue;
    const float w = jbw(cposx - cbx, cposy - cby, j, oct_dec(cg.x, cg.y), cg.z, gp, z);
    const float4 c = ldh(f.C0, q);
    R.swq += w;
    R.uCx += w * c.x; R.uCy += w * c.y; R.uCz += w * c.z;
  }
}

// fine level (A1, also the colour history) and recombination -> X
__global__ void __launch_bounds__(TW *TH) k_fine_fwd(const TwinFrame T) {
  constexpr int AP = 1, SW = TW + 2, SH = TH + 2;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const HushFrame &f = T.f;
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
  const int o = py * f.W + px, ti = (threadIdx.y + AP) * SW + threadIdx.x + AP;
  const float4 alb = ldh(f.mat, py * f.p_mat + px), emi = ldh(f.emi, py * f.p_emi + px);
  const float4 gp = sG[ti];
  if (gp.w < 0.0f) {
    T.A1[o] = make_float4(0.f, 0.f, 0.f, 0.f);
    T.X[o] = make_float4(emi.x, emi.y, emi.z, 0.f);
    sth(f.hist, o, make_float4(0.f, 0.f, 0.f, 0.f));
    return;
  }
  const int hp = (py >> 1) * f.W2 + (px >> 1);
  const float4 p0 = T.par[3 * hp], p1 = T.par[3 * hp + 1], p2 = T.par[3 * hp + 2];
  Filt1<1, true, SW> F;
  F.run(sA, sG, ti, px, py, f.W, f.H, p1.x, p2.x);
  const float4 A1 = F.out();
  T.A1[o] = A1;
  sth(f.hist, o, A1);
  Recomb R;
  recomb_fwd(T, px, py, A1, gp, R);
  float ix = R.fx, iy = R.fy, iz = R.fz;
  if (R.swh > 1e-4f) {
    ix = R.uBx / R.swh + p0.w * (R.fx - R.uAx / R.swh);
    iy = R.uBy / R.swh + p0.w * (R.fy - R.uAy / R.swh);
    iz = R.uBz / R.swh + p0.w * (R.fz - R.uAz / R.swh);
  }
  float upx = ix, upy = iy, upz = iz;
  if (R.swq > 1e-4f) { upx = R.uCx / R.swq; upy = R.uCy / R.swq; upz = R.uCz / R.swq; }
  ix = ix + (upx - ix) * p0.z;
  iy = iy + (upy - iy) * p0.z;
  iz = iz + (upz - iz) * p0.z;
  T.X[o] = make_float4(ix * alb.x + emi.x, iy * alb.y + emi.y, iz * alb.z + emi.z, 0.0f);
}

// ------------------------------------------------------------------------------------------------ TAA
HD_INL float3 tm3(float4 c) { return tmap(make_float3(c.x, c.y, c.z)); }

struct TaaF {
  float3 y[9], m1, sd, v3, cur, hh0, hh, hr, res, out;
  int q[9];
  bool inside, lo_act[3], hi_act[3], act_itm;
  float d;
};

HD_INL void taa_fwd(const TwinFrame &T, int px, int py, TaaF &A) {
  const HushFrame &f = T.f;
  const int o = py * f.W + px;
  A.cur = tm3(T.X[o]);
  A.inside = false;
  for (int j = 0; j < 9; j++) {
    A.q[j] = clampi(py + j / 3 - 1, 0, f.H - 1) * f.W + clampi(px + j % 3 - 1, 0, f.W - 1);
    A.y[j] = to_ycocg(tm3(T.X[A.q[j]]));
  }
  A.res = A.cur;
  for (int c = 0; c < 3; c++) A.lo_act[c] = A.hi_act[c] = false;
  if (!f.reset) {
    float3 m1 = make_float3(0.f, 0.f, 0.f);
    for (int j = 0; j < 9; j++) { m1.x += A.y[j].x; m1.y += A.y[j].y; m1.z += A.y[j].z; }
    m1.x /= 9.0f; m1.y /= 9.0f; m1.z /= 9.0f;
    float3 v3 = make_float3(0.f, 0.f, 0.f);
    for (int j = 0; j < 9; j++) {
      const float dx = A.y[j].x - m1.x, dy = A.y[j].y - m1.y, dz = A.y[j].z - m1.z;
      v3.x += dx * dx; v3.y += dy * dy; v3.z += dz * dz;
    }
    v3.x /= 9.0f; v3.y /= 9.0f; v3.z /= 9.0f;
    A.m1 = m1;
    A.v3 = v3;
    A.sd = make_float3(sqrtf(fmaxf(v3.x, 1e-12f)), sqrtf(fmaxf(v3.y, 1e-12f)), sqrtf(fmaxf(v3.z, 1e-12f)));
    const float4 mv = ldh(f.mv, py * f.p_mv + px);
    const float szx = (float)f.W, szy = (float)f.H;
    const float uvx = ((float)px + 0.5f + mv.x) / szx, uvy = ((float)py + 0.5f + mv.y) / szy;
    if (uvx >= 0.0f && uvy >= 0.0f && uvx <= 1.0f && uvy <= 1.0f) {
      A.inside = true;
      const float ppx = uvx * szx - 0.5f, ppy = uvy * szy - 0.5f;
      const float bxf = floorf(ppx), byf = floorf(ppy);
      const float fx = ppx - bxf, fy = ppy - byf;
      float3 hist = make_float3(0.f, 0.f, 0.f);
      for (int j = 0; j < 4; j++) {
        const int ox = j & 1, oy = j >> 1;
        const float wb = (ox == 1 ? fx : 1.0f - fx) * (oy == 1 ? fy : 1.0f - fy);
        const float4 t = ldh(f.taa_prev, clampi((int)byf + oy, 0, f.H - 1) * f.W + clampi((int)bxf + ox, 0, f.W - 1));
        hist.x += wb * t.x; hist.y += wb * t.y; hist.z += wb * t.z;
      }
      A.hh0 = to_ycocg(tmap(hist));
      float h0[3] = {A.hh0.x, A.hh0.y, A.hh0.z}, mm[3] = {m1.x, m1.y, m1.z}, ss[3] = {A.sd.x, A.sd.y, A.sd.z}, hc[3];
      for (int c = 0; c < 3; c++) {
        const float lo = mm[c] - 1.25f * ss[c], hi = mm[c] + 1.25f * ss[c];
        const float mx = fmaxf(h0[c], lo);
        A.lo_act[c] = h0[c] < lo;
        hc[c] = fminf(mx, hi);
        A.hi_act[c] = mx > hi;
      }
      A.hh = make_float3(hc[0], hc[1], hc[2]);
      A.hr = from_ycocg(A.hh);
      A.res = make_float3(A.hr.x + (A.cur.x - A.hr.x) * 0.1f, A.hr.y + (A.cur.y - A.hr.y) * 0.1f,
                          A.hr.z + (A.cur.z - A.hr.z) * 0.1f);
    }
  }
  const float l = lum3(A.res.x, A.res.y, A.res.z);
  A.act_itm = 1.0f - l > 1e-4f;
  A.d = fmaxf(1.0f - l, 1e-4f);
  A.out = make_float3(A.res.x / A.d, A.res.y / A.d, A.res.z / A.d);
}

__global__ void k_taa_fwd(const TwinFrame T) {
  const HushFrame &f = T.f;
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= f.W || py >= f.H) return;
  TaaF A;
  taa_fwd(T, px, py, A);
  const int o = py * f.W + px;
  T.out[o] = make_float4(A.out.x, A.out.y, A.out.z, 1.0f);
  sth(f.taa, o, make_float4(A.out.x, A.out.y, A.out.z, 1.0f));
}

// ------------------------------------------------------------------------------------------------ loss
// L = (1 / 3N) sum min(|out - clean| / (|clean| + 1e-2), 1) + lambda (1 / 3N) sum min(|d out - d clean| /
// (|clean| + 1e-2), 1), d = difference to the previous frame. The clip at 1 keeps the TAA's itm singularity (outputs
// up to 1e4 where the clipped history reaches luminance 1, hush.js:636) from dominating the gradient. Writes dL/dout (into gT, as the seed of the TAA adjoint) and per-CTA FP64
// partial sums.
__global__ void k_loss(const TwinFrame T, int backward) {
  const HushFrame &f = T.f;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (i < f.W * f.H) {
    const float4 o = T.out[i];
    const float ov[3] = {o.x, o.y, o.z};
    float g[3] = {0.f, 0.f, 0.f};
    for (int c = 0; c < 3; c++) {
      const float cl = T.clean[3 * i + c], den = fabsf(cl) + 1e-2f;
      const float d = ov[c] - cl;
      const double e = fabs((double)d) / den;
      l += e < 1.0 ? e : 1.0;
      g[c] = e < 1.0 ? sgn(d) / den : 0.0f;
      if (T.has_prev) {
        const float4 op = T.out_prev[i];
        const float opv[3] = {op.x, op.y, op.z};
        const float dd = (ov[c] - opv[c]) - (cl - T.clean_prev[3 * i + c]);
        const double et = fabs((double)dd) / den;
        l += (double)T.lambda_t * (et < 1.0 ? et : 1.0);
        g[c] += et < 1.0 ? T.lambda_t * sgn(dd) / den : 0.0f;
      }
    }
    l *= T.inv_n;
    if (backward) T.gT[i] = make_float4(g[0] * T.inv_n, g[1] * T.inv_n, g[2] * T.inv_n, 0.f);
  }
  // block reduction in FP64
  for (int off = 16; off > 0; off >>= 1) l += __shfl_down_sync(0xffffffffu, l, off);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (threadIdx.x == 0) T.loss_partials[blockIdx.x] = v;
  }
}

__global__ void k_reduce_f64(const double *partials, int n, double *out, double *acc) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partials[i];
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double u = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) u += __shfl_down_sync(0xffffffffu, u, off);
    if (threadIdx.x == 0) {
      *out = u;
      if (acc) *acc += u;
    }
  }
}

// ------------------------------------------------------------------------------------------------ TAA adjoint
// In two gathers, without atomics. Pass 1 (per pixel p): from dL/dout to the per-pixel coefficients of the clip box's
// adjoint, dL/d(window mean) gm and dL/d(window variance) gs per YCoCg channel, with the window mean m1, and the
// gradient of the current colour tm(X_p) itself. Pass 2 (per pixel q): dL/d tm(X_q) as that own term plus, for every
// pixel p whose clamped 3 x 3 window holds q (with the window's multiplicity at the image border), the YCoCg-adjoint
// of gm_p / 9 + gs_p 2 (y_q - m1_p) / 9.
HD_INL float3 itm_adjoint(const TaaF &A, float3 g) {
  const float inv = 1.0f / A.d;
  float3 r = make_float3(g.x * inv, g.y * inv, g.z * inv);
  if (A.act_itm) {
    const float k = (g.x * A.res.x + g.y * A.res.y + g.z * A.res.z) * inv * inv;
    r.x += k * 0.2126f; r.y += k * 0.7152f; r.z += k * 0.0722f;
  }
  return r;
}
// adjoint of tm(X) = X / (1 + lum(X)) at X
HD_INL float3 tm_adjoint(float4 Xv, float4 gt) {
  const float L1 = 1.0f + lum(Xv);
  const float k = (gt.x * Xv.x + gt.y * Xv.y + gt.z * Xv.z) / (L1 * L1);
  return make_float3(gt.x / L1 - k * 0.2126f, gt.y / L1 - k * 0.7152f, gt.z / L1 - k * 0.0722f);
}
HD_INL float3 ycocg_adjoint(float3 g) {  // transpose of to_ycocg
  return make_float3(0.25f * g.x + 0.5f * g.y - 0.25f * g.z, 0.5f * g.x + 0.5f * g.z, 0.25f * g.x - 0.5f * g.y - 0.25f * g.z);
}

// coef[3p .. 3p + 2] = (gm, gcur.x), (gs, gcur.y), (m1, gcur.z)
__global__ void k_taa_bwd_coef(const TwinFrame T, const float4 *gout, float4 *coef) {
  const HushFrame &f = T.f;
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= f.W || py >= f.H) return;
  const int o = py * f.W + px;
  TaaF A;
  taa_fwd(T, px, py, A);
  const float4 go = gout[o];
  const float3 gres = itm_adjoint(A, make_float3(go.x, go.y, go.z));
  float3 gcur = gres;
  float gm[3] = {0.f, 0.f, 0.f}, gs[3] = {0.f, 0.f, 0.f};
  if (A.inside) {
    gcur = make_float3(0.1f * gres.x, 0.1f * gres.y, 0.1f * gres.z);
    const float3 ghr = make_float3(0.9f * gres.x, 0.9f * gres.y, 0.9f * gres.z);
    // from_ycocg transpose
    const float gh[3] = {ghr.x + ghr.y + ghr.z, ghr.x - ghr.z, -ghr.x + ghr.y - ghr.z};
    const float v3[3] = {A.v3.x, A.v3.y, A.v3.z}, sd[3] = {A.sd.x, A.sd.y, A.sd.z};
    for (int c = 0; c < 3; c++) {
      const float glo = A.lo_act[c] ? gh[c] : 0.0f, ghi = A.hi_act[c] ? gh[c] : 0.0f;
      gm[c] = glo + ghi;
      gs[c] = 1.25f * (ghi - glo);
      gs[c] = v3[c] > 1e-12f ? gs[c] / (2.0f * sd[c]) : 0.0f;  // d sd / d v3
    }
  }
  coef[3 * o] = make_float4(gm[0], gm[1], gm[2], gcur.x);
  coef[3 * o + 1] = make_float4(gs[0], gs[1], gs[2], gcur.y);
  coef[3 * o + 2] = make_float4(A.m1.x, A.m1.y, A.m1.z, gcur.z);
}

// how many of the clamped offsets p + d (d = -1, 0, 1) land on q
HD_INL int window_hits(int p, int q, int n) {
  return (clampi(p - 1, 0, n - 1) == q) + (p == q) + (clampi(p + 1, 0, n - 1) == q);
}

// gT[q] = dL/d tm(X_q) (set, not added)
__global__ void k_taa_bwd_gather(const TwinFrame T, const float4 *coef, float4 *gT) {
  const HushFrame &f = T.f;
  const int qx = blockIdx.x * blockDim.x + threadIdx.x, qy = blockIdx.y * blockDim.y + threadIdx.y;
  if (qx >= f.W || qy >= f.H) return;
  const int o = qy * f.W + qx;
  const float3 y = to_ycocg(tm3(T.X[o]));
  float gx = coef[3 * o].w, gyy = coef[3 * o + 1].w, gz = coef[3 * o + 2].w;
  for (int py = max(qy - 1, 0); py <= min(qy + 1, f.H - 1); py++) {
    const int my = window_hits(py, qy, f.H);
    if (!my) continue;
    for (int px = max(qx - 1, 0); px <= min(qx + 1, f.W - 1); px++) {
      const int m = my * window_hits(px, qx, f.W);
      if (!m) continue;
      const int p = py * f.W + px;
      const float4 a = coef[3 * p], b = coef[3 * p + 1], c = coef[3 * p + 2];
      float3 g;
      g.x = a.x / 9.0f + b.x * 2.0f * (y.x - c.x) / 9.0f;
      g.y = a.y / 9.0f + b.y * 2.0f * (y.y - c.y) / 9.0f;
      g.z = a.z / 9.0f + b.z * 2.0f * (y.z - c.z) / 9.0f;
      const float3 t = ycocg_adjoint(g);
      const float k = (float)m;
      gx += k * t.x; gyy += k * t.y; gz += k * t.z;
    }
  }
  gT[o] = make_float4(gx, gyy, gz, 0.f);
}

// dX += tm adjoint of the tone-mapped-colour gradient at every pixel (the per-pass TAA adjoint's second step; the fused
// frame folds it into k_fine_bwd, where sky pixels need no dX).
__global__ void k_tm_bwd(const TwinFrame T, const float4 *gtm, float4 *dX) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= T.f.W * T.f.H) return;
  const float3 g = tm_adjoint(T.X[o], gtm[o]);
  const float4 d = dX[o];
  dX[o] = make_float4(d.x + g.x, d.y + g.y, d.z + g.z, d.w);
}

// Pass 2 (per full pixel): dL/dX from the tm gradient; then recombination, fine-level parameter and mid-level input
// gradients.
// SEED_TM: the seed is the gradient w.r.t. the tone-mapped colour tm(X) (the fused frame); else w.r.t. X itself (the
// per-pass pair, whose TAA adjoint has already applied the tm adjoint).
// dL/dC0 of the recombination's coarse term (window sweep only): up = sum w C0 / sum w, ill2 = ill + (up - ill) beta,
// so each quarter-res tap's colour gets g2 beta w / sum w (its variance none). The taps' weights are recomputed as
// recomb_fwd() forms them, so the per-frame adjoint keeps no per-tap state.
HD_INL void recomb_coarse_adj(const TwinFrame &T, int px, int py, float4 gp, float swq, float beta, float3 g2) {
  const HushFrame &f = T.f;
  const int qsx = (f.W + 3) / 4, qsy = (f.H + 3) / 4;
  const float cposx = ((float)px + 0.5f) / 4.0f - 0.5f, cposy = ((float)py + 0.5f) / 4.0f - 0.5f;
  const float cbx = floorf(cposx), cby = floorf(cposy);
  for (int j = 0; j < 4; j++) {
    const int qx = (int)cbx + (j & 1), qy = (int)cby + (j >> 1);
    if (qx < 0 || qy < 0 || qx >= qsx || qy >= qsy) continue;
    const int q = qy * f.W4 + qx;
    const float4 cg = ldh(f.CG, q);
    if (cg.z < 0.0f) continue;
    const float k = beta * jbw(cposx - cbx, cposy - cby, j, oct_dec(cg.x, cg.y), cg.z, gp, gp.w) / swq;
    float *d = &T.dC0[q].x;
    atomicAdd(d, g2.x * k);
    atomicAdd(d + 1, g2.y * k);
    atomicAdd(d + 2, g2.z * k);
  }
}

template <bool SEED_TM>
__global__ void __launch_bounds__(TW *TH) k_fine_bwd(const TwinFrame T, const float4 *gT) {
  constexpr int AP = 1, SW = TW + 2, SH = TH + 2;
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  const HushFrame &f = T.f;
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
  const bool in = px < f.W && py < f.H;
  const int hp = (min(py, f.H - 1) >> 1) * f.W2 + (min(px, f.W - 1) >> 1);
  float q4[4] = {0.f, 0.f, 0.f, 0.f};  // this pixel's dL/d(beta, kappa, s0, c0)
  const int ti = (threadIdx.y + AP) * SW + threadIdx.x + AP;
  const float4 gp = sG[ti];
  if (in && gp.w >= 0.0f) {  // sky: X = emission, no dependence on the parameters
    const int o = py * f.W + px;
    const float4 gt = gT[o];
    const float3 gX = SEED_TM ? tm_adjoint(T.X[o], gt) : make_float3(gt.x, gt.y, gt.z);
    const float4 alb = ldh(f.mat, py * f.p_mat + px);
    const float4 p0 = T.par[3 * hp], p1 = T.par[3 * hp + 1], p2 = T.par[3 * hp + 2];
    Filt1<1, true, SW> F;
    F.run(sA, sG, ti, px, py, f.W, f.H, p1.x, p2.x);
    const float4 A1 = F.out();
    Recomb R;
    recomb_fwd(T, px, py, A1, gp, R);
    float ix = R.fx, iy = R.fy, iz = R.fz;
    const bool mid = R.swh > 1e-4f;
    if (mid) {
      ix = R.uBx / R.swh + p0.w * (R.fx - R.uAx / R.swh);
      iy = R.uBy / R.swh + p0.w * (R.fy - R.uAy / R.swh);
      iz = R.uBz / R.swh + p0.w * (R.fz - R.uAz / R.swh);
    }
    // X = ill2 * alb + emi, ill2 = ill + (up - ill) beta
    const float3 g2 = make_float3(gX.x * alb.x, gX.y * alb.y, gX.z * alb.z);
    float3 gill = g2;
    float gbeta = 0.0f;
    if (R.swq > 1e-4f) {
      const float upx = R.uCx / R.swq, upy = R.uCy / R.swq, upz = R.uCz / R.swq;
      gbeta = g2.x * (upx - ix) + g2.y * (upy - iy) + g2.z * (upz - iz);
      gill = make_float3(g2.x * (1.0f - p0.z), g2.y * (1.0f - p0.z), g2.z * (1.0f - p0.z));
    }
    float3 gf = gill;
    float gkappa = 0.0f;
    if (mid) {
      gkappa = gill.x * (R.fx - R.uAx / R.swh) + gill.y * (R.fy - R.uAy / R.swh) + gill.z * (R.fz - R.uAz / R.swh);
      gf = make_float3(gill.x * p0.w, gill.y * p0.w, gill.z * p0.w);
      for (int j = 0; j < 4; j++) {
        if (!R.vh[j]) continue;
        const float w = R.wh[j] / R.swh;
        float *d = &T.dB3[R.qh[j]].x;  // the level's variance gets no gradient from the recombination
        atomicAdd(d, gill.x * w);
        atomicAdd(d + 1, gill.y * w);
        atomicAdd(d + 2, gill.z * w);
      }
    }
    float gv1 = 0.0f;  // the fine level's variance reaches X through nothing; only the history may seed it
    if (T.gA1) {       // the next frame reads this fine level as its colour history
      const float4 h = T.gA1[o];
      gf = make_float3(gf.x + h.x, gf.y + h.y, gf.z + h.z);
      gv1 = h.w;
    }
    float ds, dc, dgv = 0.0f;
    F.adjoint(sA, ti, gf, gv1, p1.x, ds, dc, T.dA0, o, f.W, &dgv);
    if (T.dA0 && dgv != 0.0f) {  // the 3x3 variance prefilter (clamp-to-edge taps): 1/16 corners, 1/8 edges, 1/4 centre
#pragma unroll
      for (int j = 0; j < 9; j++) {
        const int dx = j % 3 - 1, dy = j / 3 - 1;
        const float k = (dx == 0 && dy == 0) ? 0.25f : ((dx == 0 || dy == 0) ? 0.125f : 0.0625f);
        const int q = clampi(py + dy, 0, f.H - 1) * f.W + clampi(px + dx, 0, f.W - 1);
        atomicAdd(&T.dA0[q].w, k * dgv);
      }
    }
    q4[0] = gbeta; q4[1] = gkappa; q4[2] = ds; q4[3] = dc;
  }
  // the 2 x 2 pixels of a half-res block are lanes l, l ^ 1, l ^ 16 and l ^ 17 of one warp (16-pixel rows, even
  // tile origin): their parameter gradients are summed in the warp and added once
#pragma unroll
  for (int k = 0; k < 4; k++) {
    q4[k] += __shfl_xor_sync(0xffffffffu, q4[k], 1);
    q4[k] += __shfl_xor_sync(0xffffffffu, q4[k], 16);
  }
  if (in && !(threadIdx.x & 1) && !(threadIdx.y & 1) && (q4[0] != 0.f || q4[1] != 0.f || q4[2] != 0.f || q4[3] != 0.f)) {
    float *d0 = &T.dpar[3 * hp].x, *d1 = &T.dpar[3 * hp + 1].x, *d2 = &T.dpar[3 * hp + 2].x;
    atomicAdd(d0 + 2, q4[0]);
    atomicAdd(d0 + 3, q4[1]);
    atomicAdd(d1 + 0, q4[2]);
    atomicAdd(d2 + 0, q4[3]);
  }
}

// The recombination's adjoint into the block means and the coarse level (window sweep only; k_fine_bwd does the
// rest): ill = uB / sum_h w + kappa (f - uA / sum_h w) and ill2 = ill + (up - ill) beta, up = sum_q w C0 / sum_q w, so
// each half-res tap's block-mean colour gets -kappa w / sum_h w dL/d ill and each quarter-res tap's colour
// beta w / sum_q w dL/d ill2 (X = ill2 albedo + emission). The tap weights do not depend on the levels, so nothing
// of the fine level is recomputed.
template <bool SEED_TM>
__global__ void __launch_bounds__(TW *TH) k_fine_pyr_bwd(const TwinFrame T, const float4 *gT) {
  const HushFrame &f = T.f;
  const int px = blockIdx.x * TW + threadIdx.x, py = blockIdx.y * TH + threadIdx.y;
  if (px >= f.W || py >= f.H) return;
  const int o = py * f.W + px;
  const float4 key = ldh(f.key, o);
  if (key.z < 0.0f) return;  // sky: X = emission
  float4 gp = oct_dec(key.x, key.y);
  gp.w = key.z;
  const int hp = (py >> 1) * f.W2 + (px >> 1);
  const float4 gt = gT[o];
  const float3 gX = SEED_TM ? tm_adjoint(T.X[o], gt) : make_float3(gt.x, gt.y, gt.z);
  const float4 alb = ldh(f.mat, py * f.p_mat + px), p0 = T.par[3 * hp];
  const float3 g2 = make_float3(gX.x * alb.x, gX.y * alb.y, gX.z * alb.z);
  Recomb R;
  recomb_fwd(T, px, py, make_float4(0.f, 0.f, 0.f, 0.f), gp, R);
  float3 gill = g2;
  if (R.swq > 1e-4f) {
    gill = make_float3(g2.x * (1.0f - p0.z), g2.y * (1.0f - p0.z), g2.z * (1.0f - p0.z));
    recomb_coarse_adj(T, px, py, gp, R.swq, p0.z, g2);
  }
  if (R.swh > 1e-4f) {
    for (int j = 0; j < 4; j++) {
      if (!R.vh[j]) continue;
      const float k = -p0.w * R.wh[j] / R.swh;
      float *a = &T.dAh[R.qh[j]].x;
      atomicAdd(a, gill.x * k);
      atomicAdd(a + 1, gill.y * k);
      atomicAdd(a + 2, gill.z * k);
    }
  }
}

// ------------------------------------------------------------------------------------------------ TEMPORAL adjoint
// Adjoint of TEMPORAL's pixel() (hush.js:111-223) through the two outputs that carry gradient across frames: the
// colour + variance A0 (the fine level's input) and the moments (m1, m2, fast mean, history length) that the next
// frame reprojects. Seeds gA (dL/dA0) and gM (dL/d moments; may be NULL); it ADDS dL/d(previous colour history) into
// dhist, dL/d(previous moments) into dmom and dL/d(previous frame's alpha, gamma) into dag (half-res, per pixel of
// the previous par0). The f16 storage of A0, the moments, the history and par0 counts as the identity (a straight-
// through gradient). The forward is recomputed from the frame's G-buffer and the previous frame's stored history
// with temporal_pixel()'s arithmetic: the 3x3 statistics (no gradient: they depend on this frame's inputs only), the
// bilinear reprojection with its key tests or the 3x3 fallback (the tap weights depend on the motion only, so the
// history enters linearly), the anti-lag clamp mu +- gamma sd (hush.js:195), the blend a = max(alpha, 1 / len)
// (hush.js:196-199), the moment updates (hush.js:200) and the variance lerp (hush.js:206-207). The lag metric and the
// block features are not differentiated: the MLP's inputs are held fixed.
__global__ void __launch_bounds__(TW *TH) k_temporal_bwd(const TwinFrame T, const float4 *gA, const float4 *gM,
                                                         float4 *dhist, float4 *dmom, float2 *dag) {
  constexpr int SW = TW + 2, SH = TH + 2;
  __shared__ float4 sI[SW * SH];
  const HushFrame &f = T.f;
  const int li = threadIdx.y * TW + threadIdx.x;
  const int ox = blockIdx.x * TW - 1, oy = blockIdx.y * TH - 1;
  for (int i = li; i < SW * SH; i += TW * TH) {  // the illumination tile of k_temporal
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
  if (px >= f.W || py >= f.H || f.reset) return;
  const int W = f.W, H = f.H;
  const float4 nd = ldh(f.nd, py * f.p_nd + px);
  if (nd.w < 0.0f) return;
  const float4 mv = ldh(f.mv, py * f.p_mv + px);
  const int o = py * W + px;
  const int ti = (threadIdx.y + 1) * SW + threadIdx.x + 1;
  const float4 illum = sI[ti];
  const float l = lum(illum);
  float s1x = 0.f, s1y = 0.f, s1z = 0.f, cnt = 0.f;
  for (int j = 0; j < 9; j++) {
    const float4 c = sI[ti + (j / 3 - 1) * SW + (j % 3 - 1)];
    s1x += c.x * c.w; s1y += c.y * c.w; s1z += c.z * c.w;
    cnt += c.w;
  }
  cnt = fmaxf(cnt, 1.0f);
  const float mu[3] = {s1x / cnt, s1y / cnt, s1z / cnt};
  const float slm = lum3(mu[0], mu[1], mu[2]);
  float sv[3] = {0.f, 0.f, 0.f}, svar = 0.f;
  for (int j = 0; j < 9; j++) {
    const float4 c = sI[ti + (j / 3 - 1) * SW + (j % 3 - 1)];
    const float dx = c.x - mu[0], dy = c.y - mu[1], dz = c.z - mu[2];
    const float dl = lum(c) - slm;
    sv[0] += c.w * dx * dx; sv[1] += c.w * dy * dy; sv[2] += c.w * dz * dz;
    svar += c.w * dl * dl;
  }
  const float sd[3] = {sqrtf(fmaxf(sv[0] / cnt, 1e-12f)), sqrtf(fmaxf(sv[1] / cnt, 1e-12f)),
                       sqrtf(fmaxf(sv[2] / cnt, 1e-12f))};
  svar /= cnt;
  // reprojection: the taps, their normalised weights and whether the history is used
  const float ppx = (float)px + mv.x, ppy = (float)py + mv.y;
  const float bxf = floorf(ppx), byf = floorf(ppy);
  const float fx = ppx - bxf, fy = ppy - byf;
  const int bix = __float2int_rz(bxf), biy = __float2int_rz(byf);
  const int cx = __float2int_rz(floorf(ppx + 0.5f)), cy = __float2int_rz(floorf(ppy + 0.5f));
  int tq[9];
  float tw[9];
  int nt = 0;
  float hc[3] = {0.f, 0.f, 0.f};
  float4 hm = make_float4(0.f, 0.f, 0.f, 0.f);
  float sumW = 0.f;
  const float wts[4] = {(1.0f - fx) * (1.0f - fy), fx * (1.0f - fy), (1.0f - fx) * fy, fx * fy};
  for (int i = 0; i < 4; i++) {
    const int qx = bix + (i & 1), qy = biy + (i >> 1);
    if (wts[i] > 0.0f && qx >= 0 && qy >= 0 && qx < W && qy < H &&
        check_key(ldh(f.key_prev, qy * W + qx), nd, mv.w, mv.z)) {
      const int q = qy * W + qx;
      const float4 c = ldh(f.hist_prev, q), m = ldh(f.mom_prev, q);
      sumW += wts[i];
      hc[0] += wts[i] * c.x; hc[1] += wts[i] * c.y; hc[2] += wts[i] * c.z;
      hm.x += wts[i] * m.x; hm.y += wts[i] * m.y; hm.z += wts[i] * m.z; hm.w += wts[i] * m.w;
      tq[nt] = q;
      tw[nt] = wts[i];
      nt++;
    }
  }
  bool has = false;
  if (sumW >= 0.01f) {
    for (int c = 0; c < 3; c++) hc[c] /= sumW;
    hm.x /= sumW; hm.y /= sumW; hm.z /= sumW; hm.w /= sumW;
    for (int k = 0; k < nt; k++) tw[k] /= sumW;
    has = true;
  } else {
    float n3 = 0.f;
    hc[0] = hc[1] = hc[2] = 0.f;
    hm = make_float4(0.f, 0.f, 0.f, 0.f);
    nt = 0;
    for (int j = 0; j < 9; j++) {
      const int qx = cx + j % 3 - 1, qy = cy + j / 3 - 1;
      if (qx >= 0 && qy >= 0 && qx < W && qy < H && check_key(ldh(f.key_prev, qy * W + qx), nd, mv.w, mv.z)) {
        const int q = qy * W + qx;
        const float4 c = ldh(f.hist_prev, q), m = ldh(f.mom_prev, q);
        n3 += 1.0f;
        hc[0] += c.x; hc[1] += c.y; hc[2] += c.z;
        hm.x += m.x; hm.y += m.y; hm.z += m.z; hm.w += m.w;
        tq[nt] = q;
        nt++;
      }
    }
    if (n3 > 0.0f) {
      for (int c = 0; c < 3; c++) hc[c] /= n3;
      hm.x /= n3; hm.y /= n3; hm.z /= n3; hm.w /= n3;
      for (int k = 0; k < nt; k++) tw[k] = 1.0f / n3;
      has = true;
    }
  }
  has = has && hm.w > 0.0f;
  if (!has) return;  // A0 and the moments come from this frame alone
  const int hq = (clampi(cy, 0, H - 1) >> 1) * f.W2 + (clampi(cx, 0, W - 1) >> 1);
  const float4 pq = ldh(f.par0_prev, hq);
  const float alpha = pq.x, gamma = pq.y;
  // forward of the blend
  const float il[3] = {illum.x, illum.y, illum.z};
  float hcl[3];
  int clampside[3];  // -1 clamped to mu - gamma sd, +1 to mu + gamma sd, 0 not clamped
  for (int c = 0; c < 3; c++) {
    const float lo = mu[c] - gamma * sd[c], hi = mu[c] + gamma * sd[c];
    hcl[c] = fminf(fmaxf(hc[c], lo), hi);
    clampside[c] = hc[c] < lo ? -1 : (hc[c] > hi ? 1 : 0);
  }
  const float len1 = fminf(hm.w + 1.0f, HMAX);
  const float inv = 1.0f / len1;
  const bool a_is_alpha = alpha >= inv;
  const float a = fmaxf(alpha, inv);
  const float nmx = hm.x + (l - hm.x) * a, nmy = hm.y + (l * l - hm.y) * a;
  const bool b_is_inv = inv > 1.0f / 6.0f;
  const float b = fmaxf(1.0f / 6.0f, inv);
  const float tv = nmy - nmx * nmx;
  const float tvar = fmaxf(tv, 0.0f);
  const float kk = fminf(len1 / 4.0f, 1.0f);
  // seeds
  const float4 gAo = gA ? gA[o] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 gMo = gM ? gM[o] : make_float4(0.f, 0.f, 0.f, 0.f);
  float g_nmx = gMo.x, g_nmy = gMo.y, g_nf = gMo.z, g_len = gMo.w;
  // A.w = svar + (tvar - svar) k
  const float g_tvar = gAo.w * kk;
  if (len1 < 4.0f) g_len += gAo.w * (tvar - svar) * 0.25f;
  if (tv > 0.0f) { g_nmy += g_tvar; g_nmx += -2.0f * nmx * g_tvar; }
  // nfast = hm.z + (l - hm.z) b
  float g_hm[4] = {0.f, 0.f, g_nf * (1.0f - b), 0.f};
  if (b_is_inv) g_len += g_nf * (l - hm.z) * (-inv * inv);
  // moments m1 / m2 and the colour blend
  float g_a = g_nmx * (l - hm.x) + g_nmy * (l * l - hm.y);
  g_hm[0] = g_nmx * (1.0f - a);
  g_hm[1] = g_nmy * (1.0f - a);
  const float gcol[3] = {gAo.x, gAo.y, gAo.z};
  float g_hc[3], g_gamma = 0.0f;
  for (int c = 0; c < 3; c++) {
    g_a += gcol[c] * (il[c] - hcl[c]);
    const float g_hcl = gcol[c] * (1.0f - a);
    g_hc[c] = clampside[c] == 0 ? g_hcl : 0.0f;
    g_gamma += clampside[c] == 0 ? 0.0f : g_hcl * (float)clampside[c] * sd[c];
  }
  float g_alpha = 0.0f;
  if (a_is_alpha) g_alpha = g_a;
  else g_len += g_a * (-inv * inv);
  if (hm.w + 1.0f < HMAX) g_hm[3] = g_len;
  // the history taps (bilinear weights / sumW, or 1 / n3 in the fallback)
  for (int k = 0; k < nt; k++) {
    const float w = tw[k];
    if (g_hc[0] != 0.f || g_hc[1] != 0.f || g_hc[2] != 0.f) atomic_add4(dhist + tq[k], make_float4(w * g_hc[0], w * g_hc[1], w * g_hc[2], 0.f));
    if (g_hm[0] != 0.f || g_hm[1] != 0.f || g_hm[2] != 0.f || g_hm[3] != 0.f)
      atomic_add4(dmom + tq[k], make_float4(w * g_hm[0], w * g_hm[1], w * g_hm[2], w * g_hm[3]));
  }
  if (g_alpha != 0.f) atomicAdd(&dag[hq].x, g_alpha);
  if (g_gamma != 0.f) atomicAdd(&dag[hq].y, g_gamma);
}

// ------------------------------------------------------------------------------------------------ MLP adjoint
// One row (half-res pixel) per thread: the forward layers, the heads adjoint, then the deltas of the three layers.
// Each row's activations and deltas go to shared memory as one record (stride MB_REC, odd, so the rows' writes fall
// in distinct banks), written as they are formed so that few stay live in registers. The CTA then forms its weight
// gradient as 120 items, one per thread: a (layer, output j, column chunk) of the weight matrix with its bias as the
// last column, accumulated over the CTA's rows in row order with one delta load per row shared by the chunk's
// columns, and writes it as one partial.
constexpr int MB_ROWS = 128, MB_REC = 97;
constexpr int RF = 0, RH1 = 20, RH2 = 36, RD1 = 52, RD2 = 68, RD3 = 84;  // fe | h1 | h2 | d1 | d2 | d3 in a record
constexpr int MB_ITEMS = 120, MB_CHUNK = 9;
__global__ void __launch_bounds__(MB_ROWS) k_mlp_bwd(const TwinFrame T) {
  extern __shared__ float sm[];
  float *th = sm;         // NW
  float *rec = th + NW;   // [ROWS][MB_REC]
  for (int i = threadIdx.x; i < NW; i += MB_ROWS) th[i] = T.theta[i];
  __syncthreads();
  const HushFrame &f = T.f;
  const int r = threadIdx.x;
  const int o = blockIdx.x * MB_ROWS + r;
  float *my = rec + r * MB_REC;
  if (o < f.W2 * f.H2 && f3_guide_tw(f.F3, o).w >= 0.0f) {
    float fe[20];
    load_features(f, o, fe);
#pragma unroll
    for (int i = 0; i < 20; i++) my[RF + i] = fe[i];
    // forward (hush.js:683-704: bias, then the inputs in increasing index)
#pragma unroll 2
    for (int j = 0; j < 16; j++) {
      float a = th[B1o + j];
#pragma unroll
      for (int i = 0; i < 20; i++) a = a + fe[i] * th[W1o + j * 20 + i];
      my[RH1 + j] = fmaxf(a, 0.0f);
    }
    float h[16];
#pragma unroll
    for (int i = 0; i < 16; i++) h[i] = my[RH1 + i];
#pragma unroll 2
    for (int j = 0; j < 16; j++) {
      float a = th[B2o + j];
#pragma unroll
      for (int i = 0; i < 16; i++) a = a + h[i] * th[W2o + j * 16 + i];
      my[RH2 + j] = fmaxf(a, 0.0f);
    }
#pragma unroll
    for (int i = 0; i < 16; i++) h[i] = my[RH2 + i];
    float out[12];
#pragma unroll
    for (int j = 0; j < 12; j++) {
      float a = th[B3o + j];
#pragma unroll
      for (int i = 0; i < 16; i++) a = a + h[i] * th[W3o + j * 16 + i];
      out[j] = a;
    }
    // heads (hush.js:357-362); alpha and gamma act on the next frame's temporal blend only, so within a frame their
    // dL/dpar is zero; the per-pass MLP adjoint still carries a seed given for them
    const float4 q0 = T.dpar[3 * o], q1 = T.dpar[3 * o + 1], q2 = T.dpar[3 * o + 2];
    const float4 p0 = T.par[3 * o], p1 = T.par[3 * o + 1], p2 = T.par[3 * o + 2];
    float d3[12];
    const float sa = sigmoidf_(out[0]), sg = sigmoidf_(out[1]);
    d3[0] = q0.x * (31.0f / 32.0f) * sa * (1.0f - sa);
    d3[1] = q0.y * 7.5f * sg * (1.0f - sg);
    d3[2] = q0.z * p0.z * (1.0f - p0.z);
    d3[3] = q0.w * p0.w * (1.0f - p0.w);
    const float ps[4] = {p1.x, p1.y, p1.z, p1.w}, pc[4] = {p2.x, p2.y, p2.z, p2.w};
    const float gs[4] = {q1.x, q1.y, q1.z, q1.w}, gc[4] = {q2.x, q2.y, q2.z, q2.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      d3[4 + k] = fabsf(out[4 + k]) < 5.0f ? gs[k] * ps[k] : 0.0f;
      d3[8 + k] = fabsf(out[8 + k]) < 4.0f ? gc[k] * pc[k] : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < 12; j++) my[RD3 + j] = d3[j];
    // deltas: d2 = relu'(h2) * W3^T d3 (h holds h2), d1 = relu'(h1) * W2^T d2
    float d2[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      float a = 0.f;
#pragma unroll
      for (int j = 0; j < 12; j++) a += d3[j] * th[W3o + j * 16 + i];
      d2[i] = h[i] > 0.0f ? a : 0.0f;
      my[RD2 + i] = d2[i];
    }
#pragma unroll
    for (int i = 0; i < 16; i++) h[i] = my[RH1 + i];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      float a = 0.f;
#pragma unroll
      for (int j = 0; j < 16; j++) a += d2[j] * th[W2o + j * 16 + i];
      my[RD1 + i] = h[i] > 0.0f ? a : 0.0f;
    }
  } else {  // rows outside the image or on sky carry zeros
#pragma unroll 4
    for (int i = 0; i < MB_REC - 1; i++) my[i] = 0.0f;
  }
  __syncthreads();
  // weight gradient of the CTA. Item it: layer 1 rows j in 3 chunks of 7 of its 21 columns, layer 2 rows in chunks
  // 6 / 6 / 5 of 17, layer 3 rows in chunks 9 / 8 of 17; the last column of a row is its bias (x = 1).
  const int it = threadIdx.x;
  if (it >= MB_ITEMS) return;
  int L, j, c0, c1;
  if (it < 48) { L = 0; j = it / 3; c0 = 7 * (it % 3); c1 = c0 + 7; }
  else if (it < 96) { L = 1; j = (it - 48) / 3; c0 = 6 * ((it - 48) % 3); c1 = min(c0 + 6, 17); }
  else { L = 2; j = (it - 96) / 2; c0 = 9 * ((it - 96) % 2); c1 = min(c0 + 9, 17); }
  const int n_in = L == 0 ? 20 : 16;
  const int d_off = (L == 0 ? RD1 : (L == 1 ? RD2 : RD3)) + j;
  const int x_off = (L == 0 ? RF : (L == 1 ? RH1 : RH2)) + c0;
  const int w_off = (L == 0 ? W1o : (L == 1 ? W2o : W3o)) + j * n_in + c0;
  const int b_off = (L == 0 ? B1o : (L == 1 ? B2o : B3o)) + j;
  const int nx = min(c1, n_in) - c0;
  const bool bias = c1 > n_in;
  float acc[MB_CHUNK], accb = 0.f;
#pragma unroll
  for (int c = 0; c < MB_CHUNK; c++) acc[c] = 0.f;
#pragma unroll 4
  for (int k = 0; k < MB_ROWS; k++) {
    const float *R = rec + k * MB_REC;
    const float dv = R[d_off];
#pragma unroll
    for (int c = 0; c < MB_CHUNK; c++)
      if (c < nx) acc[c] += dv * R[x_off + c];
    accb += dv;
  }
  float *part = T.partials + (size_t)blockIdx.x * NW;
#pragma unroll
  for (int c = 0; c < MB_CHUNK; c++)
    if (c < nx) part[w_off + c] = acc[c];
  if (bias) part[b_off] = accb;
}
constexpr size_t MB_SMEM = (size_t)(NW + MB_ROWS * MB_REC) * sizeof(float);

// dtheta += sum over CTAs of the partials, in FP64 and in a fixed order: 32 parameters per block on the lanes, the
// CTAs split over the 8 warps (c = w, w + 8, ...), then the 8 warp sums added in warp order.
constexpr int RP_THREADS = 256, RP_PARAMS = 32;
__global__ void __launch_bounds__(RP_THREADS) k_reduce_partials(const float *partials, int nparts, double *grad) {
  __shared__ double ws[RP_THREADS / 32][RP_PARAMS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int p = blockIdx.x * RP_PARAMS + lane;
  double a = 0.0;
  if (p < NW)
    for (int c = w; c < nparts; c += RP_THREADS / 32) a += (double)partials[(size_t)c * NW + p];
  ws[w][lane] = a;
  __syncthreads();
  if (w == 0 && p < NW) {
    double s = 0.0;
    for (int k = 0; k < RP_THREADS / 32; k++) s += ws[k][lane];
    grad[p] += s;
  }
}
constexpr int RP_BLOCKS = (NW + RP_PARAMS - 1) / RP_PARAMS;

// ------------------------------------------------------------------------------------------------ MLP on tensor cores
// The twin's MLP as tcgen05 GEMM tiles on bf16 (or f16) operands with FP32 accumulation in TMEM: 128 rows per CTA
// (one per thread), each layer one M = 128, N = 16 MMA (K = 32 / 16 / 16); the adjoint's delta products d2 = d3 W3
// and d1 = d2 W2 the same way, and the CTA's whole weight gradient as one M = 128, N = 64, K = 128 product of the
// deltas (rows m: d1 | d2 | d3) and the activations (rows n: features | h1 | h2 | 1, the last giving the biases) over
// the CTA's rows. Operands are K-major without swizzle (8-row x 16-byte core matrices); one thread issues and commits,
// everyone waits on the mbarrier with a bounded poll and reads its own TMEM lane (warp w: lanes 32 w ..). Bias, ReLU,
// the heads and their adjoint stay FP32, as do the FP32 master weights the operands are rounded from.
constexpr int TC_ROWS = 128;
constexpr uint32_t TC_POLLS = 1u << 22;
struct TcTrainSmem {
  alignas(8) uint64_t mbar;
  uint32_t tmem;
  float bias[44];                                  // b1 | b2 | b3
  alignas(128) uint8_t x[TC_ROWS * 32 * 2];        // layer 1 A: rows x 32 (20 features, zero padded), kcore 4
  alignas(128) uint8_t h[TC_ROWS * 16 * 2];        // layer 2 / 3 and delta-product A: rows x 16, kcore 2
  alignas(128) uint8_t w1[16 * 32 * 2];            // B: W1 (n = output, k = input), kcore 4
  alignas(128) uint8_t w2[16 * 16 * 2];            // B: W2
  alignas(128) uint8_t w3[16 * 16 * 2];            // B: W3 (outputs 12..15 zero)
  alignas(128) uint8_t w3t[16 * 16 * 2];           // B of d2 = d3 W3: W3^T (k = 12..15 zero)
  alignas(128) uint8_t w2t[16 * 16 * 2];           // B of d1 = d2 W2: W2^T
  alignas(128) uint8_t ag[128 * TC_ROWS * 2];      // weight-gradient A: deltas (m) x rows (k), kcore 16
  alignas(128) uint8_t bg[64 * TC_ROWS * 2];       // weight-gradient B: activations (n) x rows (k), kcore 16
};
constexpr size_t TC_SMEM_FWD = offsetof(TcTrainSmem, ag) + 128, TC_SMEM_BWD = sizeof(TcTrainSmem) + 128;

template <bool BF16>
HD_INL uint16_t tc_op(float v) {
  if constexpr (BF16) return __bfloat16_as_ushort(__float2bfloat16_rn(v));
  else return __half_as_ushort(__float2half_rn(v));
}
template <bool BF16>
HD_INL uint4 tc_pack8(const float *v) {
  uint4 q;
  q.x = (uint32_t)tc_op<BF16>(v[0]) | ((uint32_t)tc_op<BF16>(v[1]) << 16);
  q.y = (uint32_t)tc_op<BF16>(v[2]) | ((uint32_t)tc_op<BF16>(v[3]) << 16);
  q.z = (uint32_t)tc_op<BF16>(v[4]) | ((uint32_t)tc_op<BF16>(v[5]) << 16);
  q.w = (uint32_t)tc_op<BF16>(v[6]) | ((uint32_t)tc_op<BF16>(v[7]) << 16);
  return q;
}
HD_INL TcTrainSmem &tc_smem(unsigned char *raw) {  // 128-byte aligned view of the dynamic shared memory
  return *reinterpret_cast<TcTrainSmem *>((reinterpret_cast<uintptr_t>(raw) + 127) & ~(uintptr_t)127);
}
template <bool BF16>
HD_INL void tc_put(uint8_t *base, int row, int k, int kcore, float v) {
  *reinterpret_cast<uint16_t *>(base + umma::kmajor_off(row, k, kcore)) = tc_op<BF16>(v);
}

// Set-up shared by both kernels: TMEM (ncols), the mbarrier, the weight operands and FP32 biases from theta.
template <bool BF16>
__device__ void tc_setup(TcTrainSmem &S, const float *theta, uint32_t ncols) {
  const int li = threadIdx.x;
  if (li < 32) {
    umma::tmem_alloc(umma::smem_u32(&S.tmem), ncols);
    umma::tmem_relinquish();
  }
  if (li == 0) umma::mbar_init(umma::smem_u32(&S.mbar), 1);
  for (int e = li; e < 16 * 32; e += TC_ROWS) {
    const int n = e / 32, k = e % 32;
    tc_put<BF16>(S.w1, n, k, 4, k < 20 ? theta[W1o + n * 20 + k] : 0.0f);
  }
  for (int e = li; e < 16 * 16; e += TC_ROWS) {
    const int n = e / 16, k = e % 16;
    tc_put<BF16>(S.w2, n, k, 2, theta[W2o + n * 16 + k]);
    tc_put<BF16>(S.w3, n, k, 2, n < 12 ? theta[W3o + n * 16 + k] : 0.0f);
    tc_put<BF16>(S.w3t, n, k, 2, k < 12 ? theta[W3o + k * 16 + n] : 0.0f);
    tc_put<BF16>(S.w2t, n, k, 2, theta[W2o + k * 16 + n]);
  }
  if (li < 16) { S.bias[li] = theta[B1o + li]; S.bias[16 + li] = theta[B2o + li]; }
  if (li < 12) S.bias[32 + li] = theta[B3o + li];
}

// One product D[row][n] = sum_k A[row][k] B[n][k] into TMEM columns [0, N); waits (bounded) and loads this thread's
// first 16 columns into d. Returns false if the wait gave up.
HD_INL bool tc_product(TcTrainSmem &S, const uint8_t *a, int kcore_a, const uint8_t *b, int kcore_b, int kblocks,
                       uint32_t idesc, uint32_t &phase, float *d) {
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  const uint32_t mbar = umma::smem_u32(&S.mbar);
  if (threadIdx.x == 0) {
    umma::fence_after_sync();
    const uint32_t a0 = umma::smem_u32(a), b0 = umma::smem_u32(b);
    for (int kb = 0; kb < kblocks; kb++)
      umma::mma_f16(S.tmem, umma::sdesc(a0 + 256u * kb, 128, 128 * kcore_a),
                    umma::sdesc(b0 + 256u * kb, 128, 128 * kcore_b), idesc, kb > 0 ? 1u : 0u);
    umma::commit(mbar);
  }
  const bool ok = umma::mbar_wait_bounded(mbar, phase, TC_POLLS);
  phase ^= 1u;
  umma::fence_after_sync();
  if (d) umma::ld16(S.tmem + ((uint32_t)(32 * (threadIdx.x >> 5)) << 16), d);
  return ok;
}

// The three layers for this thread's row: fe (zeros for a dead row) -> h1, h2 (post-ReLU, FP32) and out (FP32).
template <bool BF16>
__device__ bool tc_forward(TcTrainSmem &S, const float *fe, float *h1, float *h2, float *out, uint32_t &phase) {
  constexpr uint32_t ID = umma::idesc_f16(BF16 ? 1 : 0, 128, 16);
  const int li = threadIdx.x;
  float v[8];
#pragma unroll
  for (int c = 0; c < 4; c++) {
#pragma unroll
    for (int e = 0; e < 8; e++) v[e] = 8 * c + e < 20 ? fe[8 * c + e] : 0.0f;
    *reinterpret_cast<uint4 *>(S.x + umma::kmajor_off(li, 8 * c, 4)) = tc_pack8<BF16>(v);
  }
  float d[16];
  bool ok = tc_product(S, S.x, 4, S.w1, 4, 2, ID, phase, d);
#pragma unroll
  for (int j = 0; j < 16; j++) h1[j] = fmaxf(d[j] + S.bias[j], 0.0f);
  *reinterpret_cast<uint4 *>(S.h + umma::kmajor_off(li, 0, 2)) = tc_pack8<BF16>(h1);
  *reinterpret_cast<uint4 *>(S.h + umma::kmajor_off(li, 8, 2)) = tc_pack8<BF16>(h1 + 8);
  ok &= tc_product(S, S.h, 2, S.w2, 2, 1, ID, phase, d);
#pragma unroll
  for (int j = 0; j < 16; j++) h2[j] = fmaxf(d[j] + S.bias[16 + j], 0.0f);
  *reinterpret_cast<uint4 *>(S.h + umma::kmajor_off(li, 0, 2)) = tc_pack8<BF16>(h2);
  *reinterpret_cast<uint4 *>(S.h + umma::kmajor_off(li, 8, 2)) = tc_pack8<BF16>(h2 + 8);
  ok &= tc_product(S, S.h, 2, S.w3, 2, 1, ID, phase, d);
#pragma unroll
  for (int j = 0; j < 12; j++) out[j] = d[j] + S.bias[32 + j];
  return ok;
}

HD_INL void tc_release(TcTrainSmem &S, uint32_t ncols) {
  umma::fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) {
    umma::fence_after_sync();
    umma::tmem_dealloc(S.tmem, ncols);
  }
}

template <bool BF16>
__global__ void __launch_bounds__(TC_ROWS) k_mlp_fwd_tc(const TwinFrame T) {
  extern __shared__ unsigned char tc_raw[];
  TcTrainSmem &S = tc_smem(tc_raw);
  tc_setup<BF16>(S, T.theta, 32);
  const HushFrame &f = T.f;
  const int o = blockIdx.x * TC_ROWS + threadIdx.x;
  const bool in = o < f.W2 * f.H2;
  const bool live = in && f3_guide_tw(f.F3, o).w >= 0.0f;
  float fe[20], h1[16], h2[16], out[12];
  if (live) load_features(f, o, fe);
  else
#pragma unroll
    for (int i = 0; i < 20; i++) fe[i] = 0.0f;
  uint32_t phase = 0;
  const bool ok = tc_forward<BF16>(S, fe, h1, h2, out, phase);
  tc_release(S, 32);
  if (!ok) atomicOr(f.err, 2u);
  if (!in) return;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  if (T.zero_adj) { T.dpar[3 * o] = z4; T.dpar[3 * o + 1] = z4; T.dpar[3 * o + 2] = z4; }
  if (!live) {
    T.par[3 * o] = z4; T.par[3 * o + 1] = z4; T.par[3 * o + 2] = z4;
    sth(f.par0, o, z4); sth(f.par1, o, z4); sth(f.par2, o, z4);
    return;
  }
  float4 p0, p1, p2;
  mlp_heads(out, p0, p1, p2);
  T.par[3 * o] = p0; T.par[3 * o + 1] = p1; T.par[3 * o + 2] = p2;
  sth(f.par0, o, p0); sth(f.par1, o, p1); sth(f.par2, o, p2);
}

template <bool BF16>
__global__ void __launch_bounds__(TC_ROWS) k_mlp_bwd_tc(const TwinFrame T) {
  extern __shared__ unsigned char tc_raw[];
  TcTrainSmem &S = tc_smem(tc_raw);
  tc_setup<BF16>(S, T.theta, 64);
  const HushFrame &f = T.f;
  const int li = threadIdx.x;
  const int o = blockIdx.x * TC_ROWS + li;
  const bool live = o < f.W2 * f.H2 && f3_guide_tw(f.F3, o).w >= 0.0f;
  float fe[20], h1[16], h2[16], out[12];
  if (live) load_features(f, o, fe);
  else
#pragma unroll
    for (int i = 0; i < 20; i++) fe[i] = 0.0f;
  uint32_t phase = 0;
  bool ok = tc_forward<BF16>(S, fe, h1, h2, out, phase);
  // heads adjoint (hush.js:357-362), FP32; dead rows carry zero deltas
  float d3[16];
#pragma unroll
  for (int j = 0; j < 16; j++) d3[j] = 0.0f;
  if (live) {
    const float4 q0 = T.dpar[3 * o], q1 = T.dpar[3 * o + 1], q2 = T.dpar[3 * o + 2];
    const float4 p0 = T.par[3 * o], p1 = T.par[3 * o + 1], p2 = T.par[3 * o + 2];
    const float sa = sigmoidf_(out[0]), sg = sigmoidf_(out[1]);
    d3[0] = q0.x * (31.0f / 32.0f) * sa * (1.0f - sa);
    d3[1] = q0.y * 7.5f * sg * (1.0f - sg);
    d3[2] = q0.z * p0.z * (1.0f - p0.z);
    d3[3] = q0.w * p0.w * (1.0f - p0.w);
    const float ps[4] = {p1.x, p1.y, p1.z, p1.w}, pc[4] = {p2.x, p2.y, p2.z, p2.w};
    const float gs[4] = {q1.x, q1.y, q1.z, q1.w}, gc[4] = {q2.x, q2.y, q2.z, q2.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      d3[4 + k] = fabsf(out[4 + k]) < 5.0f ? gs[k] * ps[k] : 0.0f;
      d3[8 + k] = fabsf(out[8 + k]) < 4.0f ? gc[k] * pc[k] : 0.0f;
    }
  }
  // d2 = relu'(h2) (d3 W3), d1 = relu'(h1) (d2 W2)
  constexpr uint32_t ID = umma::idesc_f16(BF16 ? 1 : 0, 128, 16);
  *reinterpret_cast<uint4 *>(S.h + umma::kmajor_off(li, 0, 2)) = tc_pack8<BF16>(d3);
  *reinterpret_cast<uint4 *>(S.h + umma::kmajor_off(li, 8, 2)) = tc_pack8<BF16>(d3 + 8);
  float d[16], d2[16], d1[16];
  ok &= tc_product(S, S.h, 2, S.w3t, 2, 1, ID, phase, d);
#pragma unroll
  for (int i = 0; i < 16; i++) d2[i] = h2[i] > 0.0f ? d[i] : 0.0f;
  *reinterpret_cast<uint4 *>(S.h + umma::kmajor_off(li, 0, 2)) = tc_pack8<BF16>(d2);
  *reinterpret_cast<uint4 *>(S.h + umma::kmajor_off(li, 8, 2)) = tc_pack8<BF16>(d2 + 8);
  ok &= tc_product(S, S.h, 2, S.w2t, 2, 1, ID, phase, d);
#pragma unroll
  for (int i = 0; i < 16; i++) d1[i] = h1[i] > 0.0f ? d[i] : 0.0f;
  // the weight-gradient operands: column k = this row
#pragma unroll
  for (int m = 0; m < 16; m++) {
    tc_put<BF16>(S.ag, m, li, 16, d1[m]);
    tc_put<BF16>(S.ag, 16 + m, li, 16, d2[m]);
  }
#pragma unroll
  for (int m = 0; m < 12; m++) tc_put<BF16>(S.ag, 32 + m, li, 16, d3[m]);
#pragma unroll
  for (int n = 0; n < 20; n++) tc_put<BF16>(S.bg, n, li, 16, fe[n]);
#pragma unroll
  for (int n = 0; n < 16; n++) {
    tc_put<BF16>(S.bg, 20 + n, li, 16, h1[n]);
    tc_put<BF16>(S.bg, 36 + n, li, 16, h2[n]);
  }
  tc_put<BF16>(S.bg, 52, li, 16, 1.0f);
  // G[m][n] = sum over rows: rows m >= 44 of A and n >= 53 of B are never written; they only reach entries of G
  // that are not read
  ok &= tc_product(S, S.ag, 16, S.bg, 16, TC_ROWS / 16, umma::idesc_f16(BF16 ? 1 : 0, 128, 64), phase, nullptr);
  float *part = T.partials + (size_t)blockIdx.x * NW;
  if (li < 64) {  // warps 0 and 1 hold lanes (delta rows m) 0..63
    float g[64];
    const uint32_t ta = S.tmem + ((uint32_t)(32 * (li >> 5)) << 16);
    umma::ld16(ta, g);
    umma::ld16(ta + 16, g + 16);
    umma::ld16(ta + 32, g + 32);
    umma::ld16(ta + 48, g + 48);
    const int m = li;
    if (m < 16) {
      for (int i = 0; i < 20; i++) part[W1o + m * 20 + i] = g[i];
      part[B1o + m] = g[52];
    } else if (m < 32) {
      for (int i = 0; i < 16; i++) part[W2o + (m - 16) * 16 + i] = g[20 + i];
      part[B2o + m - 16] = g[52];
    } else if (m < 44) {
      for (int i = 0; i < 16; i++) part[W3o + (m - 32) * 16 + i] = g[36 + i];
      part[B3o + m - 32] = g[52];
    }
  }
  tc_release(S, 64);
  if (!ok) atomicOr(f.err, 2u);
}

// Adam on the FP32 master weights (gradient in FP64, optionally clipped by global norm scale `scale`).
__global__ void k_adam(float *theta, float *m, float *v, const double *grad, float lr, float b1, float b2, float eps,
                       float bc1, float bc2, float scale) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NW) return;
  const float g = (float)grad[p] * scale;
  m[p] = b1 * m[p] + (1.0f - b1) * g;
  v[p] = b2 * v[p] + (1.0f - b2) * g * g;
  const float mh = m[p] / bc1, vh = v[p] / bc2;
  theta[p] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace twin
}  // namespace hush

using namespace hush;
using namespace hush::twin;

#ifndef HUSH_TRAIN_LANES
#define HUSH_TRAIN_LANES 8
#endif
// windows hush_trainer_windows runs at once (this trainer and HUSH_TRAIN_LANES - 1 helpers)
constexpr int TRAIN_LANES = HUSH_TRAIN_LANES;

struct hush_trainer_s {
  hush_t *h = nullptr;
  int W = 0, H = 0, W2 = 0, H2 = 0;
  float *theta = nullptr, *m = nullptr, *v = nullptr;
  double *grad = nullptr, *loss = nullptr, *loss_acc = nullptr, *loss_partials = nullptr;
  float4 *par = nullptr, *B[3] = {}, *A1 = nullptr, *X = nullptr, *out[2] = {}, *gT = nullptr, *gT2 = nullptr,
         *dB[3] = {}, *dpar = nullptr, *dX = nullptr, *tcoef = nullptr;
  float *partials = nullptr;
  // TEMPORAL's adjoint: seeds dA0 / dA1 (the fine level's input / output) and dmom (this frame's moments); outputs
  // dhist / dmomp (the previous frame's colour history and moments) and dag (its alpha, gamma per half-res pixel)
  float4 *dA0 = nullptr, *dA1 = nullptr, *dmom = nullptr, *dhist = nullptr, *dmomp = nullptr;
  float2 *dag = nullptr;
  // the coarse levels' per-pass pairs: COARSE1's input ah (half-res block means) and its gradient, the levels c1 / c0
  // (quarter-res) and their gradients, and down()'s quarter-res gradient (scratch of COARSE1's adjoint)
  int W4 = 0, H4 = 0;
  float4 *ah = nullptr, *dah = nullptr, *c1 = nullptr, *dc1 = nullptr, *c0 = nullptr, *dc0 = nullptr, *ddown = nullptr;
  char *coarse_pool = nullptr;
  // hush_trainer_window_bptt: the window's per-frame state records and the carried gradients (ping-pong)
  struct Rec {
    uint2 *A0, *key, *mom, *hist, *taa, *par0, *C0, *C1, *CG;
    uint4 *F[4];
    float4 *out;
  };
  std::vector<Rec> rec;
  char *rec_pool = nullptr;
  float4 *c_hist[2] = {}, *c_mom[2] = {};
  float2 *c_ag[2] = {};
  char *carry_pool = nullptr;
  int n_mlp_ctas = 0, n_loss_ctas = 0;
  int cur = 0, has_prev = 0;
  int adam_t = 0;
  char *pool = nullptr;
  TwinFrame T{};  // the frame fixed by hush_trainer_begin for the per-pass calls
  int begun = 0;
  char *win_pool = nullptr;  // hush_trainer_windows: one window of generated frames (inputs + noise-free image)
  int win_frames = 0;
  // hush_trainer_windows replays a window's training frames as a CUDA graph, one per (frame parity, output slot) at
  // the window's start; captured for one (frame count, lambda, exposure) and re-captured when those change
  int mlp_mode = HUSH_MLP_FP32;  // the twin's MLP: FP32 per thread, or bf16 / f16 tensor-core tiles
  cudaGraphExec_t win_graph[4] = {};
  int wg_frames = 0, wg_mode = -1;
  float wg_lambda = 0.f, wg_exposure = 0.f;
  // hush_trainer_windows_bptt replays a window's forward + reverse sweep as one CUDA graph: its kernel arguments are
  // fixed by the trainer's buffers, records and win_pool, the frame count, lambda, the exposure and the MLP form
  cudaGraphExec_t bptt_graph = nullptr;
  int bg_frames = 0, bg_mode = -1;
  float bg_lambda = 0.f, bg_exposure = 0.f;
  cudaStream_t cap = nullptr;
  // hush_trainer_windows runs windows concurrently on lanes: lane 0 is this trainer, lanes 1.. are helper trainers on
  // private Hush instances of the same size (their own history), reading this trainer's weights and accumulating
  // into their own gradient / loss, which are added into this trainer's after the batch
  hush_trainer_t *lane[TRAIN_LANES] = {};
  hush_t *lane_h[TRAIN_LANES] = {};
  cudaStream_t lane_st[TRAIN_LANES] = {};
  cudaEvent_t lane_ev[TRAIN_LANES] = {};
  cudaEvent_t fork_ev = nullptr;
  bool is_lane = false;
};

static int tr_fail(hush_trainer_t *t, const std::string &m) { return hush_fail(t ? t->h : nullptr, HUSH_ERR_ARG, m); }

extern "C" int hush_trainer_create(hush_t *h, const float *theta, hush_trainer_t **out) {
  if (!h || !out) return hush_fail(h, HUSH_ERR_ARG, "hush_trainer_create: NULL argument");
  *out = nullptr;
  if (h->hidden != 16) return hush_fail(h, HUSH_ERR_ARG, "hush_trainer_create: the trainer needs the h = 16 network");
  cudaSetDevice(h->dev);
  hush_trainer_t *t = new hush_trainer_t();
  t->h = h;
  t->W = h->W; t->H = h->H; t->W2 = h->W2; t->H2 = h->H2;
  const size_t full = (size_t)t->W * t->H, half = (size_t)t->W2 * t->H2;
  t->n_mlp_ctas = (int)((half + MB_ROWS - 1) / MB_ROWS);
  t->n_loss_ctas = (int)((full + 255) / 256);
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t bytes = al(NW * 4) * 3 + al(NW * 8) + al(8) * 2 + al(t->n_loss_ctas * 8) + al(half * 48) * 2 +
                       al(half * 16) * 6 + al(full * 16) * 12 + al(full * 48) + al((size_t)t->n_mlp_ctas * NW * 4) +
                       al(half * 8);
  cudaError_t e = cudaMalloc(&t->pool, bytes);
  if (e != cudaSuccess) { delete t; return hush_cuda_fail(h, e, "cudaMalloc of the trainer"); }
  cudaMemset(t->pool, 0, bytes);
  size_t off = 0;
  auto take = [&](size_t b) { char *p = t->pool + off; off += al(b); return p; };
  t->theta = (float *)take(NW * 4); t->m = (float *)take(NW * 4); t->v = (float *)take(NW * 4);
  t->grad = (double *)take(NW * 8); t->loss = (double *)take(8); t->loss_acc = (double *)take(8);
  t->loss_partials = (double *)take(t->n_loss_ctas * 8);
  t->par = (float4 *)take(half * 48); t->dpar = (float4 *)take(half * 48);
  for (int i = 0; i < 3; i++) { t->B[i] = (float4 *)take(half * 16); t->dB[i] = (float4 *)take(half * 16); }
  t->A1 = (float4 *)take(full * 16); t->X = (float4 *)take(full * 16);
  t->out[0] = (float4 *)take(full * 16); t->out[1] = (float4 *)take(full * 16);
  t->gT = (float4 *)take(full * 16); t->gT2 = (float4 *)take(full * 16); t->dX = (float4 *)take(full * 16);
  t->tcoef = (float4 *)take(full * 48);
  t->partials = (float *)take((size_t)t->n_mlp_ctas * NW * 4);
  t->dA0 = (float4 *)take(full * 16); t->dA1 = (float4 *)take(full * 16); t->dmom = (float4 *)take(full * 16);
  t->dhist = (float4 *)take(full * 16); t->dmomp = (float4 *)take(full * 16);
  t->dag = (float2 *)take(half * 8);
  e = cudaMemcpy(t->theta, theta ? theta : h->wf.data(), NW * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cudaFree(t->pool); delete t; return hush_cuda_fail(h, e, "cudaMemcpy of the weights"); }
  cudaFuncSetAttribute(k_mlp_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MB_SMEM);
  cudaFuncSetAttribute(k_mlp_bwd_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_BWD);
  cudaFuncSetAttribute(k_mlp_bwd_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_BWD);
  *out = t;
  return HUSH_OK;
}

// The coarse levels' buffers, made on first use (the per-pass API only; the frame and window paths never touch them).
static cudaError_t ensure_coarse(hush_trainer_t *t) {
  if (t->coarse_pool) return cudaSuccess;
  t->W4 = t->h->W4;
  t->H4 = t->h->H4;
  const size_t half = (size_t)t->W2 * t->H2, quarter = (size_t)t->W4 * t->H4;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t bytes = al(half * 16) * 2 + al(quarter * 16) * 5;
  cudaError_t e = cudaMalloc(&t->coarse_pool, bytes);
  if (e != cudaSuccess) {
    t->coarse_pool = nullptr;
    return e;
  }
  e = cudaMemset(t->coarse_pool, 0, bytes);
  size_t off = 0;
  auto take = [&](size_t b) { char *p = t->coarse_pool + off; off += al(b); return (float4 *)p; };
  t->ah = take(half * 16); t->dah = take(half * 16);
  t->c1 = take(quarter * 16); t->dc1 = take(quarter * 16); t->c0 = take(quarter * 16); t->dc0 = take(quarter * 16);
  t->ddown = take(quarter * 16);
  return e;
}

extern "C" void hush_trainer_destroy(hush_trainer_t *t) {
  if (!t) return;
  cudaSetDevice(t->h->dev);
  for (int l = 1; l < TRAIN_LANES; l++) {
    if (t->lane[l]) hush_trainer_destroy(t->lane[l]);
    if (t->lane_h[l]) hush_destroy(t->lane_h[l]);
  }
  for (int l = 0; l < TRAIN_LANES; l++) {
    if (t->lane_st[l]) cudaStreamDestroy(t->lane_st[l]);
    if (t->lane_ev[l]) cudaEventDestroy(t->lane_ev[l]);
  }
  if (t->fork_ev) cudaEventDestroy(t->fork_ev);
  for (cudaGraphExec_t &g : t->win_graph)
    if (g) cudaGraphExecDestroy(g);
  if (t->bptt_graph) cudaGraphExecDestroy(t->bptt_graph);
  if (t->cap) cudaStreamDestroy(t->cap);
  cudaFree(t->pool);
  cudaFree(t->coarse_pool);
  cudaFree(t->win_pool);
  cudaFree(t->rec_pool);
  cudaFree(t->carry_pool);
  delete t;
}

// The twin's MLP forward / adjoint (the adjoint includes the FP64 reduction into the gradient) in the trainer's form.
static void launch_mlp_fwd(const hush_trainer_t *t, const TwinFrame &T, cudaStream_t st) {
  const int half = T.f.W2 * T.f.H2;
  if (t->mlp_mode == HUSH_MLP_BF16) k_mlp_fwd_tc<true><<<(half + TC_ROWS - 1) / TC_ROWS, TC_ROWS, TC_SMEM_FWD, st>>>(T);
  else if (t->mlp_mode == HUSH_MLP_F16) k_mlp_fwd_tc<false><<<(half + TC_ROWS - 1) / TC_ROWS, TC_ROWS, TC_SMEM_FWD, st>>>(T);
  else k_mlp_fwd<<<(half + 127) / 128, 128, 0, st>>>(T);
}
static void launch_mlp_bwd(const hush_trainer_t *t, const TwinFrame &T, cudaStream_t st) {
  if (t->mlp_mode == HUSH_MLP_BF16) k_mlp_bwd_tc<true><<<t->n_mlp_ctas, TC_ROWS, TC_SMEM_BWD, st>>>(T);
  else if (t->mlp_mode == HUSH_MLP_F16) k_mlp_bwd_tc<false><<<t->n_mlp_ctas, TC_ROWS, TC_SMEM_BWD, st>>>(T);
  else k_mlp_bwd<<<t->n_mlp_ctas, MB_ROWS, MB_SMEM, st>>>(T);
  k_reduce_partials<<<RP_BLOCKS, RP_THREADS, 0, st>>>(t->partials, t->n_mlp_ctas, t->grad);
}

static TwinFrame make_twin(hush_trainer_t *t, const hush_inputs *in, const float *clean, const float *clean_prev,
                           float lambda_t) {
  TwinFrame T;
  std::memset(&T, 0, sizeof(T));
  T.f = hush_make_frame(t->h, in);
  T.theta = t->theta;
  T.par = t->par;
  T.B1 = t->B[0]; T.B2 = t->B[1]; T.B3 = t->B[2];
  T.A1 = t->A1; T.X = t->X;
  T.out = t->out[t->cur];
  T.out_prev = t->out[t->cur ^ 1];
  T.clean = clean;
  T.clean_prev = clean_prev;
  T.gT = t->gT;
  T.zero_adj = 0;
  T.dB1 = t->dB[0]; T.dB2 = t->dB[1]; T.dB3 = t->dB[2];
  T.dpar = t->dpar;
  T.partials = t->partials;
  T.loss_partials = t->loss_partials;
  T.lambda_t = lambda_t;
  T.has_prev = (t->has_prev && clean_prev && !t->h->reset) ? 1 : 0;
  T.inv_n = 1.0f / (3.0f * (float)t->W * (float)t->H);
  return T;
}

// Forward (and, if `backward`, the adjoint accumulated into the weight gradient) of one frame of the twin. Does not
// advance the frame: repeated calls see the same history (finite differences); hush_trainer_end_frame advances.
extern "C" int hush_trainer_frame(hush_trainer_t *t, const hush_inputs *in, const float *clean, const float *clean_prev,
                                  float lambda_t, int backward, void *stream, double *loss_out) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_frame: NULL trainer");
  if (!clean) return tr_fail(t, "hush_trainer_frame: missing clean image");
  if (t->W != t->h->W || t->H != t->h->H)
    return tr_fail(t, "hush_trainer_frame: the denoiser was resized after the trainer was created");
  int rc = hush_check_inputs(t->h, in);
  if (rc != HUSH_OK) return rc;
  cudaSetDevice(t->h->dev);
  cudaStream_t st = (cudaStream_t)stream;
  TwinFrame T = make_twin(t, in, clean, clean_prev, lambda_t);
  T.zero_adj = backward ? 1 : 0;  // the forward kernels clear the adjoint accumulators the backward adds into
  const HushFrame &f = T.f;
  // TEMPORAL and the coarse levels as the reference passes (their outputs do not depend on the weights)
  cudaError_t e = launch_pass(PASS_TEMPORAL, f, t->h->w16, st);
  if (e == cudaSuccess) e = launch_pass(PASS_COARSE1, f, t->h->w16, st);
  if (e == cudaSuccess) e = launch_pass(PASS_COARSE2, f, t->h->w16, st);
  if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "trainer pass launch");
  const dim3 blk(TW, TH), gh((f.W2 + TW - 1) / TW, (f.H2 + TH - 1) / TH), gf((f.W + TW - 1) / TW, (f.H + TH - 1) / TH);
  launch_mlp_fwd(t, T, st);
  k_mid_fwd<1><<<gh, blk, 0, st>>>(T);
  k_mid_fwd<2><<<gh, blk, 0, st>>>(T);
  k_mid_fwd<3><<<gh, blk, 0, st>>>(T);
  k_fine_fwd<<<gf, blk, 0, st>>>(T);
  k_taa_fwd<<<gf, blk, 0, st>>>(T);
  k_loss<<<t->n_loss_ctas, 256, 0, st>>>(T, backward);
  k_reduce_f64<<<1, 256, 0, st>>>(t->loss_partials, t->n_loss_ctas, t->loss, t->loss_acc);
  if (backward) {
    k_taa_bwd_coef<<<gf, blk, 0, st>>>(T, t->gT, t->tcoef);
    k_taa_bwd_gather<<<gf, blk, 0, st>>>(T, t->tcoef, t->gT2);
    k_fine_bwd<true><<<gf, blk, 0, st>>>(T, t->gT2);
    k_mid_bwd<3><<<gh, blk, 0, st>>>(T);
    k_mid_bwd<2><<<gh, blk, 0, st>>>(T);
    k_mid_bwd<1><<<gh, blk, 0, st>>>(T);
    launch_mlp_bwd(t, T, st);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "trainer kernel launch");
  if (loss_out) {
    e = cudaMemcpyAsync(loss_out, t->loss, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "reading the loss");
  }
  return HUSH_OK;
}

// Sum of the losses of the frames since the last call (read and zeroed; synchronises the stream).
extern "C" int hush_trainer_loss_sum(hush_trainer_t *t, void *stream, double *out) {
  if (!t || !out) return hush_fail(t ? t->h : nullptr, HUSH_ERR_ARG, "hush_trainer_loss_sum: NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(out, t->loss_acc, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->loss_acc, 0, 8, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "reading the loss sum");
}

extern "C" int hush_trainer_end_frame(hush_trainer_t *t) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_end_frame: NULL trainer");
  t->begun = 0;
  t->has_prev = 1;
  t->cur ^= 1;
  return hush_end_frame(t->h);
}

extern "C" int hush_trainer_reset(hush_trainer_t *t) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_reset: NULL trainer");
  t->begun = 0;
  t->has_prev = 0;
  return hush_reset(t->h);
}

extern "C" int hush_trainer_zero_grad(hush_trainer_t *t, void *stream) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_zero_grad: NULL trainer");
  cudaError_t e = cudaMemsetAsync(t->grad, 0, NW * 8, (cudaStream_t)stream);
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "cudaMemsetAsync");
}

extern "C" int hush_trainer_grad(hush_trainer_t *t, double *out) {
  if (!t || !out) return hush_fail(t ? t->h : nullptr, HUSH_ERR_ARG, "hush_trainer_grad: NULL argument");
  cudaError_t e = cudaMemcpy(out, t->grad, NW * 8, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "cudaMemcpy");
}

// Device addresses of the gradient accumulator (812 doubles) and the loss sum (1 double), valid for the trainer's
// life, so that data-parallel callers can all-reduce them in place on the trainer's stream before hush_trainer_step.
extern "C" int hush_trainer_accumulators(hush_trainer_t *t, double **grad, double **loss_sum) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_accumulators: NULL trainer");
  if (grad) *grad = t->grad;
  if (loss_sum) *loss_sum = t->loss_acc;
  return HUSH_OK;
}

extern "C" int hush_trainer_theta(hush_trainer_t *t, float *get, const float *set) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_theta: NULL trainer");
  cudaError_t e = cudaSuccess;
  if (set) e = cudaMemcpy(t->theta, set, NW * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && get) e = cudaMemcpy(get, t->theta, NW * 4, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "cudaMemcpy");
}

// dL/dpar of the last backward: 12 floats per half-res pixel (alpha gamma beta kappa s0..s3 c0..c3), and the FP32
// parameters themselves.
extern "C" int hush_trainer_par(hush_trainer_t *t, float *par, float *dpar) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_par: NULL trainer");
  const size_t n = (size_t)t->W2 * t->H2 * 48;
  cudaError_t e = cudaSuccess;
  if (par) e = cudaMemcpy(par, t->par, n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && dpar) e = cudaMemcpy(dpar, t->dpar, n, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "cudaMemcpy");
}

// The FP32 TAA output of the last forward (rgba, W x H).
extern "C" int hush_trainer_output(hush_trainer_t *t, float *out) {
  if (!t || !out) return hush_fail(t ? t->h : nullptr, HUSH_ERR_ARG, "hush_trainer_output: NULL argument");
  cudaError_t e = cudaMemcpy(out, t->out[t->cur], (size_t)t->W * t->H * 16, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "cudaMemcpy");
}

// Adam step on the accumulated gradient (global-norm clipped to `clip` if clip > 0); zeroes the gradient.
extern "C" int hush_trainer_step(hush_trainer_t *t, float lr, float beta1, float beta2, float eps, float clip,
                                 void *stream, double *grad_norm) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_step: NULL trainer");
  cudaSetDevice(t->h->dev);
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<double> g(NW);
  cudaError_t e = cudaMemcpyAsync(g.data(), t->grad, NW * 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "reading the gradient");
  double n2 = 0.0;
  for (double x : g) n2 += x * x;
  const double norm = std::sqrt(n2);
  if (grad_norm) *grad_norm = norm;
  const float scale = (clip > 0.0f && norm > clip) ? (float)(clip / norm) : 1.0f;
  t->adam_t++;
  const float bc1 = 1.0f - std::pow(beta1, (float)t->adam_t), bc2 = 1.0f - std::pow(beta2, (float)t->adam_t);
  k_adam<<<(NW + 127) / 128, 128, 0, st>>>(t->theta, t->m, t->v, t->grad, lr, beta1, beta2, eps, bc1, bc2, scale);
  e = cudaMemsetAsync(t->grad, 0, NW * 8, st);
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "cudaMemsetAsync");
}

// Rounds the FP32 master weights to the f16 blob (W1 b1 W2 b2 W3 b3, hush.js:20-21), hands it to the denoiser and,
// if blob != NULL, to the caller (812 values).
extern "C" int hush_trainer_export(hush_trainer_t *t, uint16_t *blob) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_export: NULL trainer");
  std::vector<float> th(NW);
  cudaError_t e = cudaMemcpy(th.data(), t->theta, NW * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "reading the weights");
  std::vector<uint16_t> b(NW);
  for (int i = 0; i < NW; i++) b[i] = __half_as_ushort(__float2half_rn(th[i]));
  if (blob) std::memcpy(blob, b.data(), NW * 2);
  return hush_set_weights(t->h, b.data(), NW);
}

// Windows of the analytic scene generator, trained in place: for each seed, the window's frames are generated on the
// device into trainer-owned buffers and run forward + backward as hush_train_step runs them (history reset at the
// window's start, the temporal term from its second frame on), accumulating gradient and loss without a step.
// One window's training frames on `st` from the generated frames in win_pool: history reset, then per frame forward
// + backward and end-of-frame.
static int window_frames(hush_trainer_t *t, int n_frames, size_t img, size_t per, float lambda_t, cudaStream_t st) {
  int rc = hush_trainer_reset(t);
  for (int i = 0; i < n_frames && rc == HUSH_OK; i++) {
    char *b = t->win_pool + per * i;
    hush_inputs in;
    std::memset(&in, 0, sizeof(in));
    in.radiance = b; in.normal_depth = b + img; in.motion = b + 2 * img; in.material = b + 3 * img;
    in.emission = b + 4 * img;
    const float *clean = (const float *)(b + 5 * img);
    const float *clean_prev = i ? (const float *)(t->win_pool + per * (i - 1) + 5 * img) : nullptr;
    rc = hush_trainer_frame(t, &in, clean, clean_prev, lambda_t, 1, st, nullptr);
    if (rc == HUSH_OK) rc = hush_trainer_end_frame(t);
  }
  return rc;
}

static void drop_window_graphs(hush_trainer_t *t) {
  for (cudaGraphExec_t &g : t->win_graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

// Windows of the analytic scene generator, trained in place: for each seed, the window's frames are generated on the
// device into trainer-owned buffers and run forward + backward as hush_train_step runs them (history reset at the
// window's start, the temporal term from its second frame on), accumulating gradient and loss without a step. The
// training frames of a window replay as one CUDA graph: every kernel argument of a window is fixed by the buffers,
// lambda, the exposure and the frame parity / output slot at its start, which the graph cache is keyed on; the host
// state (frame counter, history flags) advances exactly as the direct calls advance it. The generation runs outside
// the graph because its scene parameters change with the seed.
// The windows seeds[0], seeds[stride], ... in order on one trainer and stream.
static void drop_bptt_graph(hush_trainer_t *t) {
  if (t->bptt_graph) { cudaGraphExecDestroy(t->bptt_graph); t->bptt_graph = nullptr; }
}

// win_pool for n_frames generated frames (each: the five G-buffer images, img bytes apart, then the noise-free image;
// per bytes a frame). Reallocating it drops the graphs that captured its addresses.
static int ensure_win_pool(hush_trainer_t *t, int n_frames, size_t &img, size_t &per) {
  const size_t full = (size_t)t->W * t->H, cl = (full * 12 + 255) & ~(size_t)255;
  img = (full * 8 + 255) & ~(size_t)255;
  per = 5 * img + cl;
  if (t->win_frames < n_frames) {
    drop_window_graphs(t);
    drop_bptt_graph(t);
    cudaFree(t->win_pool);
    t->win_pool = nullptr;
    t->win_frames = 0;
    cudaError_t e = cudaMalloc(&t->win_pool, per * n_frames);
    if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "cudaMalloc of the window buffers");
    t->win_frames = n_frames;
  }
  return HUSH_OK;
}

// The frames of window seed `seed` generated into win_pool on `st`.
static int generate_window(hush_trainer_t *t, const hush_scene *sc, uint32_t seed, int n_frames, size_t img,
                           size_t per, cudaStream_t st) {
  hush_scene w = *sc;
  w.seed = seed;
  for (int i = 0; i < n_frames; i++) {
    char *b = t->win_pool + per * i;
    const int rc = hush_scene_frame_device(&w, i, b, b + img, b + 2 * img, b + 3 * img, b + 4 * img, b + 5 * img, st);
    if (rc != HUSH_OK) return hush_fail(t->h, rc, "training windows: scene generation failed");
  }
  return HUSH_OK;
}

static int windows_serial(hush_trainer_t *t, const hush_scene *sc, const uint32_t *seeds, int n_windows, int stride,
                          int n_frames, float lambda_t, cudaStream_t st) {
  size_t img = 0, per = 0;
  const int prc = ensure_win_pool(t, n_frames, img, per);
  if (prc != HUSH_OK) return prc;
  if (t->wg_frames != n_frames || t->wg_lambda != lambda_t || t->wg_exposure != t->h->exposure ||
      t->wg_mode != t->mlp_mode) {
    drop_window_graphs(t);
    t->wg_frames = n_frames;
    t->wg_lambda = lambda_t;
    t->wg_exposure = t->h->exposure;
    t->wg_mode = t->mlp_mode;
  }
  if (!t->cap) {
    cudaError_t e = cudaStreamCreateWithFlags(&t->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "cudaStreamCreate");
  }
  for (int k = 0; k < n_windows; k += stride) {
    const int grc = generate_window(t, sc, seeds[k], n_frames, img, per, st);
    if (grc != HUSH_OK) return grc;
    cudaGraphExec_t &g = t->win_graph[((t->h->frame & 1) << 1) | (t->cur & 1)];
    if (g) {  // replay, then advance the host state as the frames would
      cudaError_t e = cudaGraphLaunch(g, st);
      if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "cudaGraphLaunch of a training window");
      int rc = hush_trainer_reset(t);
      for (int i = 0; i < n_frames && rc == HUSH_OK; i++) rc = hush_trainer_end_frame(t);
      if (rc != HUSH_OK) return rc;
      continue;
    }
    // capture on the trainer's own stream (the caller's may be the legacy default stream, which cannot capture);
    // the host state advances during the capture exactly once, as it does for the launch that follows
    const int f0 = t->h->frame;
    const bool reset0 = t->h->reset;
    const void *last0 = t->h->last_out;
    const int cur0 = t->cur, prev0 = t->has_prev;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(t->cap, cudaStreamCaptureModeThreadLocal);
    int rc = e == cudaSuccess ? window_frames(t, n_frames, img, per, lambda_t, t->cap) : HUSH_ERR_CUDA;
    const cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(t->cap, &graph) : e;
    if (rc == HUSH_OK && e2 == cudaSuccess) e = cudaGraphInstantiate(&g, graph, 0);
    else e = e2 != cudaSuccess ? e2 : cudaErrorUnknown;
    if (graph) cudaGraphDestroy(graph);
    if (e == cudaSuccess) e = cudaGraphLaunch(g, st);
    if (e != cudaSuccess) {  // capture not possible here: undo the host state and run the frames directly
      cudaGetLastError();
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
      t->h->frame = f0; t->h->reset = reset0; t->h->last_out = last0;
      t->cur = cur0; t->has_prev = prev0;
      rc = window_frames(t, n_frames, img, per, lambda_t, st);
    }
    if (rc != HUSH_OK) return rc;
  }
  return HUSH_OK;
}

// this trainer's accumulators += the helper lanes' (in lane order), which are cleared
struct LaneAcc {
  double *grad[TRAIN_LANES], *loss[TRAIN_LANES];
  int n;
};
__global__ void k_sum_lanes(double *grad, double *loss, LaneAcc la) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < NW) {
    double g = grad[p];
    for (int l = 0; l < la.n; l++) { g += la.grad[l][p]; la.grad[l][p] = 0.0; }
    grad[p] = g;
  }
  if (p == 0) {
    double s = *loss;
    for (int l = 0; l < la.n; l++) { s += *la.loss[l]; *la.loss[l] = 0.0; }
    *loss = s;
  }
}


static int make_lanes(hush_trainer_t *t, int n) {
  hush_t *h = t->h;
  for (int l = 0; l < n; l++) {
    if (!t->lane_st[l]) {
      cudaError_t e = cudaStreamCreateWithFlags(&t->lane_st[l], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->lane_ev[l], cudaEventDisableTiming);
      if (e != cudaSuccess) return hush_cuda_fail(h, e, "creating a training lane");
    }
    if (l == 0 || t->lane[l]) continue;
    hush_desc d = hush_desc_default(t->W, t->H);
    d.exposure = h->exposure;
    d.schedule = HUSH_SCHED_PASSES;
    d.device = h->dev;
    int rc = hush_create(&d, &t->lane_h[l]);
    if (rc == HUSH_OK) rc = hush_trainer_create(t->lane_h[l], nullptr, &t->lane[l]);
    if (rc != HUSH_OK) return hush_fail(h, rc, std::string("creating a training lane: ") + hush_global_error());
    t->lane[l]->theta = t->theta;  // the helper reads this trainer's master weights
    t->lane[l]->is_lane = true;
  }
  if (!t->fork_ev) {
    cudaError_t e = cudaEventCreateWithFlags(&t->fork_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return hush_cuda_fail(h, e, "creating a training lane");
  }
  t->lane[0] = t;
  return HUSH_OK;
}

static int windows_serial_bptt(hush_trainer_t *t, const hush_scene *sc, const uint32_t *seeds, int n_windows,
                               int stride, int n_frames, float lambda_t, cudaStream_t st);

// Windows of the analytic scene generator, trained in place (hush_trainer_windows: per-frame gradient by
// windows_serial; hush_trainer_windows_bptt: through time by windows_serial_bptt): for each seed, the window's frames
// are generated on the device and run forward + backward. Up to TRAIN_LANES windows run concurrently, window k on
// lane k % lanes (each lane its own stream, history, records and accumulators, the lanes forked from and joined back
// to `stream`); the lanes' gradients and losses are then added into this trainer's in lane order.
static int run_windows(hush_trainer_t *t, const hush_scene *sc, const uint32_t *seeds, int n_windows, int n_frames,
                       float lambda_t, void *stream, bool bptt, const char *name) {
  const std::string nm(name);
  if (!t || !sc || !seeds) return hush_fail(t ? t->h : nullptr, HUSH_ERR_ARG, nm + ": NULL argument");
  if (n_windows < 1 || n_frames < 1) return tr_fail(t, nm + ": empty batch");
  if (sc->width != t->W || sc->height != t->H) return tr_fail(t, nm + ": the scene size differs from the trainer's");
  if (t->W != t->h->W || t->H != t->h->H)
    return tr_fail(t, nm + ": the denoiser was resized after the trainer was created");
  if (t->is_lane) return tr_fail(t, nm + ": called on a helper lane");
  cudaSetDevice(t->h->dev);
  cudaStream_t st = (cudaStream_t)stream;
  auto serial = [&](hush_trainer_t *lt, const uint32_t *s, int nw, int stride, cudaStream_t ls) {
    return bptt ? windows_serial_bptt(lt, sc, s, nw, stride, n_frames, lambda_t, ls)
                : windows_serial(lt, sc, s, nw, stride, n_frames, lambda_t, ls);
  };
  const int n = n_windows < TRAIN_LANES ? n_windows : TRAIN_LANES;
  if (n == 1) return serial(t, seeds, n_windows, 1, st);
  int rc = make_lanes(t, n);
  if (rc != HUSH_OK) return rc;
  cudaError_t e = cudaEventRecord(t->fork_ev, st);
  for (int l = 0; l < n && e == cudaSuccess; l++) e = cudaStreamWaitEvent(t->lane_st[l], t->fork_ev, 0);
  if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "forking the training lanes");
  for (int l = 0; l < n && rc == HUSH_OK; l++) {
    hush_trainer_t *lt = t->lane[l];
    if (l > 0) {
      hush_set_exposure(lt->h, t->h->exposure);
      lt->mlp_mode = t->mlp_mode;
      rc = serial(lt, seeds + l, n_windows - l, n, t->lane_st[l]);
      if (rc != HUSH_OK) rc = hush_fail(t->h, rc, std::string("training lane: ") + hush_last_error(lt->h));
    } else {
      rc = serial(t, seeds, n_windows, n, t->lane_st[0]);
    }
  }
  // join every lane that was forked, whatever happened above
  for (int l = 0; l < n; l++) {
    if (cudaEventRecord(t->lane_ev[l], t->lane_st[l]) == cudaSuccess) cudaStreamWaitEvent(st, t->lane_ev[l], 0);
  }
  if (rc != HUSH_OK) return rc;
  LaneAcc la{};
  la.n = n - 1;
  for (int l = 1; l < n; l++) { la.grad[l - 1] = t->lane[l]->grad; la.loss[l - 1] = t->lane[l]->loss_acc; }
  k_sum_lanes<<<(NW + 255) / 256, 256, 0, st>>>(t->grad, t->loss_acc, la);
  e = cudaGetLastError();
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "summing the training lanes");
}

extern "C" int hush_trainer_windows(hush_trainer_t *t, const hush_scene *sc, const uint32_t *seeds, int n_windows,
                                    int n_frames, float lambda_t, void *stream) {
  return run_windows(t, sc, seeds, n_windows, n_frames, lambda_t, stream, false, "hush_trainer_windows");
}

extern "C" int hush_trainer_set_mlp(hush_trainer_t *t, int mode) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_set_mlp: NULL trainer");
  if (mode != HUSH_MLP_FP32 && mode != HUSH_MLP_BF16 && mode != HUSH_MLP_F16)
    return tr_fail(t, "hush_trainer_set_mlp: unknown MLP form");
  t->mlp_mode = mode;
  return HUSH_OK;
}

// ------------------------------------------------------------------------------------------------ per-pass pairs
// The twin's passes one at a time, each as a forward / adjoint pair over the trainer's buffers: the same kernels as
// hush_trainer_frame, except that the TAA adjoint finishes with the tm adjoint (dX rather than d tm(X)) and the fine
// adjoint starts from dX.
extern "C" int hush_trainer_begin(hush_trainer_t *t, const hush_inputs *in, const float *clean, const float *clean_prev,
                                  float lambda_t, void *stream) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_begin: NULL trainer");
  t->begun = 0;
  if (!clean) return tr_fail(t, "hush_trainer_begin: missing clean image");
  if (t->W != t->h->W || t->H != t->h->H)
    return tr_fail(t, "hush_trainer_begin: the denoiser was resized after the trainer was created");
  int rc = hush_check_inputs(t->h, in);
  if (rc != HUSH_OK) return rc;
  cudaSetDevice(t->h->dev);
  cudaStream_t st = (cudaStream_t)stream;
  t->T = make_twin(t, in, clean, clean_prev, lambda_t);
  cudaError_t e = launch_pass(PASS_TEMPORAL, t->T.f, t->h->w16, st);
  if (e == cudaSuccess) e = launch_pass(PASS_COARSE1, t->T.f, t->h->w16, st);
  if (e == cudaSuccess) e = launch_pass(PASS_COARSE2, t->T.f, t->h->w16, st);
  if (e == cudaSuccess) e = ensure_coarse(t);
  if (e == cudaSuccess) {
    const int half = t->W2 * t->H2;
    k_ah_fill<<<(half + 255) / 256, 256, 0, st>>>(t->T, t->ah);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "trainer pass launch");
  t->begun = 1;
  return HUSH_OK;
}

extern "C" int hush_trainer_zero_adjoints(hush_trainer_t *t, void *stream) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_trainer_zero_adjoints: NULL trainer");
  cudaSetDevice(t->h->dev);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t full = (size_t)t->W * t->H, half = (size_t)t->W2 * t->H2;
  cudaError_t e = cudaMemsetAsync(t->dX, 0, full * 16, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->gT, 0, full * 16, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->dpar, 0, half * 48, st);
  for (int i = 0; i < 3 && e == cudaSuccess; i++) e = cudaMemsetAsync(t->dB[i], 0, half * 16, st);
  float4 *tb[5] = {t->dA0, t->dA1, t->dmom, t->dhist, t->dmomp};
  for (int i = 0; i < 5 && e == cudaSuccess; i++) e = cudaMemsetAsync(tb[i], 0, full * 16, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(t->dag, 0, half * 8, st);
  if (t->coarse_pool) {
    const size_t quarter = (size_t)t->W4 * t->H4;
    if (e == cudaSuccess) e = cudaMemsetAsync(t->dah, 0, half * 16, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->dc1, 0, quarter * 16, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->dc0, 0, quarter * 16, st);
  }
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "cudaMemsetAsync");
}

static int run_twin_pass(hush_trainer_t *t, int pass, int backward, void *stream, const char *who) {
  if (!t) return hush_fail(nullptr, HUSH_ERR_ARG, std::string(who) + ": NULL trainer");
  if (pass < 0 || pass >= HUSH_TWIN_PASSES) return tr_fail(t, std::string(who) + ": unknown pass");
  if (!t->begun) return tr_fail(t, std::string(who) + ": no frame; call hush_trainer_begin first");
  cudaSetDevice(t->h->dev);
  cudaStream_t st = (cudaStream_t)stream;
  const TwinFrame &T = t->T;
  const HushFrame &f = T.f;
  const int full = f.W * f.H;
  const dim3 blk(TW, TH), gh((f.W2 + TW - 1) / TW, (f.H2 + TH - 1) / TH), gf((f.W + TW - 1) / TW, (f.H + TH - 1) / TH);
  cudaError_t e = cudaSuccess;
  switch (pass) {
    case HUSH_TWIN_MLP:
      if (!backward) launch_mlp_fwd(t, T, st);
      else launch_mlp_bwd(t, T, st);
      break;
    case HUSH_TWIN_MID1:
      if (backward) k_mid_bwd<1><<<gh, blk, 0, st>>>(T); else k_mid_fwd<1><<<gh, blk, 0, st>>>(T);
      break;
    case HUSH_TWIN_MID2:
      if (backward) k_mid_bwd<2><<<gh, blk, 0, st>>>(T); else k_mid_fwd<2><<<gh, blk, 0, st>>>(T);
      break;
    case HUSH_TWIN_MID3:
      if (backward) k_mid_bwd<3><<<gh, blk, 0, st>>>(T); else k_mid_fwd<3><<<gh, blk, 0, st>>>(T);
      break;
    case HUSH_TWIN_FINE:
      if (backward) {  // per pass: the history seed dA1 and the input gradient dA0 as well
        TwinFrame Tb = T;
        Tb.gA1 = t->dA1;
        Tb.dA0 = t->dA0;
        k_fine_bwd<false><<<gf, blk, 0, st>>>(Tb, t->dX);
      } else {
        k_fine_fwd<<<gf, blk, 0, st>>>(T);
      }
      break;
    case HUSH_TWIN_TEMPORAL:
      if (backward) k_temporal_bwd<<<gf, blk, 0, st>>>(T, t->dA0, t->dmom, t->dhist, t->dmomp, t->dag);
      else e = launch_pass(PASS_TEMPORAL, f, t->h->w16, st);
      break;
    case HUSH_TWIN_TAA:
      if (!backward) {
        k_taa_fwd<<<gf, blk, 0, st>>>(T);
      } else {
        k_taa_bwd_coef<<<gf, blk, 0, st>>>(T, t->gT, t->tcoef);
        k_taa_bwd_gather<<<gf, blk, 0, st>>>(T, t->tcoef, t->gT2);
        k_tm_bwd<<<(full + 255) / 256, 256, 0, st>>>(T, t->gT2, t->dX);
      }
      break;
    case HUSH_TWIN_COARSE1:
    case HUSH_TWIN_COARSE2: {
      const dim3 gq((t->W4 + TW - 1) / TW, (t->H4 + TH - 1) / TH);
      if (pass == HUSH_TWIN_COARSE2) {
        if (backward) k_coarse_tw<2><<<gq, blk, 0, st>>>(T, t->c1, nullptr, t->dc0, t->dc1);
        else k_coarse_tw<2><<<gq, blk, 0, st>>>(T, t->c1, t->c0, nullptr, nullptr);
      } else if (!backward) {
        k_coarse_tw<1><<<gq, blk, 0, st>>>(T, t->ah, t->c1, nullptr, nullptr);
      } else {  // dc1 -> down()'s quarter-res gradient -> the block means
        e = cudaMemsetAsync(t->ddown, 0, (size_t)t->W4 * t->H4 * 16, st);
        if (e == cudaSuccess) k_coarse_tw<1><<<gq, blk, 0, st>>>(T, t->ah, nullptr, t->dc1, t->ddown);
        const int half = t->W2 * t->H2;
        if (e == cudaSuccess) k_down_bwd<<<(half + 255) / 256, 256, 0, st>>>(T, t->ah, t->ddown, t->dah);
      }
      break;
    }
    default:  // HUSH_TWIN_LOSS
      k_loss<<<t->n_loss_ctas, 256, 0, st>>>(T, backward);
      k_reduce_f64<<<1, 256, 0, st>>>(t->loss_partials, t->n_loss_ctas, t->loss, nullptr);
      break;
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, (std::string(who) + ": kernel launch").c_str());
}

extern "C" int hush_trainer_pass(hush_trainer_t *t, int pass, int backward, void *stream) {
  return run_twin_pass(t, pass, backward, stream, "hush_trainer_pass");
}
extern "C" int hush_mlp_fwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_MLP, 0, stream, "hush_mlp_fwd"); }
extern "C" int hush_mlp_bwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_MLP, 1, stream, "hush_mlp_bwd"); }
extern "C" int hush_mid1_fwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_MID1, 0, stream, "hush_mid1_fwd"); }
extern "C" int hush_mid1_bwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_MID1, 1, stream, "hush_mid1_bwd"); }
extern "C" int hush_mid2_fwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_MID2, 0, stream, "hush_mid2_fwd"); }
extern "C" int hush_mid2_bwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_MID2, 1, stream, "hush_mid2_bwd"); }
extern "C" int hush_mid3_fwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_MID3, 0, stream, "hush_mid3_fwd"); }
extern "C" int hush_mid3_bwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_MID3, 1, stream, "hush_mid3_bwd"); }
extern "C" int hush_fine_fwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_FINE, 0, stream, "hush_fine_fwd"); }
extern "C" int hush_fine_bwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_FINE, 1, stream, "hush_fine_bwd"); }
extern "C" int hush_taa_fwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_TAA, 0, stream, "hush_taa_fwd"); }
extern "C" int hush_taa_bwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_TAA, 1, stream, "hush_taa_bwd"); }
extern "C" int hush_loss_fwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_LOSS, 0, stream, "hush_loss_fwd"); }
extern "C" int hush_loss_bwd(hush_trainer_t *t, void *stream) { return run_twin_pass(t, HUSH_TWIN_LOSS, 1, stream, "hush_loss_bwd"); }
extern "C" int hush_temporal_fwd(hush_trainer_t *t, void *stream) {
  return run_twin_pass(t, HUSH_TWIN_TEMPORAL, 0, stream, "hush_temporal_fwd");
}
extern "C" int hush_temporal_bwd(hush_trainer_t *t, void *stream) {
  return run_twin_pass(t, HUSH_TWIN_TEMPORAL, 1, stream, "hush_temporal_bwd");
}
extern "C" int hush_coarse1_fwd(hush_trainer_t *t, void *stream) {
  return run_twin_pass(t, HUSH_TWIN_COARSE1, 0, stream, "hush_coarse1_fwd");
}
extern "C" int hush_coarse1_bwd(hush_trainer_t *t, void *stream) {
  return run_twin_pass(t, HUSH_TWIN_COARSE1, 1, stream, "hush_coarse1_bwd");
}
extern "C" int hush_coarse2_fwd(hush_trainer_t *t, void *stream) {
  return run_twin_pass(t, HUSH_TWIN_COARSE2, 0, stream, "hush_coarse2_fwd");
}
extern "C" int hush_coarse2_bwd(hush_trainer_t *t, void *stream) {
  return run_twin_pass(t, HUSH_TWIN_COARSE2, 1, stream, "hush_coarse2_bwd");
}

// ------------------------------------------------------------------------------------------------ window BPTT
// dpar's alpha / gamma (components 0, 1 of its first float4) += the gradient carried back from the next frame.
__global__ void k_add_ag(float4 *dpar, const float2 *ag, int n) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  const float2 g = ag[o];
  dpar[3 * o].x += g.x;
  dpar[3 * o].y += g.y;
}

// The state of each frame of a window that the reverse sweep reads again: TEMPORAL's outputs and key, the features,
// the coarse levels, the twin's stored history (colour, TAA, par0) and its FP32 TAA output (the next frame's temporal
// loss term). Allocated for the longest window seen.
static int ensure_records(hush_trainer_t *t, int n) {
  if ((int)t->rec.size() >= n) return HUSH_OK;
  const size_t full = (size_t)t->W * t->H, half = (size_t)t->W2 * t->H2;
  const size_t quarter = (size_t)((t->W2 + 1) / 2) * ((t->H2 + 1) / 2);
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t per = al(full * 8) * 5 + al(half * 8) + al(half * 16) * 4 + al(quarter * 8) * 3 + al(full * 16);
  drop_bptt_graph(t);  // it captured the old records' addresses
  cudaFree(t->rec_pool);
  t->rec.clear();
  cudaError_t e = cudaMalloc(&t->rec_pool, per * n);
  if (e != cudaSuccess) { t->rec_pool = nullptr; return hush_cuda_fail(t->h, e, "cudaMalloc of the window records"); }
  e = cudaMemset(t->rec_pool, 0, per * n);
  if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "cudaMemset of the window records");
  if (!t->carry_pool) {
    const size_t cb = al(full * 16) * 4 + al(half * 8) * 2;
    e = cudaMalloc(&t->carry_pool, cb);
    if (e != cudaSuccess) { t->carry_pool = nullptr; return hush_cuda_fail(t->h, e, "cudaMalloc of the carries"); }
    char *c = t->carry_pool;
    for (int k = 0; k < 2; k++) { t->c_hist[k] = (float4 *)c; c += al(full * 16); }
    for (int k = 0; k < 2; k++) { t->c_mom[k] = (float4 *)c; c += al(full * 16); }
    for (int k = 0; k < 2; k++) { t->c_ag[k] = (float2 *)c; c += al(half * 8); }
  }
  char *b = t->rec_pool;
  for (int i = 0; i < n; i++) {
    hush_trainer_t::Rec r;
    auto take = [&](size_t sz) { char *q = b; b += al(sz); return q; };
    r.A0 = (uint2 *)take(full * 8); r.key = (uint2 *)take(full * 8); r.mom = (uint2 *)take(full * 8);
    r.hist = (uint2 *)take(full * 8); r.taa = (uint2 *)take(full * 8); r.par0 = (uint2 *)take(half * 8);
    for (int k = 0; k < 4; k++) r.F[k] = (uint4 *)take(half * 16);
    r.C0 = (uint2 *)take(quarter * 8); r.C1 = (uint2 *)take(quarter * 8); r.CG = (uint2 *)take(quarter * 8);
    r.out = (float4 *)take(full * 16);
    t->rec.push_back(r);
  }
  return HUSH_OK;
}

// The twin frame of window frame i, its state in record i and its history in record i - 1 (frame 0: a reset).
static TwinFrame rec_twin(hush_trainer_t *t, const hush_inputs *in, const float *clean, const float *clean_prev, int i,
                          float lambda_t) {
  TwinFrame T = make_twin(t, in, clean, clean_prev, lambda_t);
  const hush_trainer_t::Rec &r = t->rec[i], &p = t->rec[i > 0 ? i - 1 : 0];
  HushFrame &f = T.f;
  f.reset = i == 0 ? 1 : 0;
  f.A0 = r.A0; f.key = r.key; f.mom = r.mom; f.hist = r.hist; f.taa = r.taa; f.par0 = r.par0;
  f.F0 = r.F[0]; f.F1 = r.F[1]; f.F2 = r.F[2]; f.F3 = r.F[3];
  f.C0 = r.C0; f.C1 = r.C1; f.CG = r.CG;
  f.key_prev = p.key; f.hist_prev = p.hist; f.mom_prev = p.mom; f.par0_prev = p.par0; f.taa_prev = p.taa;
  T.out = r.out;
  T.out_prev = p.out;
  T.has_prev = (i > 0 && clean_prev) ? 1 : 0;
  return T;
}

// Backpropagation through time over one window (see include/hush.h): forward over the frames, keeping each frame's
// state, then the reverse sweep, frame by frame from the last: the twin's forward again, the loss, TAA, fine (seeded
// with the gradient the next frame sent to this frame's colour history, and giving dL/dA0 and, from the second frame
// on, dL/d block means and dL/dC0), mid3..mid1 (mid1 adding into dL/d block means), the MLP (whose alpha / gamma
// seeds are the gradient the next frame sent to this frame's par0), the coarse levels' adjoints (C0 -> C1 -> down()
// -> block means) and the block means into A0, then TEMPORAL's adjoint, which sends this frame's gradient to the
// previous frame's colour history, moments and alpha / gamma.
static cudaError_t bptt_launches(hush_trainer_t *t, const hush_inputs *frames, const float *const *cleans,
                                 int n_frames, float lambda_t, cudaStream_t st);
extern "C" int hush_trainer_window_bptt(hush_trainer_t *t, const hush_inputs *frames, const float *const *cleans,
                                        int n_frames, float lambda_t, void *stream) {
  if (!t || !frames || !cleans)
    return hush_fail(t ? t->h : nullptr, HUSH_ERR_ARG, "hush_trainer_window_bptt: NULL argument");
  if (n_frames < 1) return tr_fail(t, "hush_trainer_window_bptt: empty window");
  if (t->W != t->h->W || t->H != t->h->H)
    return tr_fail(t, "hush_trainer_window_bptt: the denoiser was resized after the trainer was created");
  for (int i = 0; i < n_frames; i++) {
    if (!cleans[i]) return tr_fail(t, "hush_trainer_window_bptt: missing clean image");
    const int rc = hush_check_inputs(t->h, frames + i);
    if (rc != HUSH_OK) return rc;
  }
  cudaSetDevice(t->h->dev);
  int rc = ensure_records(t, n_frames);
  if (rc != HUSH_OK) return rc;
  cudaError_t e = ensure_coarse(t);  // the coarse levels' adjoint buffers
  if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "cudaMalloc of the coarse-level buffers");
  e = bptt_launches(t, frames, cleans, n_frames, lambda_t, (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(t->h, e, "hush_trainer_window_bptt");
}

// The launches of one window through time on `st` (inputs checked, records allocated); no host state changes, so a
// capture of them replays for every window whose inputs sit at the same addresses.
static cudaError_t bptt_launches(hush_trainer_t *t, const hush_inputs *frames, const float *const *cleans,
                                 int n_frames, float lambda_t, cudaStream_t st) {
  const int W = t->W, H = t->H, W2 = t->W2, H2 = t->H2;
  const size_t full = (size_t)W * H, half = (size_t)W2 * H2, quarter = (size_t)t->W4 * t->H4;
  const dim3 blk(TW, TH), gh((W2 + TW - 1) / TW, (H2 + TH - 1) / TH), gf((W + TW - 1) / TW, (H + TH - 1) / TH);
  const dim3 gq((t->W4 + TW - 1) / TW, (t->H4 + TH - 1) / TH);
  auto twin = [&](int i) {
    return rec_twin(t, frames + i, cleans[i], i ? cleans[i - 1] : nullptr, i, lambda_t);
  };
  auto forward = [&](const TwinFrame &T) {
    launch_mlp_fwd(t, T, st);
    k_mid_fwd<1><<<gh, blk, 0, st>>>(T);
    k_mid_fwd<2><<<gh, blk, 0, st>>>(T);
    k_mid_fwd<3><<<gh, blk, 0, st>>>(T);
    k_fine_fwd<<<gf, blk, 0, st>>>(T);
    k_taa_fwd<<<gf, blk, 0, st>>>(T);
  };
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < n_frames && e == cudaSuccess; i++) {
    const TwinFrame T = twin(i);
    e = launch_pass(PASS_TEMPORAL, T.f, t->h->w16, st);
    if (e == cudaSuccess) e = launch_pass(PASS_COARSE1, T.f, t->h->w16, st);
    if (e == cudaSuccess) e = launch_pass(PASS_COARSE2, T.f, t->h->w16, st);
    if (e != cudaSuccess) break;
    forward(T);
    k_loss<<<t->n_loss_ctas, 256, 0, st>>>(T, 0);
    k_reduce_f64<<<1, 256, 0, st>>>(t->loss_partials, t->n_loss_ctas, t->loss, t->loss_acc);
  }
  int c = 0;
  for (int k = 0; k < 2 && e == cudaSuccess; k++) {
    e = cudaMemsetAsync(t->c_hist[k], 0, full * 16, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->c_mom[k], 0, full * 16, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->c_ag[k], 0, half * 8, st);
  }
  for (int i = n_frames - 1; i >= 0 && e == cudaSuccess; i--) {
    TwinFrame T = twin(i);
    T.zero_adj = 1;
    forward(T);
    k_loss<<<t->n_loss_ctas, 256, 0, st>>>(T, 1);
    k_add_ag<<<(unsigned)((half + 255) / 256), 256, 0, st>>>(t->dpar, t->c_ag[c], (int)half);
    k_taa_bwd_coef<<<gf, blk, 0, st>>>(T, t->gT, t->tcoef);
    k_taa_bwd_gather<<<gf, blk, 0, st>>>(T, t->tcoef, t->gT2);
    e = cudaMemsetAsync(t->dA0, 0, full * 16, st);
    if (e == cudaSuccess && i > 0) e = cudaMemsetAsync(t->dah, 0, half * 16, st);
    if (e == cudaSuccess && i > 0) e = cudaMemsetAsync(t->dc0, 0, quarter * 16, st);
    if (e != cudaSuccess) break;
    T.gA1 = t->c_hist[c];
    T.dA0 = t->dA0;
    if (i > 0) {  // A0 reaches the loss also through the block means (mid1, the recombination, the coarse levels)
      T.dAh = t->dah;
      T.dC0 = t->dc0;
    }
    k_fine_bwd<true><<<gf, blk, 0, st>>>(T, t->gT2);
    if (i > 0) k_fine_pyr_bwd<true><<<gf, blk, 0, st>>>(T, t->gT2);
    k_mid_bwd<3><<<gh, blk, 0, st>>>(T);
    k_mid_bwd<2><<<gh, blk, 0, st>>>(T);
    k_mid_bwd<1><<<gh, blk, 0, st>>>(T);
    launch_mlp_bwd(t, T, st);
    if (i > 0) {
      // the coarse levels' adjoints (C0 -> C1 -> down() -> block means), then the block means into A0
      k_ah_fill<<<(unsigned)((half + 255) / 256), 256, 0, st>>>(T, t->ah);
      k_c1_fill<<<(unsigned)((quarter + 255) / 256), 256, 0, st>>>(T, t->c1);
      e = cudaMemsetAsync(t->dc1, 0, quarter * 16, st);
      if (e == cudaSuccess) e = cudaMemsetAsync(t->ddown, 0, quarter * 16, st);
      if (e != cudaSuccess) break;
      k_coarse_tw<2><<<gq, blk, 0, st>>>(T, t->c1, nullptr, t->dc0, t->dc1);
      k_coarse_tw<1><<<gq, blk, 0, st>>>(T, t->ah, nullptr, t->dc1, t->ddown);
      k_down_bwd<<<(unsigned)((half + 255) / 256), 256, 0, st>>>(T, t->ah, t->ddown, t->dah);
      k_ah_to_a0<<<(unsigned)((full + 255) / 256), 256, 0, st>>>(T, t->dah, t->dA0);
      const int n = c ^ 1;
      e = cudaMemsetAsync(t->c_hist[n], 0, full * 16, st);
      if (e == cudaSuccess) e = cudaMemsetAsync(t->c_mom[n], 0, full * 16, st);
      if (e == cudaSuccess) e = cudaMemsetAsync(t->c_ag[n], 0, half * 8, st);
      if (e != cudaSuccess) break;
      k_temporal_bwd<<<gf, blk, 0, st>>>(T, t->dA0, t->c_mom[c], t->c_hist[n], t->c_mom[n], t->c_ag[n]);
      c = n;
    }
  }
  return e;
}

// The windows seeds[0], seeds[stride], ... through time, in order on one trainer and stream: each window generated
// into win_pool on `st`, then its forward + reverse sweep (bptt_launches) replayed as one CUDA graph, captured at the
// first window and kept while the frame count, lambda, the exposure and the MLP form stay the same (the buffers it
// names are the trainer's and stay put; reallocating them drops it). Where capture is not possible the launches run
// directly.
static int windows_serial_bptt(hush_trainer_t *t, const hush_scene *sc, const uint32_t *seeds, int n_windows,
                               int stride, int n_frames, float lambda_t, cudaStream_t st) {
  size_t img = 0, per = 0;
  int rc = ensure_win_pool(t, n_frames, img, per);
  if (rc == HUSH_OK) rc = ensure_records(t, n_frames);
  if (rc != HUSH_OK) return rc;
  const cudaError_t ec = ensure_coarse(t);  // the coarse levels' adjoint buffers
  if (ec != cudaSuccess) return hush_cuda_fail(t->h, ec, "cudaMalloc of the coarse-level buffers");
  if (t->bg_frames != n_frames || t->bg_lambda != lambda_t || t->bg_exposure != t->h->exposure ||
      t->bg_mode != t->mlp_mode) {
    drop_bptt_graph(t);
    t->bg_frames = n_frames;
    t->bg_lambda = lambda_t;
    t->bg_exposure = t->h->exposure;
    t->bg_mode = t->mlp_mode;
  }
  if (!t->cap) {
    cudaError_t e = cudaStreamCreateWithFlags(&t->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "cudaStreamCreate");
  }
  std::vector<hush_inputs> in(n_frames);
  std::vector<const float *> cl(n_frames);
  for (int i = 0; i < n_frames; i++) {
    char *b = t->win_pool + per * i;
    std::memset(&in[i], 0, sizeof(hush_inputs));
    in[i].radiance = b; in[i].normal_depth = b + img; in[i].motion = b + 2 * img; in[i].material = b + 3 * img;
    in[i].emission = b + 4 * img;
    cl[i] = (const float *)(b + 5 * img);
  }
  for (int k = 0; k < n_windows; k += stride) {
    rc = generate_window(t, sc, seeds[k], n_frames, img, per, st);
    if (rc != HUSH_OK) return rc;
    if (!t->bptt_graph) {  // capture on the trainer's own stream (the caller's may be the legacy default stream)
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamBeginCapture(t->cap, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        const cudaError_t el = bptt_launches(t, in.data(), cl.data(), n_frames, lambda_t, t->cap);
        e = cudaStreamEndCapture(t->cap, &graph);
        if (e == cudaSuccess && el != cudaSuccess) e = el;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&t->bptt_graph, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) {  // capture not possible here: run the launches directly
        cudaGetLastError();
        drop_bptt_graph(t);
        e = bptt_launches(t, in.data(), cl.data(), n_frames, lambda_t, st);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "hush_trainer_windows_bptt");
        continue;
      }
    }
    const cudaError_t e = cudaGraphLaunch(t->bptt_graph, st);
    if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "cudaGraphLaunch of a window through time");
  }
  return HUSH_OK;
}

extern "C" int hush_trainer_windows_bptt(hush_trainer_t *t, const hush_scene *sc, const uint32_t *seeds,
                                         int n_windows, int n_frames, float lambda_t, void *stream) {
  return run_windows(t, sc, seeds, n_windows, n_frames, lambda_t, stream, true, "hush_trainer_windows_bptt");
}

extern "C" int hush_trainer_buffer(hush_trainer_t *t, int which, void **ptr, int *width, int *height, int *channels) {
  if (!t || !ptr) return hush_fail(t ? t->h : nullptr, HUSH_ERR_ARG, "hush_trainer_buffer: NULL argument");
  void *p = nullptr;
  int w = t->W, h = t->H, c = 4;
  switch (which) {
    case HUSH_TB_THETA: p = t->theta; w = NW; h = 1; c = 1; break;
    case HUSH_TB_GRAD: p = t->grad; w = NW; h = 1; c = 1; break;
    case HUSH_TB_LOSS: p = t->loss; w = 1; h = 1; c = 1; break;
    case HUSH_TB_PAR: p = t->par; w = t->W2; h = t->H2; c = 12; break;
    case HUSH_TB_DPAR: p = t->dpar; w = t->W2; h = t->H2; c = 12; break;
    case HUSH_TB_B1: case HUSH_TB_B2: case HUSH_TB_B3:
      p = t->B[which - HUSH_TB_B1]; w = t->W2; h = t->H2; break;
    case HUSH_TB_DB1: case HUSH_TB_DB2: case HUSH_TB_DB3:
      p = t->dB[which - HUSH_TB_DB1]; w = t->W2; h = t->H2; break;
    case HUSH_TB_A1: p = t->A1; break;
    case HUSH_TB_X: p = t->X; break;
    case HUSH_TB_DX: p = t->dX; break;
    case HUSH_TB_OUT: p = t->out[t->cur]; break;
    case HUSH_TB_OUT_PREV: p = t->out[t->cur ^ 1]; break;
    case HUSH_TB_DOUT: p = t->gT; break;
    case HUSH_TB_DA0: p = t->dA0; break;
    case HUSH_TB_DA1: p = t->dA1; break;
    case HUSH_TB_DMOM: p = t->dmom; break;
    case HUSH_TB_DHIST: p = t->dhist; break;
    case HUSH_TB_DMOM_PREV: p = t->dmomp; break;
    case HUSH_TB_DAG: p = t->dag; w = t->W2; h = t->H2; c = 2; break;
    case HUSH_TB_AH: case HUSH_TB_DAH: case HUSH_TB_C1: case HUSH_TB_DC1: case HUSH_TB_C0: case HUSH_TB_DC0: {
      const cudaError_t e = ensure_coarse(t);
      if (e != cudaSuccess) return hush_cuda_fail(t->h, e, "hush_trainer_buffer: coarse buffers");
      float4 *q[6] = {t->ah, t->dah, t->c1, t->dc1, t->c0, t->dc0};
      p = q[which - HUSH_TB_AH];
      w = which <= HUSH_TB_DAH ? t->W2 : t->W4;
      h = which <= HUSH_TB_DAH ? t->H2 : t->H4;
      break;
    }
    default: return tr_fail(t, "hush_trainer_buffer: unknown buffer");
  }
  *ptr = p;
  if (width) *width = w;
  if (height) *height = h;
  if (channels) *channels = c;
  return HUSH_OK;
}

// One optimiser step over a batch of windows, as the training loop runs it on one GPU: per window a history reset,
// then every frame forward and backward (the temporal term from the window's second frame on) and end-of-frame; then
// Adam on the summed gradient.
extern "C" int hush_train_step(hush_trainer_t *t, const hush_inputs *frames, const float *const *cleans, int n_windows,
                               int n_frames, float lambda_t, float lr, float beta1, float beta2, float eps, float clip,
                               void *stream, double *loss_mean, double *grad_norm) {
  if (!t || !frames || !cleans) return hush_fail(t ? t->h : nullptr, HUSH_ERR_ARG, "hush_train_step: NULL argument");
  if (n_windows < 1 || n_frames < 1) return tr_fail(t, "hush_train_step: empty batch");
  double s = 0.0;
  int rc = hush_trainer_loss_sum(t, stream, &s);  // restart the loss sum
  for (int w = 0; w < n_windows && rc == HUSH_OK; w++) {
    rc = hush_trainer_reset(t);
    for (int i = 0; i < n_frames && rc == HUSH_OK; i++) {
      const size_t k = (size_t)w * n_frames + i;
      rc = hush_trainer_frame(t, frames + k, cleans[k], i ? cleans[k - 1] : nullptr, lambda_t, 1, stream, nullptr);
      if (rc == HUSH_OK) rc = hush_trainer_end_frame(t);
    }
  }
  if (rc == HUSH_OK) rc = hush_trainer_loss_sum(t, stream, &s);
  if (rc != HUSH_OK) return rc;
  if (loss_mean) *loss_mean = s / ((double)n_windows * n_frames);
  return hush_trainer_step(t, lr, beta1, beta2, eps, clip, stream, grad_norm);
}

// ------------------------------------------------------------------------------------------------ no-allocation
// MLP weight gradient for callers that cannot allocate device memory: the same per-row adjoint as k_mlp_bwd, with
// its per-CTA partial sums in a fixed file-scope device array instead of trainer-owned scratch. Some hosts forbid
// device allocation after start-up (a render or training loop with a fixed memory budget, where cudaMalloc would
// synchronise the device or fail under memory pressure mid-frame) or only lend the library buffers they own (an
// engine or a browser GPU process that manages all device memory itself). The array is allocated when the library
// is loaded, on every GPU that loads it, and stays until the process exits.
namespace hush {
namespace twin {

constexpr int NA_ROWS = 64;                 // rows per chunk (one thread per row)
constexpr int NA_MAX_CTAS = 512;            // CTAs, hence partial sums, at most
constexpr long NA_MAX_ROWS = 16L << 20;     // 16,777,216 rows: a 4096 x 4096 half-resolution image

// 512 partial sums x 812 doubles = 3.33 MB, shared by every call on the device.
static __device__ __align__(256) double g_noalloc_partials[NA_MAX_CTAS * NW];

// Grid-stride over chunks of NA_ROWS rows; each CTA keeps its parameter sums in registers (thread t owns parameters
// t, t + 64, ...) and writes them once to partials[blockIdx.x]: every slot the reduction reads is overwritten first,
// so nothing has to start at zero. A chunk's 64 rows are summed in FP32 (as the trainer sums its 128-row CTAs), the
// chunks of a CTA in FP64, so the error does not grow with the number of chunks a CTA takes.
__global__ void __launch_bounds__(NA_ROWS) k_mlp_grad_noalloc(const uint4 *F0, const uint4 *F1, const uint4 *F2,
                                                              const uint4 *F3, const float4 *dpar, const float *theta,
                                                              int rows, double *partials) {
  __shared__ float th[NW];
  __shared__ float sd3[12][NA_ROWS], sd2[16][NA_ROWS], sd1[16][NA_ROWS], sf[20][NA_ROWS], sh1[16][NA_ROWS],
      sh2[16][NA_ROWS];
  for (int i = threadIdx.x; i < NW; i += NA_ROWS) th[i] = theta[i];
  constexpr int PER = (NW + NA_ROWS - 1) / NA_ROWS;  // 13 parameters per thread
  double acc[PER];
#pragma unroll
  for (int k = 0; k < PER; k++) acc[k] = 0.0;
  HushFrame f;
  f.F0 = const_cast<uint4 *>(F0); f.F1 = const_cast<uint4 *>(F1); f.F2 = const_cast<uint4 *>(F2);
  __syncthreads();
  const int nchunks = (rows + NA_ROWS - 1) / NA_ROWS;
  for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
    const int r = threadIdx.x, o = chunk * NA_ROWS + r;
    float fe[20], h1[16], h2[16], out[12], d3[12], d2[16], d1[16];
#pragma unroll
    for (int i = 0; i < 20; i++) fe[i] = 0.f;
#pragma unroll
    for (int i = 0; i < 16; i++) h1[i] = h2[i] = d2[i] = d1[i] = 0.f;
#pragma unroll
    for (int i = 0; i < 12; i++) d3[i] = 0.f;
    if (o < rows && f3_guide_tw(F3, o).w >= 0.0f) {
      load_features(f, o, fe);
      mlp_full(th, fe, h1, h2, out);
      const float4 q0 = dpar[3 * o], q1 = dpar[3 * o + 1], q2 = dpar[3 * o + 2];
      float4 p0, p1, p2;
      mlp_heads(out, p0, p1, p2);
      // the heads' adjoint as k_mlp_bwd forms it, alpha and gamma seeds included
      const float sa = sigmoidf_(out[0]), sg = sigmoidf_(out[1]);
      d3[0] = q0.x * (31.0f / 32.0f) * sa * (1.0f - sa);
      d3[1] = q0.y * 7.5f * sg * (1.0f - sg);
      d3[2] = q0.z * p0.z * (1.0f - p0.z);
      d3[3] = q0.w * p0.w * (1.0f - p0.w);
      const float ps[4] = {p1.x, p1.y, p1.z, p1.w}, pc[4] = {p2.x, p2.y, p2.z, p2.w};
      const float gs[4] = {q1.x, q1.y, q1.z, q1.w}, gc[4] = {q2.x, q2.y, q2.z, q2.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        d3[4 + k] = fabsf(out[4 + k]) < 5.0f ? gs[k] * ps[k] : 0.0f;
        d3[8 + k] = fabsf(out[8 + k]) < 4.0f ? gc[k] * pc[k] : 0.0f;
      }
#pragma unroll
      for (int i = 0; i < 16; i++) {
        float a = 0.f;
#pragma unroll
        for (int j = 0; j < 12; j++) a += d3[j] * th[W3o + j * 16 + i];
        d2[i] = h2[i] > 0.0f ? a : 0.0f;
      }
#pragma unroll
      for (int i = 0; i < 16; i++) {
        float a = 0.f;
#pragma unroll
        for (int j = 0; j < 16; j++) a += d2[j] * th[W2o + j * 16 + i];
        d1[i] = h1[i] > 0.0f ? a : 0.0f;
      }
    }
#pragma unroll
    for (int i = 0; i < 12; i++) sd3[i][r] = d3[i];
#pragma unroll
    for (int i = 0; i < 16; i++) { sd2[i][r] = d2[i]; sd1[i][r] = d1[i]; sh1[i][r] = h1[i]; sh2[i][r] = h2[i]; }
#pragma unroll
    for (int i = 0; i < 20; i++) sf[i][r] = fe[i];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int p = threadIdx.x + k * NA_ROWS;
      if (p >= NW) continue;
      const float *dv, *xv = nullptr;
      if (p < B1o) { dv = sd1[p / 20]; xv = sf[p % 20]; }
      else if (p < W2o) { dv = sd1[p - B1o]; }
      else if (p < B2o) { const int q = p - W2o; dv = sd2[q / 16]; xv = sh1[q % 16]; }
      else if (p < W3o) { dv = sd2[p - B2o]; }
      else if (p < B3o) { const int q = p - W3o; dv = sd3[q / 16]; xv = sh2[q % 16]; }
      else { dv = sd3[p - B3o]; }
      float a = 0.f;
      if (xv) for (int j = 0; j < NA_ROWS; j++) a += dv[j] * xv[j];
      else for (int j = 0; j < NA_ROWS; j++) a += dv[j];
      acc[k] += (double)a;
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < PER; k++) {
    const int p = threadIdx.x + k * NA_ROWS;
    if (p < NW) partials[(size_t)blockIdx.x * NW + p] = acc[k];
  }
}

// dtheta = sum over the grid's partials, in FP64 (overwrites dtheta)
__global__ void k_mlp_grad_noalloc_reduce(const double *partials, int nparts, double *dtheta) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NW) return;
  double a = 0.0;
  for (int c = 0; c < nparts; c++) a += partials[(size_t)c * NW + p];
  dtheta[p] = a;
}

}  // namespace twin
}  // namespace hush

#include <mutex>

// Host-side address of g_noalloc_partials per device: the symbol's name in host code is only a stand-in, so the
// device address is looked up once per device (with that device current) and cached.
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[64] = {};

extern "C" int hush_mlp_grad_noalloc(const void *F0, const void *F1, const void *F2, const void *F3,
                                     const float *dpar, const float *theta, int width2, int height2, double *dtheta,
                                     void *stream) {
  using namespace hush::twin;
  if (!F0 || !F1 || !F2 || !F3 || !dpar || !theta || !dtheta)
    return hush_fail(nullptr, HUSH_ERR_ARG, "hush_mlp_grad_noalloc: NULL argument");
  if (width2 <= 0 || height2 <= 0)
    return hush_fail(nullptr, HUSH_ERR_ARG, "hush_mlp_grad_noalloc: bad size " + std::to_string(width2) + "x" +
                                                std::to_string(height2));
  const long rows = (long)width2 * (long)height2;
  if (rows > NA_MAX_ROWS)
    return hush_fail(nullptr, HUSH_ERR_ARG,
                     "hush_mlp_grad_noalloc: " + std::to_string(rows) + " rows exceed the maximum of " +
                         std::to_string(NA_MAX_ROWS) + " (the fixed scratch holds " + std::to_string(NA_MAX_CTAS) +
                         " partial sums)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return hush_cuda_fail(nullptr, e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_mlp_grad_noalloc: device ordinal >= 64");
  double *partials = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_partials);
      if (e != cudaSuccess) return hush_cuda_fail(nullptr, e, "cudaGetSymbolAddress of the fixed scratch");
      g_noalloc_ptr[dev] = (double *)p;
    }
    partials = g_noalloc_ptr[dev];
  }
  const int nchunks = (int)((rows + NA_ROWS - 1) / NA_ROWS);
  const int grid = nchunks < NA_MAX_CTAS ? nchunks : NA_MAX_CTAS;
  cudaStream_t st = (cudaStream_t)stream;
  k_mlp_grad_noalloc<<<grid, NA_ROWS, 0, st>>>((const uint4 *)F0, (const uint4 *)F1, (const uint4 *)F2,
                                               (const uint4 *)F3, (const float4 *)dpar, theta, (int)rows, partials);
  k_mlp_grad_noalloc_reduce<<<(NW + 127) / 128, 128, 0, st>>>(partials, grid, dtheta);
  e = cudaGetLastError();
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(nullptr, e, "hush_mlp_grad_noalloc launch");
}
