// Per-pixel device functions of the Hush passes. Each mirrors one WGSL function of the reference
// (src/denoise/hush.js) with its operation order; the kernels around them decide the tiling and fusion.
#pragma once
#include "common.cuh"

namespace hush {

// Everything one frame's kernels need: sizes, borrowed inputs (row pitch in texels), the previous frame's history
// and this frame's outputs. Internal images are dense (pitch = their width).
struct HushFrame {
  int W, H, W2, H2, W4, H4;
  int reset;        // flags bit 1 of the reference uniform (hush.js:827)
  float exposure;
  const uint2 *rad, *nd, *mv, *mat, *emi;
  int p_rad, p_nd, p_mv, p_mat, p_emi;
  const uint2 *key_prev, *hist_prev, *mom_prev, *par0_prev, *taa_prev;
  uint2 *A0, *X, *mom, *key, *hist, *taa, *par0, *par1, *par2, *Bh0, *Bh1, *C0, *C1, *CG;
  uint4 *F0, *F1, *F2, *F3;
  // half-res planes of the fused path: block means (F2.zw) and guide (F3.xy) as rgba16float, and the guides decoded
  // once by their producer as f32 (normal, depth): Gd at half, CGd at quarter resolution
  uint2 *Ah, *Gh;
  float4 *Gd, *CGd;
  const float *w_glob;  // decoded f32 weights in device memory (any hidden width)
  int hidden;
  int mlp_half;         // the reference's `f16` option: INFER's MLP in f16 arithmetic (mlp_fwd_half)
  unsigned int *err;    // device error word (bounded waits in the tensor-core MLP)
};

// Weights of the shipped width (h = 16) passed by value: kernel parameters live in the constant bank, so every
// thread of a warp reads the same weight in one broadcast (the reference bakes them in as WGSL literals, hush.js:750).
constexpr int H16_COUNT = 16 * 16 + 34 * 16 + 12;  // 812
struct MlpW16 {
  float w[H16_COUNT];
};

// ------------------------------------------------------------------------------------------------ MLP
// mlpCode (hush.js:683-704): per output, bias + sum_i input_i * w_i in increasing i; ReLU on the hidden layers.
template <int HD>
HD_INL void mlp_fwd(const float *__restrict__ w, const float *f, float *o) {
  constexpr int W1 = 0, B1 = HD * N_FEAT, W2 = B1 + HD, B2 = W2 + HD * HD, W3 = B2 + HD, B3 = W3 + N_OUT * HD;
  float h1[HD], h2[HD];
#pragma unroll
  for (int j = 0; j < HD; j++) {
    float a = w[B1 + j];
#pragma unroll
    for (int i = 0; i < N_FEAT; i++) a = a + f[i] * w[W1 + j * N_FEAT + i];
    h1[j] = fmaxf(a, 0.0f);
  }
#pragma unroll
  for (int j = 0; j < HD; j++) {
    float a = w[B2 + j];
#pragma unroll
    for (int i = 0; i < HD; i++) a = a + h1[i] * w[W2 + j * HD + i];
    h2[j] = fmaxf(a, 0.0f);
  }
#pragma unroll
  for (int j = 0; j < N_OUT; j++) {
    float a = w[B3 + j];
#pragma unroll
    for (int i = 0; i < HD; i++) a = a + h2[i] * w[W3 + j * HD + i];
    o[j] = a;
  }
}

// Any hidden width, weights in global memory.
HD_INL void mlp_fwd_dyn(const float *__restrict__ w, int hd, const float *f, float *o) {
  const int W1 = 0, B1 = hd * N_FEAT, W2 = B1 + hd, B2 = W2 + hd * hd, W3 = B2 + hd, B3 = W3 + N_OUT * hd;
  float h1[256];
  for (int j = 0; j < hd; j++) {
    float a = __ldg(w + B1 + j);
    for (int i = 0; i < N_FEAT; i++) a = a + f[i] * __ldg(w + W1 + j * N_FEAT + i);
    h1[j] = fmaxf(a, 0.0f);
  }
  float h2[256];
  for (int j = 0; j < hd; j++) {
    float a = __ldg(w + B2 + j);
    for (int i = 0; i < hd; i++) a = a + h1[i] * __ldg(w + W2 + j * hd + i);
    h2[j] = fmaxf(a, 0.0f);
  }
  for (int j = 0; j < N_OUT; j++) {
    float a = __ldg(w + B3 + j);
    for (int i = 0; i < hd; i++) a = a + h2[i] * __ldg(w + W3 + j * hd + i);
    o[j] = a;
  }
}

// mlpCode with f16 = true (hush.js:683-703, chosen by the `f16` option at hush.js:740, 750): inputs, weights and
// biases are f16 values; every product input * weight and every running sum bias + p0 + p1 + ... is rounded to f16
// (round to nearest even) in that left-to-right order, ReLU is max(., 0h), and the outputs widen to f32. Two units per
// f16x2 instruction; `mul.rn` / `add.rn` carry an explicit rounding mode, so they are never contracted into an FMA.
HD_INL uint32_t hmul2_rn(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("mul.rn.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
HD_INL uint32_t hadd2_rn(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("add.rn.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
HD_INL uint32_t hrelu2(uint32_t a) {  // max(a, 0) per half; a NaN half gives 0
  uint32_t r;
  asm("max.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(0u));
  return r;
}
HD_INL uint32_t h2pack(float a, float b) {  // (a, b) as f16 bits, low half first
  return (uint32_t)__half_as_ushort(__float2half_rn(a)) | ((uint32_t)__half_as_ushort(__float2half_rn(b)) << 16);
}
HD_INL uint32_t hdup(uint32_t h16) { return (h16 & 0xffffu) * 0x10001u; }
HD_INL float hlo(uint32_t a) { return __half2float(__ushort_as_half((uint16_t)(a & 0xffffu))); }
HD_INL float hhi(uint32_t a) { return __half2float(__ushort_as_half((uint16_t)(a >> 16))); }

// One f16 layer from decoded f32 weights (row-major (out, in)); in / out hold f16 bits per unit.
HD_INL void mlp_layer_half(const float *__restrict__ w, int wo, int bo, int nin, int nout, const uint16_t *in,
                           bool relu, uint16_t *out) {
  for (int j = 0; j < nout; j += 2) {
    const bool two = j + 1 < nout;
    uint32_t a = h2pack(w[bo + j], two ? w[bo + j + 1] : 0.0f);
    for (int i = 0; i < nin; i++)
      a = hadd2_rn(a, hmul2_rn(hdup(in[i]), h2pack(w[wo + j * nin + i], two ? w[wo + (j + 1) * nin + i] : 0.0f)));
    if (relu) a = hrelu2(a);
    out[j] = (uint16_t)(a & 0xffffu);
    if (two) out[j + 1] = (uint16_t)(a >> 16);
  }
}
// Any hidden width (<= 256) from decoded weights, as the per-pass INFER runs it.
HD_INL void mlp_fwd_half(const float *__restrict__ w, int hd, const float *f, float *o) {
  const int W1 = 0, B1 = hd * N_FEAT, W2 = B1 + hd, B2 = W2 + hd * hd, W3 = B2 + hd, B3 = W3 + N_OUT * hd;
  uint16_t x[N_FEAT], h1[256], h2[256], oh[N_OUT];
  for (int i = 0; i < N_FEAT; i++) x[i] = __half_as_ushort(__float2half_rn(f[i]));
  mlp_layer_half(w, W1, B1, N_FEAT, hd, x, true, h1);
  mlp_layer_half(w, W2, B2, hd, hd, h1, true, h2);
  mlp_layer_half(w, W3, B3, hd, N_OUT, h2, false, oh);
  for (int j = 0; j < N_OUT; j++) o[j] = __half2float(__ushort_as_half(oh[j]));
}

// Output heads (hush.js:357-362): par0 = (alpha, gamma, beta, kappa), par1 = s, par2 = c.
HD_INL void mlp_heads(const float *o, float4 &p0, float4 &p1, float4 &p2) {
  p0.x = 1.0f / 32.0f + (31.0f / 32.0f) * sigmoidf_(o[0]);
  p0.y = 0.5f + 7.5f * sigmoidf_(o[1]);
  p0.z = sigmoidf_(o[2]);
  p0.w = sigmoidf_(o[3]);
  p1.x = 0.25f * expf(fminf(fmaxf(o[4], -5.0f), 5.0f));
  p1.y = 0.25f * expf(fminf(fmaxf(o[5], -5.0f), 5.0f));
  p1.z = 0.25f * expf(fminf(fmaxf(o[6], -5.0f), 5.0f));
  p1.w = 0.25f * expf(fminf(fmaxf(o[7], -5.0f), 5.0f));
  p2.x = expf(fminf(fmaxf(o[8], -4.0f), 4.0f));
  p2.y = expf(fminf(fmaxf(o[9], -4.0f), 4.0f));
  p2.z = expf(fminf(fmaxf(o[10], -4.0f), 4.0f));
  p2.w = expf(fminf(fmaxf(o[11], -4.0f), 4.0f));
}

// ------------------------------------------------------------------------------------------------ a-trous
// atrousFn (hush.js:431-476) over shared-memory tiles sA (colour, variance) and sG (decoded normal, depth) of row
// stride SW. (lx, ly) is the centre's tile position, (qx, qy) its image position, (w, h) the image size for the
// inside() test. The tiles hold clamp-to-edge loads. CHECK = false: the caller knows every tap lies inside the image
// (an interior tile), so the inside() test is always true and is left out.
template <int R, int STEP, bool PREF, int SW, bool CHECK = true>
HD_INL float4 filt(const float4 *sA, const float4 *sG, int lx, int ly, int qx, int qy, int w, int h, float s,
                   float c) {
  const int ti = ly * SW + lx;
  const float4 gp = sG[ti];
  const float4 center = sA[ti];
  float gv;
  if (PREF) {
    gv = 0.0625f * (sA[ti - SW - 1].w + sA[ti - SW + 1].w + sA[ti + SW - 1].w + sA[ti + SW + 1].w) +
         0.125f * (sA[ti - SW].w + sA[ti - 1].w + sA[ti + 1].w + sA[ti + SW].w) + 0.25f * center.w;
  } else {
    gv = center.w;
  }
  const float lc = lum(center);
  const float sl = s / (sqrtf(fmaxf(gv, 1e-12f)) + 1e-6f);
  const float zl = sG[ti - 1].w, zr = sG[ti + 1].w, zu = sG[ti - SW].w, zd = sG[ti + SW].w;
  const float gx = fminf(zr > 0.0f ? fabsf(zr - gp.w) : 1e9f, zl > 0.0f ? fabsf(zl - gp.w) : 1e9f);
  const float gy = fminf(zd > 0.0f ? fabsf(zd - gp.w) : 1e9f, zu > 0.0f ? fabsf(zu - gp.w) : 1e9f);
  const float zg = fminf(fmaxf(gx, gy), gp.w);
  // 1 / (zg * sqrt(d) * step + 1e-3) per distinct squared distance d (the literal is sqrt(d) * step as f32)
  float iz[9];
#pragma unroll
  for (int d = 1; d <= 2 * R * R; d++) {
    const float k = d == 1 ? 1.0f * STEP
                    : d == 2 ? 1.41421356237309515f * STEP
                    : d == 4 ? 2.0f * STEP
                    : d == 5 ? 2.23606797749978981f * STEP
                    : d == 8 ? 2.82842712474619029f * STEP
                             : 0.0f;
    iz[d] = 1.0f / (zg * k + 1e-3f);
  }
  constexpr float hc = R == 1 ? 0.5f : 0.375f;
  const float cw = (hc * hc) * c;
  float sw = cw;
  float scx = center.x * cw, scy = center.y * cw, scz = center.z * cw;
  float sv = center.w * cw * cw;
#pragma unroll
  for (int dy = -R; dy <= R; dy++) {
#pragma unroll
    for (int dx = -R; dx <= R; dx++) {
      if (dx == 0 && dy == 0) continue;
      const float hx = R == 1 ? (dx == 0 ? 0.5f : 0.25f) : (dx == 0 ? 0.375f : (dx == 1 || dx == -1) ? 0.25f : 0.0625f);
      const float hy = R == 1 ? (dy == 0 ? 0.5f : 0.25f) : (dy == 0 ? 0.375f : (dy == 1 || dy == -1) ? 0.25f : 0.0625f);
      const int o = dy * STEP * SW + dx * STEP;
      const float4 gq = sG[ti + o];
      const int tx = qx + dx * STEP, ty = qy + dy * STEP;
      if ((!CHECK || (tx >= 0 && ty >= 0 && tx < w && ty < h)) && gq.w >= 0.0f) {
        const float4 cq = sA[ti + o];
        const float wt = (hx * hy) * pow128(fmaxf(dot3(gq, gp), 0.0f)) *
                         expf(-fabsf(gq.w - gp.w) * iz[dx * dx + dy * dy] - sl * fabsf(lum(cq) - lc));
        sw += wt;
        scx += wt * cq.x;
        scy += wt * cq.y;
        scz += wt * cq.z;
        sv += wt * wt * cq.w;
      }
    }
  }
  return make_float4(scx / sw, scy / sw, scz / sw, sv / (sw * sw));
}

// 2^x on the special-function unit (the hardware approximation WGSL's exp may use as well).
HD_INL float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
constexpr float LOG2E = 1.4426950408889634f;
// log2 of the B-spline tap weights h: 1/4, 1/2 (R = 1) and 1/16, 1/4, 3/8 (R = 2)
HD_INL constexpr float lg_h(int R, int d) {
  return R == 1 ? (d == 0 ? -1.0f : -2.0f) : (d == 0 ? -1.4150374992788438f : (d == 1 || d == -1) ? -2.0f : -4.0f);
}

// The fused schedule's atrousFn: the weights of filt() with exp(x) taken as 2^(x log2 e), log2 e folded into the
// per-centre factors (1 / (zg dist step + 1e-3) and s / sd) and the tap's B-spline weight h_x h_y folded into the
// exponent as log2(h_x) + log2(h_y); CHECK = false leaves out the inside() test on interior tiles. Same operation
// order as filt() otherwise; the differences are last-place roundings of the weights.
template <int R, int STEP, bool PREF, int SW, bool CHECK>
HD_INL float4 filt_x(const float4 *sA, const float4 *sG, int lx, int ly, int qx, int qy, int w, int h, float s,
                     float c) {
  const int ti = ly * SW + lx;
  const float4 gp = sG[ti];
  const float4 center = sA[ti];
  float gv;
  if (PREF) {
    gv = 0.0625f * (sA[ti - SW - 1].w + sA[ti - SW + 1].w + sA[ti + SW - 1].w + sA[ti + SW + 1].w) +
         0.125f * (sA[ti - SW].w + sA[ti - 1].w + sA[ti + 1].w + sA[ti + SW].w) + 0.25f * center.w;
  } else {
    gv = center.w;
  }
  const float lc = lum(center);
  const float sll = LOG2E * s / (sqrtf(fmaxf(gv, 1e-12f)) + 1e-6f);
  const float zl = sG[ti - 1].w, zr = sG[ti + 1].w, zu = sG[ti - SW].w, zd = sG[ti + SW].w;
  const float gx = fminf(zr > 0.0f ? fabsf(zr - gp.w) : 1e9f, zl > 0.0f ? fabsf(zl - gp.w) : 1e9f);
  const float gy = fminf(zd > 0.0f ? fabsf(zd - gp.w) : 1e9f, zu > 0.0f ? fabsf(zu - gp.w) : 1e9f);
  const float zg = fminf(fmaxf(gx, gy), gp.w);
  float izl[9];
#pragma unroll
  for (int d = 1; d <= 2 * R * R; d++) {
    const float k = d == 1 ? 1.0f * STEP
                    : d == 2 ? 1.41421356237309515f * STEP
                    : d == 4 ? 2.0f * STEP
                    : d == 5 ? 2.23606797749978981f * STEP
                    : d == 8 ? 2.82842712474619029f * STEP
                             : 0.0f;
    izl[d] = LOG2E / (zg * k + 1e-3f);
  }
  constexpr float hc = R == 1 ? 0.5f : 0.375f;
  const float cw = (hc * hc) * c;
  float sw = cw;
  float scx = center.x * cw, scy = center.y * cw, scz = center.z * cw;
  float sv = center.w * cw * cw;
  // the taps in the WGSL's order (row-major, centre left out), two at a time: the pair's (n.n)^128 chains, weights
  // and squared weights are packed FP32x2 operations (lane by lane the scalar arithmetic), the accumulation stays in
  // tap order
  constexpr int NTAP = (2 * R + 1) * (2 * R + 1) - 1;
#pragma unroll
  for (int k = 0; k < NTAP; k += 2) {
    int dxs[2], dys[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int t = k + u < NTAP / 2 ? k + u : k + u + 1;  // skip the centre
      dxs[u] = t % (2 * R + 1) - R;
      dys[u] = t / (2 * R + 1) - R;
    }
    const int o0 = dys[0] * STEP * SW + dxs[0] * STEP, o1 = dys[1] * STEP * SW + dxs[1] * STEP;
    const float4 g0 = sG[ti + o0], g1 = sG[ti + o1];
    const float4 c0 = sA[ti + o0], c1 = sA[ti + o1];
    bool ok0 = g0.w >= 0.0f, ok1 = g1.w >= 0.0f;
    if (CHECK) {
      const int x0 = qx + dxs[0] * STEP, y0 = qy + dys[0] * STEP, x1 = qx + dxs[1] * STEP, y1 = qy + dys[1] * STEP;
      ok0 = ok0 && x0 >= 0 && y0 >= 0 && x0 < w && y0 < h;
      ok1 = ok1 && x1 >= 0 && y1 >= 0 && x1 < w && y1 < h;
    }
    float2 pp = make_float2(fmaxf(dot3(g0, gp), 0.0f), fmaxf(dot3(g1, gp), 0.0f));
#pragma unroll
    for (int i = 0; i < 7; i++) pp = __fmul2_rn(pp, pp);  // (n.n)^128
    const float a0 = fmaf(-fabsf(g0.w - gp.w), izl[dxs[0] * dxs[0] + dys[0] * dys[0]],
                          fmaf(-sll, fabsf(lum(c0) - lc), lg_h(R, dxs[0]) + lg_h(R, dys[0])));
    const float a1 = fmaf(-fabsf(g1.w - gp.w), izl[dxs[1] * dxs[1] + dys[1] * dys[1]],
                          fmaf(-sll, fabsf(lum(c1) - lc), lg_h(R, dxs[1]) + lg_h(R, dys[1])));
    const float2 wt = __fmul2_rn(pp, make_float2(ex2_approx(a0), ex2_approx(a1)));
    const float2 ww = __fmul2_rn(wt, wt);
    if (ok0) {
      sw += wt.x;
      scx += wt.x * c0.x;
      scy += wt.x * c0.y;
      scz += wt.x * c0.z;
      sv += ww.x * c0.w;
    }
    if (ok1) {
      sw += wt.y;
      scx += wt.y * c1.x;
      scy += wt.y * c1.y;
      scz += wt.y * c1.z;
      sv += ww.y * c1.w;
    }
  }
  return make_float4(scx / sw, scy / sw, scz / sw, sv / (sw * sw));
}

// ------------------------------------------------------------------------------------------------ TEMPORAL
// History key test (hush.js:103-105).
HD_INL bool check_key(float4 k, float4 n, float zPrev, float obj) {
  return k.z >= 0.0f && k.w == obj && fabsf(k.z - zPrev) <= 0.05f * zPrev + 0.01f &&
         dot3(oct_dec(k.x, k.y), n) >= 0.9f;
}

// Per-pixel feature inputs of pixel() (hush.js:111-223), the five vec4 P0..P4.
struct PixP {
  float4 P0, P1, P2, P3, P4;
};
HD_INL PixP pixp_default() {
  PixP R;
  R.P0 = R.P1 = R.P3 = R.P4 = make_float4(0.f, 0.f, 0.f, 0.f);
  R.P2 = make_float4(0.f, 0.f, -1.0f, 0.f);
  return R;
}

// pixel(): temporal accumulation of one pixel at (px, py), illumination tile sI (row stride SW, centre at (lx, ly)).
// Writes A0, mom, key and returns the feature inputs.
template <int SW>
HD_INL PixP temporal_pixel(const HushFrame &f, int px, int py, const float4 *sI, int lx, int ly) {
  PixP R = pixp_default();
  const int W = f.W, H = f.H;
  const float4 nd = ldh(f.nd, py * f.p_nd + px);
  const float4 mv = ldh(f.mv, py * f.p_mv + px);
  const int oi = py * W + px;
  if (nd.w < 0.0f) {
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    sth(f.A0, oi, z);
    sth(f.mom, oi, z);
    sth(f.key, oi, make_float4(0.f, 0.f, -1.0f, mv.z));
    return R;
  }
  const float4 mr = ldh(f.mat, py * f.p_mat + px);
  const int ti = ly * SW + lx;
  const float4 illum = sI[ti];
  const float l = lum(illum);
  float s1x = 0.f, s1y = 0.f, s1z = 0.f, cnt = 0.f;
#pragma unroll
  for (int j = 0; j < 9; j++) {
    const float4 c = sI[ti + (j / 3 - 1) * SW + (j % 3 - 1)];
    s1x += c.x * c.w; s1y += c.y * c.w; s1z += c.z * c.w;
    cnt += c.w;
  }
  cnt = fmaxf(cnt, 1.0f);
  const float mux = s1x / cnt, muy = s1y / cnt, muz = s1z / cnt;
  const float slm = lum3(mux, muy, muz);
  float svx = 0.f, svy = 0.f, svz = 0.f, svar = 0.f;
#pragma unroll
  for (int j = 0; j < 9; j++) {
    const float4 c = sI[ti + (j / 3 - 1) * SW + (j % 3 - 1)];
    const float dx = c.x - mux, dy = c.y - muy, dz = c.z - muz;
    const float dl = lum(c) - slm;
    svx += c.w * dx * dx; svy += c.w * dy * dy; svz += c.w * dz * dz;
    svar += c.w * dl * dl;
  }
  const float sdx = sqrtf(fmaxf(svx / cnt, 1e-12f)), sdy = sqrtf(fmaxf(svy / cnt, 1e-12f)),
              sdz = sqrtf(fmaxf(svz / cnt, 1e-12f));
  svar /= cnt;
  bool has = false;
  float hcx = 0.f, hcy = 0.f, hcz = 0.f;
  float4 hm = make_float4(0.f, 0.f, 0.f, 0.f);
  float v = 0.f, alpha = 1.0f, gamma = 1.0f;
  if (!f.reset) {
    const float ppx = (float)px + mv.x, ppy = (float)py + mv.y;
    const float bx = floorf(ppx), by = floorf(ppy);
    const float fx = ppx - bx, fy = ppy - by;
    const int bix = __float2int_rz(bx), biy = __float2int_rz(by);
    float sumW = 0.f;
    const float wts[4] = {(1.0f - fx) * (1.0f - fy), fx * (1.0f - fy), (1.0f - fx) * fy, fx * fy};
    float4 k4[4], c4[4], m4[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int q = clampi(biy + (i >> 1), 0, H - 1) * W + clampi(bix + (i & 1), 0, W - 1);
      k4[i] = ldh(f.key_prev, q);
      c4[i] = ldh(f.hist_prev, q);
      m4[i] = ldh(f.mom_prev, q);
    }
    const int cx = __float2int_rz(floorf(ppx + 0.5f)), cy = __float2int_rz(floorf(ppy + 0.5f));
    const float4 pq = ldh(f.par0_prev, (clampi(cy, 0, H - 1) >> 1) * f.W2 + (clampi(cx, 0, W - 1) >> 1));
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int qx = bix + (i & 1), qy = biy + (i >> 1);
      if (wts[i] > 0.0f && qx >= 0 && qy >= 0 && qx < W && qy < H && check_key(k4[i], nd, mv.w, mv.z)) {
        sumW += wts[i];
        hcx += wts[i] * c4[i].x; hcy += wts[i] * c4[i].y; hcz += wts[i] * c4[i].z;
        hm.x += wts[i] * m4[i].x; hm.y += wts[i] * m4[i].y; hm.z += wts[i] * m4[i].z; hm.w += wts[i] * m4[i].w;
      }
    }
    if (sumW >= 0.01f) {
      hcx /= sumW; hcy /= sumW; hcz /= sumW;
      hm.x /= sumW; hm.y /= sumW; hm.z /= sumW; hm.w /= sumW;
      v = sumW;
      has = true;
    } else {
      float n3 = 0.f;
      hcx = hcy = hcz = 0.f;
      hm = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int j = 0; j < 9; j++) {
        const int qx = cx + j % 3 - 1, qy = cy + j / 3 - 1;
        if (qx >= 0 && qy >= 0 && qx < W && qy < H && check_key(ldh(f.key_prev, qy * W + qx), nd, mv.w, mv.z)) {
          n3 += 1.0f;
          const float4 c = ldh(f.hist_prev, qy * W + qx), m = ldh(f.mom_prev, qy * W + qx);
          hcx += c.x; hcy += c.y; hcz += c.z;
          hm.x += m.x; hm.y += m.y; hm.z += m.z; hm.w += m.w;
        }
      }
      if (n3 > 0.0f) {
        hcx /= n3; hcy /= n3; hcz /= n3;
        hm.x /= n3; hm.y /= n3; hm.z /= n3; hm.w /= n3;
        v = 0.1f;
        has = true;
      }
    }
    alpha = pq.x;
    gamma = pq.y;
  }
  has = has && hm.w > 0.0f;
  float colx = illum.x, coly = illum.y, colz = illum.z;
  float nmx = l, nmy = l * l, nfast = l, len1 = 1.0f, lag = 0.0f;
  if (has) {
    const float hclx = fminf(fmaxf(hcx, mux - gamma * sdx), mux + gamma * sdx);
    const float hcly = fminf(fmaxf(hcy, muy - gamma * sdy), muy + gamma * sdy);
    const float hclz = fminf(fmaxf(hcz, muz - gamma * sdz), muz + gamma * sdz);
    len1 = fminf(hm.w + 1.0f, HMAX);
    const float a = fmaxf(alpha, 1.0f / len1);
    colx = hclx + (illum.x - hclx) * a;
    coly = hcly + (illum.y - hcly) * a;
    colz = hclz + (illum.z - hclz) * a;
    nmx = hm.x + (l - hm.x) * a;
    nmy = hm.y + (l * l - hm.y) * a;
    nfast = hm.z + (l - hm.z) * fmaxf(1.0f / 6.0f, 1.0f / len1);
    const float lh = lum3(hcx, hcy, hcz);
    lag = fabsf(slm - lh) / (sqrtf(fmaxf(svar / cnt, 1e-12f)) + 0.02f * lh + 1e-3f);
  } else {
    v = 0.0f;
  }
  const float tvar = fmaxf(nmy - nmx * nmx, 0.0f);
  const float4 A = make_float4(colx, coly, colz, svar + (tvar - svar) * fminf(len1 / 4.0f, 1.0f));
  const float2 oc = oct_enc(nd.x, nd.y, nd.z);
  sth(f.A0, oi, A);
  sth(f.mom, oi, make_float4(nmx, nmy, nfast, len1));
  sth(f.key, oi, make_float4(oc.x, oc.y, nd.w, mv.z));
  const float E = f.exposure;
  const float4 Aq = make_float4(qf16(A.x), qf16(A.y), qf16(A.z), qf16(A.w));
  const float m1 = E * qf16(nmx);
  const float m2 = E * E * qf16(nmy);
  R.P0 = make_float4(E * lum(Aq), E * qf16(l), fmaxf(m2 - m1 * m1, 0.0f), len1);
  R.P1 = make_float4(qf16(v), qf16(lag), E * qf16(nfast), m1);
  R.P2 = make_float4(qf16(oc.x), qf16(oc.y), qf16(nd.w), qf16(sqrtf(mv.x * mv.x + mv.y * mv.y)));
  R.P3 = mr;
  R.P4 = Aq;
  return R;
}

// Block features of block() (hush.js:226-282) from the four pixels' P (j = 0..3 in (x, y) = (j & 1, j >> 1)) and
// the 4x4 illumination neighbourhood of the block (tile sI, top-left of the neighbourhood at tile index t0).
// Returns the 20 features in f[], the block mean colour AC, and the guide (oct normal, Z, count) in G; ok = nv > 0.
template <int SW>
HD_INL bool block_features(const PixP *P, const float4 *sI, int t0, float E, float *f, float4 &AC, float4 &G) {
  float nv = 0.f;
  float4 S0 = make_float4(0.f, 0.f, 0.f, 0.f), S1 = S0, S3 = S0;
  AC = S0;
  float Nx = 0.f, Ny = 0.f, Nz = 0.f, MV = 0.f, Z = 0.f;
  float la[4], zs[4];
  float4 ns[4];
  bool ok[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    ok[j] = P[j].P2.z >= 0.0f;
    la[j] = 0.f; zs[j] = 0.f;
    ns[j] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!ok[j]) continue;
    nv += 1.0f;
    la[j] = P[j].P0.x;
    ns[j] = oct_dec(P[j].P2.x, P[j].P2.y);
    zs[j] = P[j].P2.z;
    S0.x += P[j].P0.x; S0.y += P[j].P0.y; S0.z += P[j].P0.z; S0.w += P[j].P0.w;
    S1.x += P[j].P1.x; S1.y += P[j].P1.y; S1.z += P[j].P1.z; S1.w += P[j].P1.w;
    Nx += ns[j].x; Ny += ns[j].y; Nz += ns[j].z;
    S3.x += P[j].P3.x; S3.y += P[j].P3.y; S3.z += P[j].P3.z; S3.w += P[j].P3.w;
    AC.x += P[j].P4.x; AC.y += P[j].P4.y; AC.z += P[j].P4.z; AC.w += P[j].P4.w;
    MV += P[j].P2.w;
    Z += P[j].P2.z;
  }
  if (nv == 0.0f) {
    G = make_float4(0.f, 0.f, -1.0f, 0.f);
    return false;
  }
  const float k = 1.0f / nv;
  S0.x *= k; S0.y *= k; S0.z *= k; S0.w *= k;
  S1.x *= k; S1.y *= k; S1.z *= k; S1.w *= k;
  Nx *= k; Ny *= k; Nz *= k;
  S3.x *= k; S3.y *= k; S3.z *= k; S3.w *= k;
  AC.x *= k; AC.y *= k; AC.z *= k; AC.w *= k;
  MV *= k;
  Z *= k;
  const float Lacc = S0.x;
  float VA = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++)
    if (ok[j]) VA += (la[j] - Lacc) * (la[j] - Lacc);
  VA *= k;
  float s1 = 0.f, n4 = 0.f;
  float lq[16];
#pragma unroll
  for (int j = 0; j < 16; j++) {
    const float4 t = sI[t0 + (j >> 2) * SW + (j & 3)];
    lq[j] = E * qf16(lum(t));
    s1 += t.w * E * qf16(lum(t));
    n4 += t.w;
  }
  const float mu4 = s1 / fmaxf(n4, 1.0f);
  float var4 = 0.f;
#pragma unroll
  for (int j = 0; j < 16; j++) {
    const float w = sI[t0 + (j >> 2) * SW + (j & 3)].w;
    const float d = lq[j] - mu4;
    var4 += w * d * d;
  }
  var4 /= fmaxf(n4, 1.0f);
  const float nl = fmaxf(sqrtf(Nx * Nx + Ny * Ny + Nz * Nz), 1e-6f);
  const float4 Nn = make_float4(Nx / nl, Ny / nl, Nz / nl, 0.f);
  float zmax = -1e30f, zmin = 1e30f, mind = 1e30f;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    if (ok[j]) {
      zmax = fmaxf(zmax, zs[j]);
      zmin = fminf(zmin, zs[j]);
      mind = fminf(mind, dot3(ns[j], Nn));
    }
  }
  const float dz = fminf(fmaxf((zmax - zmin) / fmaxf(zmin, 1e-6f), 0.0f), 1.0f);
  const float dn = fminf(fmaxf(1.0f - mind, 0.0f), 2.0f);
  const float2 oc = oct_enc(Nn.x, Nn.y, Nn.z);
  f[0] = log1p_w(Lacc); f[1] = log1p_w(S0.y); f[2] = log1p_w(S0.z); f[3] = log1p_w(var4);
  f[4] = S0.w / HMAX; f[5] = S1.x; f[6] = log1p_w(S1.y);
  f[7] = log1p_w(fabsf(S1.z - S1.w) / (S1.w + 1e-3f));
  f[8] = oc.x; f[9] = oc.y; f[10] = dz; f[11] = dn;
  f[12] = S3.x; f[13] = S3.y; f[14] = S3.z; f[15] = S3.w;
  f[16] = 1.0f - nv / 4.0f; f[17] = log1p_w(MV); f[18] = log1p_w(mu4); f[19] = log1p_w(VA);
  G = make_float4(oc.x, oc.y, Z, nv);
  return true;
}

// ------------------------------------------------------------------------------------------------ FINE_FINAL
// jbw() for the fused schedule: rzl = log2(e) / (0.05 z + 1e-3), formed once per pixel; exp as 2^(x log2 e).
HD_INL float jbw_x(float frx, float fry, int j, float4 nq, float zq, float4 n, float z, float rzl) {
  const float wb = ((j & 1) == 1 ? frx : 1.0f - frx) * ((j >> 1) == 1 ? fry : 1.0f - fry);
  const float dn = fmaxf(dot3(nq, n), 0.0f);
  const float dn2 = dn * dn;
  const float dn4 = dn2 * dn2;
  return wb * ex2_approx(-fabsf(zq - z) * rzl) * dn4 * dn4;
}
HD_INL float jbw(float frx, float fry, int j, float4 nq, float zq, float4 n, float z) {  // hush.js:552-558
  const float wb = ((j & 1) == 1 ? frx : 1.0f - frx) * ((j >> 1) == 1 ? fry : 1.0f - fry);
  const float dn = fmaxf(dot3(nq, n), 0.0f);
  const float dn2 = dn * dn;
  const float dn4 = dn2 * dn2;
  return wb * expf(-fabsf(zq - z) / (0.05f * z + 1e-3f)) * dn4 * dn4;
}

// ------------------------------------------------------------------------------------------------ TAA
HD_INL float3 to_ycocg(float3 c) {
  return make_float3(c.x * 0.25f + c.y * 0.5f + c.z * 0.25f, c.x * 0.5f - c.z * 0.5f,
                     -c.x * 0.25f + c.y * 0.5f - c.z * 0.25f);
}
HD_INL float3 from_ycocg(float3 c) { return make_float3(c.x + c.y - c.z, c.x + c.z, c.x - c.y - c.z); }
HD_INL float3 tmap(float3 c) {
  const float d = 1.0f + lum3(c.x, c.y, c.z);
  return make_float3(c.x / d, c.y / d, c.z / d);
}
HD_INL float3 itmap(float3 c) {
  const float d = fmaxf(1.0f - lum3(c.x, c.y, c.z), 1e-4f);
  return make_float3(c.x / d, c.y / d, c.z / d);
}

}  // namespace hush
