// Two-pixel lanes for the fused a-trous stages: each thread filters two horizontally adjacent pixels with packed
// FP32x2 arithmetic (fma / mul / add .rn.f32x2 on sm_100a), so every tap's weight and accumulation costs one packed
// instruction for both pixels instead of one scalar instruction each.
//
// The halo tile is held in shared memory in the pair layout: entry (r, e) holds the two texels at columns c and c + 1
// of row r of the staged window, as four float4 arrays (structure of arrays, so a warp's 16-byte loads of
// consecutive entries touch consecutive addresses):
//   g0 = (nx, nx', ny, ny'), g1 = (nz, nz', z, z')   decoded guide: normal and depth
//   c0 = (r, r', g, g'),     c1 = (b, b', v, v')     colour and variance
// OVL = true: an entry at every column c (step-1 filters and the 3x3 variance prefilter reach odd offsets);
// OVL = false: entries at even columns only (steps 2 and 4, whose taps keep the pair's alignment).
#pragma once
#include "hush_device.cuh"

namespace hush {

HD_INL float2 f2(float a, float b) { return make_float2(a, b); }
HD_INL float2 lo2(float4 v) { return make_float2(v.x, v.y); }
HD_INL float2 hi2(float4 v) { return make_float2(v.z, v.w); }
HD_INL float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
HD_INL float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
HD_INL float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
HD_INL float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
HD_INL float2 abs2(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
HD_INL float2 bc2(float a) { return make_float2(a, a); }

// Pair-layout tile pointers and its geometry (EW entries per row).
struct PairTile {
  float4 *g0, *g1, *c0, *c1;
};

// Entry index of (row, column) in a tile with EW entries per row.
template <bool OVL, int EW>
HD_INL int pe(int r, int c) {
  return r * EW + (OVL ? c : (c >> 1));
}
// Depth of the texel at (row, column), any column.
template <bool OVL, int EW>
HD_INL float pz(const PairTile &T, int r, int c) {
  if (OVL || !(c & 1)) return T.g1[pe<OVL, EW>(r, c)].z;
  return T.g1[pe<OVL, EW>(r, c - 1)].w;
}

// atrousFn (hush.js:431-476) for the two pixels at tile position (row, col) and (row, col + 1), col even; (qx, qy)
// the left pixel's image position, (w, h) the image size for the inside() test (left out with CHECK = false). The
// weights are filt_x()'s: exp as 2^(x log2 e) with log2 e in the per-centre factors and log2(h_x h_y) in the exponent;
// a tap outside the image or on sky gets weight 0 on its lane. Writes both pixels' (colour, variance); a lane whose
// centre is sky produces a meaningless value that the caller discards.
template <int R, int STEP, bool PREF, bool OVL, bool CHECK, int EW>
HD_INL void filt_pair(const PairTile &T, int row, int col, int qx, int qy, int w, int h, float2 s, float2 c,
                      float4 &out0, float4 &out1) {
  static_assert(OVL || (!PREF && STEP % 2 == 0), "the even-column layout serves even steps without prefilter");
  const int e = pe<OVL, EW>(row, col);
  const float4 G0 = T.g0[e], G1 = T.g1[e], C0 = T.c0[e], C1 = T.c1[e];
  const float2 nx = lo2(G0), ny = hi2(G0), nz = lo2(G1), zp = hi2(G1);
  const float2 cr = lo2(C0), cg = hi2(C0), cb = lo2(C1), cv = hi2(C1);
  float2 gv;
  if constexpr (PREF) {
    auto v = [&](int dx, int dy) { return hi2(T.c1[pe<OVL, EW>(row + dy, col + dx)]); };
    const float2 corner = add2(add2(add2(v(-1, -1), v(1, -1)), v(-1, 1)), v(1, 1));
    const float2 edge = add2(add2(add2(v(0, -1), v(-1, 0)), v(1, 0)), v(0, 1));
    gv = fma2(bc2(0.25f), cv, fma2(bc2(0.125f), edge, mul2(bc2(0.0625f), corner)));
  } else {
    gv = cv;
  }
  const float2 lc = fma2(bc2(0.0722f), cb, fma2(bc2(0.7152f), cg, mul2(bc2(0.2126f), cr)));
  float2 sll, zg;
  {
    const float g[2] = {gv.x, gv.y}, sv[2] = {s.x, s.y}, zc[2] = {zp.x, zp.y};
    float sl2[2], zg2[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
      sl2[k] = LOG2E * sv[k] / (sqrtf(fmaxf(g[k], 1e-12f)) + 1e-6f);
      const float zl = pz<OVL, EW>(T, row, col + k - 1), zr = pz<OVL, EW>(T, row, col + k + 1);
      const float zu = pz<OVL, EW>(T, row - 1, col + k), zd = pz<OVL, EW>(T, row + 1, col + k);
      const float gx = fminf(zr > 0.0f ? fabsf(zr - zc[k]) : 1e9f, zl > 0.0f ? fabsf(zl - zc[k]) : 1e9f);
      const float gy = fminf(zd > 0.0f ? fabsf(zd - zc[k]) : 1e9f, zu > 0.0f ? fabsf(zu - zc[k]) : 1e9f);
      zg2[k] = fminf(fmaxf(gx, gy), zc[k]);
    }
    sll = f2(sl2[0], sl2[1]);
    zg = f2(zg2[0], zg2[1]);
  }
  float2 izl[9];
#pragma unroll
  for (int d = 1; d <= 2 * R * R; d++) {
    const float k = d == 1 ? 1.0f * STEP
                    : d == 2 ? 1.41421356237309515f * STEP
                    : d == 4 ? 2.0f * STEP
                    : d == 5 ? 2.23606797749978981f * STEP
                    : d == 8 ? 2.82842712474619029f * STEP
                             : 0.0f;
    izl[d] = f2(LOG2E / (zg.x * k + 1e-3f), LOG2E / (zg.y * k + 1e-3f));
  }
  constexpr float hc = R == 1 ? 0.5f : 0.375f;
  const float2 cw = mul2(bc2(hc * hc), c);
  float2 sw = cw;
  float2 sr = mul2(cr, cw), sg = mul2(cg, cw), sb = mul2(cb, cw);
  float2 sv = mul2(mul2(cv, cw), cw);
  const float2 nsll = f2(-sll.x, -sll.y);
#pragma unroll
  for (int dy = -R; dy <= R; dy++) {
#pragma unroll
    for (int dx = -R; dx <= R; dx++) {
      if (dx == 0 && dy == 0) continue;
      const int q = pe<OVL, EW>(row + dy * STEP, col + dx * STEP);
      const float4 Q0 = T.g0[q], Q1 = T.g1[q], D0 = T.c0[q], D1 = T.c1[q];
      const float2 zq = hi2(Q1);
      bool ok0 = zq.x >= 0.0f, ok1 = zq.y >= 0.0f;
      if constexpr (CHECK) {
        const int tx = qx + dx * STEP, ty = qy + dy * STEP;
        const bool iy = ty >= 0 && ty < h;
        ok0 = ok0 && iy && tx >= 0 && tx < w;
        ok1 = ok1 && iy && tx + 1 >= 0 && tx + 1 < w;
      }
      const float2 dot = fma2(lo2(Q1), nz, fma2(hi2(Q0), ny, mul2(lo2(Q0), nx)));
      float2 p = f2(fmaxf(dot.x, 0.0f), fmaxf(dot.y, 0.0f));
      p = mul2(p, p); p = mul2(p, p); p = mul2(p, p); p = mul2(p, p);
      p = mul2(p, p); p = mul2(p, p); p = mul2(p, p);  // (n . n)^128
      const float2 lq = fma2(bc2(0.0722f), lo2(D1), fma2(bc2(0.7152f), hi2(D0), mul2(bc2(0.2126f), lo2(D0))));
      const float2 dz = abs2(sub2(zq, zp)), dl = abs2(sub2(lq, lc));
      const float lh = lg_h(R, dx) + lg_h(R, dy);
      const float2 arg = fma2(f2(-dz.x, -dz.y), izl[dx * dx + dy * dy], fma2(nsll, dl, bc2(lh)));
      float2 wt = mul2(p, f2(ex2_approx(arg.x), ex2_approx(arg.y)));
      wt = f2(ok0 ? wt.x : 0.0f, ok1 ? wt.y : 0.0f);
      sw = add2(sw, wt);
      sr = fma2(wt, lo2(D0), sr);
      sg = fma2(wt, hi2(D0), sg);
      sb = fma2(wt, lo2(D1), sb);
      sv = fma2(mul2(wt, wt), hi2(D1), sv);
    }
  }
  out0 = make_float4(sr.x / sw.x, sg.x / sw.x, sb.x / sw.x, sv.x / (sw.x * sw.x));
  out1 = make_float4(sr.y / sw.y, sg.y / sw.y, sb.y / sw.y, sv.y / (sw.y * sw.y));
}

// One pair entry from two texels: a = (colour, variance) and g = (normal, depth) of columns c and c + 1.
HD_INL void pair_put(const PairTile &T, int e, float4 a0, float4 a1, float4 q0, float4 q1) {
  T.g0[e] = make_float4(q0.x, q1.x, q0.y, q1.y);
  T.g1[e] = make_float4(q0.z, q1.z, q0.w, q1.w);
  T.c0[e] = make_float4(a0.x, a1.x, a0.y, a1.y);
  T.c1[e] = make_float4(a0.z, a1.z, a0.w, a1.w);
}

}  // namespace hush
