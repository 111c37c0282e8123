// CPU oracle for the Hush denoise path: TEST INFRASTRUCTURE ONLY (see hush_oracle.h).
//
// Each function below restates one WGSL pass of the reference (src/denoise/hush.js) pixel by pixel, with the WGSL
// expression order kept so that the f32 mode rounds like an unfused f32 shader. Workgroup tiles in the WGSL are
// caches of pure functions of the global position (the TEMPORAL tile is zero outside the image, the a-trous / TAA
// tiles are clamp-to-edge loads), so the restatement indexes global positions directly.
#include "hush_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ------------------------------------------------------------------------------------------------ f16 storage
inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// Exact f16 -> f32 (textureLoad of rgba16float, unpack2x16float; halfToFloat hush.js:706-711).
inline float h2f(uint16_t h) {
  uint32_t s = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  if (e == 0) { float v = (float)m * 5.9604644775390625e-08f; return s ? -v : v; }
  if (e == 31) return bitsf(s | 0x7f800000u | (m << 13));
  return bitsf(s | ((e + 112u) << 23) | (m << 13));
}

// f32 -> f16 rounded toward zero: an rgba16float storage write (hush.js:98 models it this way). Finite values above
// the f16 range become +-65504 (round toward zero never reaches infinity); f16 subnormals are kept.
inline uint16_t f2h_rz(float f) {
  uint32_t x = fbits(f);
  uint16_t s = (uint16_t)((x >> 16) & 0x8000u);
  uint32_t ax = x & 0x7fffffffu;
  if (ax > 0x7f800000u) return s | 0x7fffu;
  if (ax == 0x7f800000u) return s | 0x7c00u;
  if (ax >= 0x477fe000u) return s | 0x7bffu;
  if (ax >= 0x38800000u) return (uint16_t)(s | (((ax >> 23) - 112u) << 10) | ((ax >> 13) & 0x3ffu));
  uint32_t e = ax >> 23;
  if (e <= 102u) return s;
  uint32_t m = (ax & 0x7fffffu) | 0x800000u;
  return (uint16_t)(s | (m >> (126u - e)));
}

// qf16 (hush.js:68, 99): clamp to the f16 range, then drop the low 13 mantissa bits.
inline float qf16f(float x) {
  float c = std::min(std::max(x, -65504.0f), 65504.0f);
  return bitsf(fbits(c) & 0xffffe000u);
}

template <class T> inline T qf16(T x) { return (T)qf16f((float)x); }
template <class T> inline T st16(T x) { return (T)h2f(f2h_rz((float)x)); }

// ------------------------------------------------------------------------------------------------ small vectors
template <class T> struct v2 { T x, y; };
template <class T> struct v3 { T x, y, z; };
template <class T> struct v4 {
  T x, y, z, w;
  v3<T> rgb() const { return {x, y, z}; }
};

template <class T> inline v3<T> operator+(v3<T> a, v3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline v3<T> operator-(v3<T> a, v3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline v3<T> operator*(v3<T> a, v3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline v3<T> operator/(v3<T> a, v3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> inline v3<T> operator*(T s, v3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline v3<T> operator*(v3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline v3<T> operator/(v3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline v4<T> operator+(v4<T> a, v4<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class T> inline v4<T> operator*(T s, v4<T> a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
template <class T> inline v4<T> operator*(v4<T> a, T s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class T> inline v4<T> operator/(v4<T> a, T s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }
template <class T> inline v3<T> vmin(v3<T> a, v3<T> b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
template <class T> inline v3<T> vmax(v3<T> a, v3<T> b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
template <class T> inline v3<T> v3s(T s) { return {s, s, s}; }

template <class T> inline T dot3(v3<T> a, v3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline T length3(v3<T> a) { return std::sqrt(dot3(a, a)); }

// COMMON helpers (hush.js:31-47).
template <class T> inline T lum(v3<T> c) { return c.x * T(0.2126f) + c.y * T(0.7152f) + c.z * T(0.0722f); }
template <class T> inline v2<T> octEnc(v3<T> n) {
  T den = std::max(std::abs(n.x) + std::abs(n.y) + std::abs(n.z), T(1e-20f));
  v3<T> v = n / den;
  v2<T> s = {v.x >= T(0) ? T(1) : T(-1), v.y >= T(0) ? T(1) : T(-1)};
  if (v.z < T(0)) return {(T(1) - std::abs(v.y)) * s.x, (T(1) - std::abs(v.x)) * s.y};
  return {v.x, v.y};
}
template <class T> inline v3<T> octDec(v2<T> e) {
  v3<T> v = {e.x, e.y, T(1) - std::abs(e.x) - std::abs(e.y)};
  T t = std::max(-v.z, T(0));
  v.x += v.x >= T(0) ? -t : t;
  v.y += v.y >= T(0) ? -t : t;
  return v / std::max(length3(v), T(1e-20f));
}
template <class T> inline T log1p_w(T x) { return std::log(T(1) + x); }  // hush.js:47 (log(1 + x), not log1p)
template <class T> inline T pow128(T x) {
  T x2 = x * x, x4 = x2 * x2, x8 = x4 * x4, x16 = x8 * x8, x32 = x16 * x16, x64 = x32 * x32;
  return x64 * x64;
}
template <class T> inline T sigmoid(T x) { return T(1) / (T(1) + std::exp(-x)); }
template <class T> inline T clampT(T x, T lo, T hi) { return std::min(std::max(x, lo), hi); }

const float HMAX = 32.0f;
const float COARSE_S = 0.25f;  // hush.js:26

// ------------------------------------------------------------------------------------------------ images
struct Img {
  int w = 0, h = 0, ch = 4;
  std::vector<uint16_t> d;
  void alloc(int W, int H, int C = 4) { w = W; h = H; ch = C; d.assign((size_t)W * H * C, 0); }
  template <class T> v4<T> ld(int x, int y, int o = 0) const {
    const uint16_t *p = &d[((size_t)y * w + x) * ch + o];
    return {T(h2f(p[0])), T(h2f(p[1])), T(h2f(p[2])), T(h2f(p[3]))};
  }
  template <class T> void st(int x, int y, v4<T> v) {
    uint16_t *p = &d[((size_t)y * w + x) * ch];
    p[0] = f2h_rz((float)v.x); p[1] = f2h_rz((float)v.y); p[2] = f2h_rz((float)v.z); p[3] = f2h_rz((float)v.w);
  }
  // pack2x16float of qf16 values into texel slot k (hush.js:101 pk)
  template <class T> void pk(int x, int y, int k, T a, T b) {
    uint16_t *p = &d[((size_t)y * w + x) * ch + 2 * k];
    p[0] = f2h_rz(qf16f((float)a)); p[1] = f2h_rz(qf16f((float)b));
  }
  void zero_texel(int x, int y) { std::fill_n(&d[((size_t)y * w + x) * ch], ch, (uint16_t)0); }
};

struct In {  // borrowed frame inputs, dense W x H x 4
  const uint16_t *p;
  int w;
  template <class T> v4<T> ld(int x, int y) const {
    const uint16_t *q = p + ((size_t)y * w + x) * 4;
    return {T(h2f(q[0])), T(h2f(q[1])), T(h2f(q[2])), T(h2f(q[3]))};
  }
};

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
inline int floordiv2(int v) { return v >> 1; }

}  // namespace

// ================================================================================================ Hush state
struct ho_hush {
  int W = 0, H = 0, W2 = 0, H2 = 0, W4 = 0, H4 = 0;
  int frame = 0;
  bool reset = true;
  float exposure = 1.0f;
  int hidden = 16;
  int fp64 = 0;
  int mlp_half = 0;  // the `f16` option: the MLP in f16 arithmetic (hush.js:683-703, 740)
  std::vector<float> wf;  // decoded weights (exact f16 values)
  Img A0, X, Bh[2], mom[2], key[2], hist[2], taa[2], par0[2], par1, par2, F[4], C[2], CG;
  Img *buf(int id) {
    switch (id) {
      case HO_BUF_A0: return &A0; case HO_BUF_X: return &X; case HO_BUF_BH0: return &Bh[0]; case HO_BUF_BH1: return &Bh[1];
      case HO_BUF_MOM0: return &mom[0]; case HO_BUF_MOM1: return &mom[1]; case HO_BUF_KEY0: return &key[0];
      case HO_BUF_KEY1: return &key[1]; case HO_BUF_HIST0: return &hist[0]; case HO_BUF_HIST1: return &hist[1];
      case HO_BUF_TAA0: return &taa[0]; case HO_BUF_TAA1: return &taa[1]; case HO_BUF_PAR0_0: return &par0[0];
      case HO_BUF_PAR0_1: return &par0[1]; case HO_BUF_PAR1: return &par1; case HO_BUF_PAR2: return &par2;
      case HO_BUF_F0: return &F[0]; case HO_BUF_F1: return &F[1]; case HO_BUF_F2: return &F[2]; case HO_BUF_F3: return &F[3];
      case HO_BUF_C0: return &C[0]; case HO_BUF_C1: return &C[1]; case HO_BUF_CG: return &CG;
    }
    return nullptr;
  }
};

namespace {

// ------------------------------------------------------------------------------------------------ MLP
// mlpCode (hush.js:683-704): per output, bias + sum of input*weight in increasing input order, ReLU on the hidden
// layers; layout W1 b1 W2 b2 W3 b3 (hush.js:684).
template <class T> void mlp(const float *w, int Hd, const T *f, T *o) {
  const int NF = 20, NO = 12;
  const int W1 = 0, B1 = Hd * NF, W2 = B1 + Hd, B2 = W2 + Hd * Hd, W3 = B2 + Hd, B3 = W3 + NO * Hd;
  std::vector<T> h1(Hd), h2(Hd);
  for (int j = 0; j < Hd; j++) {
    T a = T(w[B1 + j]);
    for (int i = 0; i < NF; i++) a = a + f[i] * T(w[W1 + j * NF + i]);
    h1[j] = std::max(a, T(0));
  }
  for (int j = 0; j < Hd; j++) {
    T a = T(w[B2 + j]);
    for (int i = 0; i < Hd; i++) a = a + h1[i] * T(w[W2 + j * Hd + i]);
    h2[j] = std::max(a, T(0));
  }
  for (int j = 0; j < NO; j++) {
    T a = T(w[B3 + j]);
    for (int i = 0; i < Hd; i++) a = a + h2[i] * T(w[W3 + j * Hd + i]);
    o[j] = a;
  }
}

// mlpCode with f16 = true (hush.js:683-703, selected by the `f16` option at hush.js:740, 750): every value is an f16
// (features converted with f16(), weights and biases f16 literals), each product input * weight and each running sum
// bias + p0 + p1 + ... rounds to f16 in that left-to-right order (vec4h arithmetic: a multiply and an add per term,
// each correctly rounded, round to nearest even), ReLU as max(., 0h); the outputs widen to f32 (vec4f(oh_k)). Every
// f16 product and every sum of two f16 values is exact in double, so rounding the double once gives the correctly
// rounded f16 result.
double h16(double x) {  // round to the nearest f16 value (ties to even), overflow to infinity
  if (std::isnan(x)) return x;
  const double ax = std::fabs(x);
  if (ax >= 65520.0) return std::copysign(INFINITY, x);
  int e;
  std::frexp(ax, &e);                      // ax = m * 2^e, m in [0.5, 1)
  const int q = std::max(e - 11, -24);     // f16 spacing: 2^(e - 11) for normal values, 2^-24 below 2^-14
  const double u = std::ldexp(1.0, q);
  return std::copysign(std::nearbyint(ax / u) * u, x);  // default rounding mode: to nearest, ties to even
}
void mlp_half(const float *w, int Hd, const float *f, float *o) {
  const int NF = 20, NO = 12;
  const int W1 = 0, B1 = Hd * NF, W2 = B1 + Hd, B2 = W2 + Hd * Hd, W3 = B2 + Hd, B3 = W3 + NO * Hd;
  std::vector<double> x(NF), h1(Hd), h2(Hd);
  for (int i = 0; i < NF; i++) x[i] = h16(f[i]);
  auto layer = [&](const std::vector<double> &in, int nin, int wo, int bo, int nout, bool relu, double *out) {
    for (int j = 0; j < nout; j++) {
      double a = w[bo + j];  // f16 values already
      for (int i = 0; i < nin; i++) a = h16(a + h16(in[i] * (double)w[wo + j * nin + i]));
      out[j] = relu ? (a > 0.0 ? a : 0.0) : a;  // max(., 0h); a NaN sum gives 0, as the GPU's max.f16x2 does
    }
  };
  layer(x, NF, W1, B1, Hd, true, h1.data());
  layer(h1, Hd, W2, B2, Hd, true, h2.data());
  std::vector<double> oo(NO);
  layer(h2, Hd, W3, B3, NO, false, oo.data());
  for (int j = 0; j < NO; j++) o[j] = (float)oo[j];
}

// ------------------------------------------------------------------------------------------------ a-trous
// atrousFn (hush.js:431-476): one (2R+1)^2 edge-aware iteration at global pixel q. A(p) / G(p) return the tile
// contents at the (unclamped) global position p: colour+variance and decoded (normal, depth), both clamp-to-edge.
template <class T, class FA, class FG>
v4<T> filt(int R, int step, bool prefilter, int qx, int qy, int SW, int SH, T s, T c, FA A, FG G) {
  static const float h3[3] = {0.25f, 0.5f, 0.25f};
  static const float h5[5] = {1.0f / 16, 1.0f / 4, 3.0f / 8, 1.0f / 4, 1.0f / 16};
  const float *h = R == 1 ? h3 : h5;
  v4<T> gp = G(qx, qy);
  v4<T> center = A(qx, qy);
  T gv;
  if (prefilter) {
    gv = T(0.0625f) * (A(qx - 1, qy - 1).w + A(qx + 1, qy - 1).w + A(qx - 1, qy + 1).w + A(qx + 1, qy + 1).w) +
         T(0.125f) * (A(qx, qy - 1).w + A(qx - 1, qy).w + A(qx + 1, qy).w + A(qx, qy + 1).w) + T(0.25f) * center.w;
  } else {
    gv = center.w;
  }
  T lc = lum(center.rgb());
  T sl = s / (std::sqrt(std::max(gv, T(1e-12f))) + T(1e-6f));
  T zl = G(qx - 1, qy).w, zr = G(qx + 1, qy).w, zu = G(qx, qy - 1).w, zd = G(qx, qy + 1).w;
  T gx = std::min(zr > T(0) ? std::abs(zr - gp.w) : T(1e9f), zl > T(0) ? std::abs(zl - gp.w) : T(1e9f));
  T gy = std::min(zd > T(0) ? std::abs(zd - gp.w) : T(1e9f), zu > T(0) ? std::abs(zu - gp.w) : T(1e9f));
  T zg = std::min(std::max(gx, gy), gp.w);
  // iz_k = 1 / (zg * sqrt(d_k) * step + 1e-3) for the distinct squared tap distances d_k (hush.js:433-434, 467);
  // the WGSL literal is the JS double sqrt(d)*step read as f32.
  T iz[9];
  for (int d = 1; d <= 8; d++) {
    T k = std::is_same<T, float>::value ? T((float)(std::sqrt((double)d) * step)) : T(std::sqrt((double)d) * step);
    iz[d] = T(1) / (zg * k + T(1e-3f));
  }
  T cw = T(h[R] * h[R]) * c;
  T sw = cw;
  v3<T> sc = center.rgb() * cw;
  T sv = center.w * cw * cw;
  for (int dy = -R; dy <= R; dy++) {
    for (int dx = -R; dx <= R; dx++) {
      if (dx == 0 && dy == 0) continue;
      int ox = dx * step, oy = dy * step;
      int tx = qx + ox, ty = qy + oy;
      v4<T> gq = G(tx, ty);
      if (tx >= 0 && ty >= 0 && tx < SW && ty < SH && gq.w >= T(0)) {
        v4<T> cq = A(tx, ty);
        T w = T(h[dx + R] * h[dy + R]) * pow128(std::max(dot3(gq.rgb(), gp.rgb()), T(0))) *
              std::exp(-std::abs(gq.w - gp.w) * iz[dx * dx + dy * dy] - sl * std::abs(lum(cq.rgb()) - lc));
        sw += w;
        sc = sc + w * cq.rgb();
        sv += w * w * cq.w;
      }
    }
  }
  v3<T> o = sc / sw;
  return {o.x, o.y, o.z, sv / (sw * sw)};
}

// ------------------------------------------------------------------------------------------------ TEMPORAL
// hush.js:79-308. Per 2x2 block: pixel() for the four pixels, then block() for the features.
template <class T> struct PixOut { v4<T> P[5]; };

template <class T> bool check_key(v4<T> k, v3<T> n, T zPrev, T obj) {  // hush.js:103-105
  return k.z >= T(0) && k.w == obj && std::abs(k.z - zPrev) <= T(0.05f) * zPrev + T(0.01f) &&
         dot3(octDec(v2<T>{k.x, k.y}), n) >= T(0.9f);
}

template <class T> void pass_temporal(ho_hush *S, const ho_inputs *in) {
  const int W = S->W, H = S->H;
  const int cur = S->frame & 1, prev = cur ^ 1;
  const bool reset = S->reset;
  const T E = T(S->exposure);
  In rad{in->radiance, W}, ndI{in->normal_depth, W}, mvI{in->motion, W}, matI{in->material, W};
  // the sI tile contents as a function of the global position (hush.js:287-294): zero outside the image / on sky
  std::vector<v4<T>> sI((size_t)W * H);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      v4<T> e = {0, 0, 0, 0};
      if (ndI.ld<T>(x, y).w >= T(0)) {
        v3<T> r = rad.ld<T>(x, y).rgb(), m = matI.ld<T>(x, y).rgb();
        v3<T> il = r / vmax(m, v3s(T(1e-3f)));
        e = {il.x, il.y, il.z, T(1)};
      }
      sI[(size_t)y * W + x] = e;
    }
  }
  auto I = [&](int x, int y) -> v4<T> {
    if (x < 0 || y < 0 || x >= W || y >= H) return {0, 0, 0, 0};
    return sI[(size_t)y * W + x];
  };
  auto inside = [&](int x, int y) { return x >= 0 && y >= 0 && x < W && y < H; };
  Img &kP = S->key[prev], &cP = S->hist[prev], &mP = S->mom[prev], &pP = S->par0[prev];

  // pixel() (hush.js:111-223)
  auto pixel = [&](int px, int py) -> PixOut<T> {
    PixOut<T> R;
    for (auto &v : R.P) v = {0, 0, 0, 0};
    R.P[2] = {0, 0, T(-1), 0};
    v4<T> nd = ndI.ld<T>(px, py), mv = mvI.ld<T>(px, py);
    if (nd.w < T(0)) {
      S->A0.st<T>(px, py, {0, 0, 0, 0});
      S->mom[cur].st<T>(px, py, {0, 0, 0, 0});
      S->key[cur].st<T>(px, py, {0, 0, T(-1), mv.z});
      return R;
    }
    v3<T> n = nd.rgb();
    v4<T> mr = matI.ld<T>(px, py);
    v3<T> illum = I(px, py).rgb();
    T l = lum(illum);
    v3<T> s1 = v3s(T(0));
    T cnt = 0;
    for (int j = 0; j < 9; j++) {
      v4<T> c = I(px + j % 3 - 1, py + j / 3 - 1);
      s1 = s1 + c.rgb() * c.w;
      cnt += c.w;
    }
    cnt = std::max(cnt, T(1));
    v3<T> mu = s1 / cnt;
    T slm = lum(mu);
    v3<T> sv3 = v3s(T(0));
    T svar = 0;
    for (int j = 0; j < 9; j++) {
      v4<T> c = I(px + j % 3 - 1, py + j / 3 - 1);
      v3<T> d = c.rgb() - mu;
      T dl = lum(c.rgb()) - slm;
      sv3 = sv3 + c.w * d * d;
      svar += c.w * dl * dl;
    }
    v3<T> sd = {std::sqrt(std::max(sv3.x / cnt, T(1e-12f))), std::sqrt(std::max(sv3.y / cnt, T(1e-12f))),
                std::sqrt(std::max(sv3.z / cnt, T(1e-12f)))};
    svar /= cnt;
    bool has = false;
    v3<T> hc = v3s(T(0));
    v4<T> hm = {0, 0, 0, 0};
    T v = 0, alpha = 1, gamma = 1;
    if (!reset) {
      T ppx = T(px) + mv.x, ppy = T(py) + mv.y;
      T bx = std::floor(ppx), by = std::floor(ppy);
      T fx = ppx - bx, fy = ppy - by;
      int bix = (int)bx, biy = (int)by;
      T sumW = 0;
      T wts[4] = {(T(1) - fx) * (T(1) - fy), fx * (T(1) - fy), (T(1) - fx) * fy, fx * fy};
      v4<T> k4[4], m4[4];
      v3<T> c4[4];
      for (int i = 0; i < 4; i++) {
        int qx = clampi(bix + (i & 1), 0, W - 1), qy = clampi(biy + (i >> 1), 0, H - 1);
        k4[i] = kP.ld<T>(qx, qy);
        c4[i] = cP.ld<T>(qx, qy).rgb();
        m4[i] = mP.ld<T>(qx, qy);
      }
      int cx = (int)std::floor(ppx + T(0.5f)), cy = (int)std::floor(ppy + T(0.5f));
      v4<T> pq = pP.ld<T>(clampi(cx, 0, W - 1) >> 1, clampi(cy, 0, H - 1) >> 1);
      for (int i = 0; i < 4; i++) {
        if (wts[i] > T(0) && inside(bix + (i & 1), biy + (i >> 1)) && check_key(k4[i], n, mv.w, mv.z)) {
          sumW += wts[i];
          hc = hc + wts[i] * c4[i];
          hm = hm + wts[i] * m4[i];
        }
      }
      if (sumW >= T(0.01f)) {
        hc = hc / sumW;
        hm = hm / sumW;
        v = sumW;
        has = true;
      } else {
        T n3 = 0;
        hc = v3s(T(0));
        hm = {0, 0, 0, 0};
        for (int j = 0; j < 9; j++) {
          int qx = cx + j % 3 - 1, qy = cy + j / 3 - 1;
          if (inside(qx, qy) && check_key(kP.ld<T>(qx, qy), n, mv.w, mv.z)) {
            n3 += T(1);
            hc = hc + cP.ld<T>(qx, qy).rgb();
            hm = hm + mP.ld<T>(qx, qy);
          }
        }
        if (n3 > T(0)) {
          hc = hc / n3;
          hm = hm / n3;
          v = T(0.1f);
          has = true;
        }
      }
      alpha = pq.x;
      gamma = pq.y;
    }
    has = has && hm.w > T(0);
    v3<T> color = illum;
    v2<T> nm = {l, l * l};
    T nfast = l, len1 = 1, lag = 0;
    if (has) {
      v3<T> hcl = vmin(vmax(hc, mu - gamma * sd), mu + gamma * sd);
      len1 = std::min(hm.w + T(1), T(HMAX));
      T a = std::max(alpha, T(1) / len1);
      color = hcl + (illum - hcl) * a;
      nm = {hm.x + (l - hm.x) * a, hm.y + (l * l - hm.y) * a};
      nfast = hm.z + (l - hm.z) * std::max(T(1.0f / 6.0f), T(1) / len1);
      T lh = lum(hc);
      lag = std::abs(slm - lh) / (std::sqrt(std::max(svar / cnt, T(1e-12f))) + T(0.02f) * lh + T(1e-3f));
    } else {
      v = 0;
    }
    T tvar = std::max(nm.y - nm.x * nm.x, T(0));
    v4<T> A = {color.x, color.y, color.z, svar + (tvar - svar) * std::min(len1 / T(4), T(1))};
    v2<T> oc = octEnc(n);
    S->A0.st<T>(px, py, A);
    S->mom[cur].st<T>(px, py, {nm.x, nm.y, nfast, len1});
    S->key[cur].st<T>(px, py, {oc.x, oc.y, nd.w, mv.z});
    // feature inputs from the values as stored (hush.js:212-221)
    v4<T> Aq = {qf16(A.x), qf16(A.y), qf16(A.z), qf16(A.w)};
    T m1 = E * qf16(nm.x);
    T m2 = E * E * qf16(nm.y);
    R.P[0] = {E * lum(Aq.rgb()), E * qf16(l), std::max(m2 - m1 * m1, T(0)), len1};
    R.P[1] = {qf16(v), qf16(lag), E * qf16(nfast), m1};
    R.P[2] = {qf16(oc.x), qf16(oc.y), qf16(nd.w), qf16(std::sqrt(mv.x * mv.x + mv.y * mv.y))};
    R.P[3] = mr;
    R.P[4] = Aq;
    return R;
  };

  // block() (hush.js:226-282)
#pragma omp parallel for schedule(dynamic, 1)
  for (int Y = 0; Y < S->H2; Y++) {
    for (int X = 0; X < S->W2; X++) {
      PixOut<T> Pj[4];
      for (int j = 0; j < 4; j++) {
        int px = 2 * X + (j & 1), py = 2 * Y + (j >> 1);
        if (inside(px, py)) {
          Pj[j] = pixel(px, py);
        } else {
          for (auto &v : Pj[j].P) v = {0, 0, 0, 0};
          Pj[j].P[2] = {0, 0, T(-1), 0};
        }
      }
      T nv = 0;
      v4<T> S0 = {0, 0, 0, 0}, S1 = S0, S3 = S0, AC = S0;
      v3<T> N = v3s(T(0));
      T MV = 0, Z = 0;
      T la[4] = {0, 0, 0, 0}, zs[4] = {0, 0, 0, 0};
      v3<T> ns[4];
      bool ok[4];
      for (int j = 0; j < 4; j++) {
        const v4<T> *P = Pj[j].P;
        ok[j] = P[2].z >= T(0);
        if (!ok[j]) continue;
        nv += T(1);
        la[j] = P[0].x;
        ns[j] = octDec(v2<T>{P[2].x, P[2].y});
        zs[j] = P[2].z;
        S0 = S0 + P[0]; S1 = S1 + P[1]; N = N + ns[j]; S3 = S3 + P[3]; AC = AC + P[4]; MV += P[2].w; Z += P[2].z;
      }
      Img *F = S->F;
      if (nv == T(0)) {
        F[0].zero_texel(X, Y); F[1].zero_texel(X, Y); F[2].zero_texel(X, Y); F[3].zero_texel(X, Y);
        F[3].pk<T>(X, Y, 0, T(0), T(0));
        F[3].pk<T>(X, Y, 1, T(-1), T(0));
        continue;
      }
      T k = T(1) / nv;
      S0 = S0 * k; S1 = S1 * k; N = N * k; S3 = S3 * k; AC = AC * k; MV *= k; Z *= k;
      T Lacc = S0.x;
      T VA = 0;
      for (int j = 0; j < 4; j++) if (ok[j]) VA += (la[j] - Lacc) * (la[j] - Lacc);
      VA *= k;
      T s1 = 0, n4 = 0;
      for (int j = 0; j < 16; j++) {
        v4<T> t = I(2 * X + (j & 3) - 1, 2 * Y + (j >> 2) - 1);
        s1 += t.w * E * qf16(lum(t.rgb()));
        n4 += t.w;
      }
      T mu4 = s1 / std::max(n4, T(1));
      T var4 = 0;
      for (int j = 0; j < 16; j++) {
        v4<T> t = I(2 * X + (j & 3) - 1, 2 * Y + (j >> 2) - 1);
        T d = E * qf16(lum(t.rgb())) - mu4;
        var4 += t.w * d * d;
      }
      var4 /= std::max(n4, T(1));
      v3<T> Nn = N / std::max(length3(N), T(1e-6f));
      T zmax = T(-1e30f), zmin = T(1e30f), mind = T(1e30f);
      for (int j = 0; j < 4; j++) {
        if (ok[j]) { zmax = std::max(zmax, zs[j]); zmin = std::min(zmin, zs[j]); mind = std::min(mind, dot3(ns[j], Nn)); }
      }
      T dz = clampT((zmax - zmin) / std::max(zmin, T(1e-6f)), T(0), T(1));
      T dn = clampT(T(1) - mind, T(0), T(2));
      v2<T> oc = octEnc(Nn);
      T f[20] = {log1p_w(Lacc), log1p_w(S0.y), log1p_w(S0.z), log1p_w(var4), S0.w / T(HMAX), S1.x, log1p_w(S1.y),
                 log1p_w(std::abs(S1.z - S1.w) / (S1.w + T(1e-3f))), oc.x, oc.y, dz, dn, S3.x, S3.y, S3.z, S3.w,
                 T(1) - nv / T(4), log1p_w(MV), log1p_w(mu4), log1p_w(VA)};
      for (int t = 0; t < 4; t++) F[0].pk<T>(X, Y, t, f[2 * t], f[2 * t + 1]);
      for (int t = 0; t < 4; t++) F[1].pk<T>(X, Y, t, f[8 + 2 * t], f[8 + 2 * t + 1]);
      F[2].pk<T>(X, Y, 0, f[16], f[17]); F[2].pk<T>(X, Y, 1, f[18], f[19]);
      F[2].pk<T>(X, Y, 2, AC.x, AC.y); F[2].pk<T>(X, Y, 3, AC.z, AC.w);
      F[3].pk<T>(X, Y, 0, oc.x, oc.y); F[3].pk<T>(X, Y, 1, Z, nv);
      uint16_t *p3 = &F[3].d[((size_t)Y * F[3].w + X) * 8];
      p3[4] = p3[5] = p3[6] = p3[7] = 0;
    }
  }
}

// Packed half-res accessors: F2.zw = mean colour + variance, F3 = (oct normal, depth, count).
template <class T> inline v4<T> f2_ac(const Img &F2, int x, int y) { return F2.ld<T>(x, y, 4); }
template <class T> inline v4<T> f3_g(const Img &F3, int x, int y) { return F3.ld<T>(x, y, 0); }
template <class T> inline v4<T> guide_dec(v4<T> g) {  // (octDec(xy), z)
  v3<T> n = octDec(v2<T>{g.x, g.y});
  return {n.x, n.y, n.z, g.z};
}

// ------------------------------------------------------------------------------------------------ INFER (+mid1)
// hush.js:312-368
template <class T> void pass_infer(ho_hush *S) {
  const int W2 = S->W2, H2 = S->H2, cur = S->frame & 1;
  const Img &F0 = S->F[0], &F1 = S->F[1], &F2 = S->F[2], &F3 = S->F[3];
  auto A = [&](int x, int y) { return f2_ac<T>(F2, clampi(x, 0, W2 - 1), clampi(y, 0, H2 - 1)); };
  auto G = [&](int x, int y) { return guide_dec(f3_g<T>(F3, clampi(x, 0, W2 - 1), clampi(y, 0, H2 - 1))); };
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H2; y++) {
    for (int x = 0; x < W2; x++) {
      if (G(x, y).w < T(0)) {
        S->par0[cur].st<T>(x, y, {0, 0, 0, 0}); S->par1.st<T>(x, y, {0, 0, 0, 0});
        S->par2.st<T>(x, y, {0, 0, 0, 0}); S->Bh[0].st<T>(x, y, {0, 0, 0, 0});
        continue;
      }
      T f[20], o[12];
      v4<T> a = F0.ld<T>(x, y, 0), b = F0.ld<T>(x, y, 4), c = F1.ld<T>(x, y, 0), d = F1.ld<T>(x, y, 4),
            e = F2.ld<T>(x, y, 0);
      v4<T> q[5] = {a, b, c, d, e};
      for (int i = 0; i < 5; i++) { f[4 * i] = q[i].x; f[4 * i + 1] = q[i].y; f[4 * i + 2] = q[i].z; f[4 * i + 3] = q[i].w; }
      if (S->mlp_half) {
        float ff[20], oh[12];
        for (int i = 0; i < 20; i++) ff[i] = (float)f[i];
        mlp_half(S->wf.data(), S->hidden, ff, oh);
        for (int i = 0; i < 12; i++) o[i] = T(oh[i]);
      } else {
        mlp<T>(S->wf.data(), S->hidden, f, o);
      }
      T alpha = T(1.0f / 32.0f) + T(31.0f / 32.0f) * sigmoid(o[0]);
      T gamma = T(0.5f) + T(7.5f) * sigmoid(o[1]);
      T beta = sigmoid(o[2]);
      T kappa = sigmoid(o[3]);
      T s[4], cc[4];
      for (int i = 0; i < 4; i++) s[i] = T(0.25f) * std::exp(clampT(o[4 + i], T(-5), T(5)));
      for (int i = 0; i < 4; i++) cc[i] = std::exp(clampT(o[8 + i], T(-4), T(4)));
      S->par0[cur].st<T>(x, y, {alpha, gamma, beta, kappa});
      S->par1.st<T>(x, y, {s[0], s[1], s[2], s[3]});
      S->par2.st<T>(x, y, {cc[0], cc[1], cc[2], cc[3]});
      S->Bh[0].st<T>(x, y, filt<T>(1, 1, true, x, y, W2, H2, qf16(s[1]), qf16(cc[1]), A, G));
    }
  }
}

// ------------------------------------------------------------------------------------------------ mid2 / mid3
// atrousShader kind mid2 / mid3 (hush.js:482-525, 753-754): 3x3, step 2 / 4, learned s_k, c_k.
template <class T> void pass_mid(ho_hush *S, int k) {
  const int W2 = S->W2, H2 = S->H2;
  const int step = k == 2 ? 2 : 4, comp = k == 2 ? 2 : 3;
  const Img &src = S->Bh[k == 2 ? 0 : 1];
  Img &dst = S->Bh[k == 2 ? 1 : 0];
  const Img &F3 = S->F[3];
  auto A = [&](int x, int y) { return src.ld<T>(clampi(x, 0, W2 - 1), clampi(y, 0, H2 - 1)); };
  auto G = [&](int x, int y) { return guide_dec(f3_g<T>(F3, clampi(x, 0, W2 - 1), clampi(y, 0, H2 - 1))); };
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H2; y++) {
    for (int x = 0; x < W2; x++) {
      if (G(x, y).w < T(0)) { dst.st<T>(x, y, {0, 0, 0, 0}); continue; }
      v4<T> p1 = S->par1.ld<T>(x, y), p2 = S->par2.ld<T>(x, y);
      T s = comp == 2 ? p1.z : p1.w, c = comp == 2 ? p2.z : p2.w;
      dst.st<T>(x, y, filt<T>(1, step, false, x, y, W2, H2, s, c, A, G));
    }
  }
}

// ------------------------------------------------------------------------------------------------ COARSE1
// hush.js:372-422. down() 2x2 count-weighted half -> quarter, then a 5x5 step-1 a-trous with s = COARSE_S.
template <class T> struct Down { v4<T> c, g; };
template <class T> Down<T> down(const ho_hush *S, int Qx, int Qy) {
  const Img &F2 = S->F[2], &F3 = S->F[3];
  T N = 0, vr = 0, z = 0;
  v3<T> col = v3s(T(0)), nrm = v3s(T(0));
  for (int j = 0; j < 4; j++) {
    int hx = Qx * 2 + (j & 1), hy = Qy * 2 + (j >> 1);
    if (hx >= S->W2 || hy >= S->H2) continue;
    v4<T> g3 = f3_g<T>(F3, hx, hy);
    if (g3.w <= T(0)) continue;  // oz.y = count
    v4<T> a = f2_ac<T>(F2, hx, hy);
    T w = g3.w;
    N += w;
    col = col + w * a.rgb();
    vr += w * a.w;
    nrm = nrm + w * octDec(v2<T>{g3.x, g3.y});
    z += w * g3.z;
  }
  if (N == T(0)) return {{0, 0, 0, 0}, {0, 0, T(-1), 0}};
  v2<T> o = octEnc(nrm / std::max(length3(nrm), T(1e-6f)));
  v3<T> cm = col / N;
  return {{qf16(cm.x), qf16(cm.y), qf16(cm.z), qf16(vr / N / N)}, {qf16(o.x), qf16(o.y), qf16(z / N), T(0)}};
}

template <class T> void pass_coarse1(ho_hush *S) {
  const int W4 = S->W4, H4 = S->H4;
  // the tile holds down() of clamped quarter positions; compute the whole quarter image once
  std::vector<v4<T>> dc((size_t)W4 * H4), dg((size_t)W4 * H4);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H4; y++) {
    for (int x = 0; x < W4; x++) {
      Down<T> d = down<T>(S, x, y);
      dc[(size_t)y * W4 + x] = d.c;
      dg[(size_t)y * W4 + x] = d.g;
      S->CG.st<T>(x, y, d.g);
    }
  }
  auto A = [&](int x, int y) { return dc[(size_t)clampi(y, 0, H4 - 1) * W4 + clampi(x, 0, W4 - 1)]; };
  auto G = [&](int x, int y) { return guide_dec(dg[(size_t)clampi(y, 0, H4 - 1) * W4 + clampi(x, 0, W4 - 1)]); };
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H4; y++) {
    for (int x = 0; x < W4; x++) {
      if (G(x, y).w < T(0)) { S->C[1].st<T>(x, y, {0, 0, 0, 0}); continue; }
      S->C[1].st<T>(x, y, filt<T>(2, 1, true, x, y, W4, H4, T(COARSE_S), T(1), A, G));
    }
  }
}

// atrousShader kind coarse (hush.js:752): 5x5, step 2, prefilter, fixed s, c = 1; C1 -> C0 with guide CG.
template <class T> void pass_coarse2(ho_hush *S) {
  const int W4 = S->W4, H4 = S->H4;
  auto A = [&](int x, int y) { return S->C[1].ld<T>(clampi(x, 0, W4 - 1), clampi(y, 0, H4 - 1)); };
  auto G = [&](int x, int y) { return guide_dec(S->CG.ld<T>(clampi(x, 0, W4 - 1), clampi(y, 0, H4 - 1))); };
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H4; y++) {
    for (int x = 0; x < W4; x++) {
      if (G(x, y).w < T(0)) { S->C[0].st<T>(x, y, {0, 0, 0, 0}); continue; }
      S->C[0].st<T>(x, y, filt<T>(2, 2, true, x, y, W4, H4, T(COARSE_S), T(1), A, G));
    }
  }
}

// ------------------------------------------------------------------------------------------------ FINE_FINAL
// hush.js:530-622
template <class T> T jbw(T frx, T fry, int j, v3<T> nq, T zq, v3<T> n, T z) {  // hush.js:552-558
  T wb = ((j & 1) == 1 ? frx : T(1) - frx) * ((j >> 1) == 1 ? fry : T(1) - fry);
  T dn = std::max(dot3(nq, n), T(0));
  T dn2 = dn * dn;
  T dn4 = dn2 * dn2;
  return wb * std::exp(-std::abs(zq - z) / (T(0.05f) * z + T(1e-3f))) * dn4 * dn4;
}

template <class T> void pass_fine_final(ho_hush *S, const ho_inputs *in) {
  const int W = S->W, H = S->H, cur = S->frame & 1;
  In matI{in->material, W}, emiI{in->emission, W};
  const Img &A0 = S->A0, &key = S->key[cur], &F2 = S->F[2], &F3 = S->F[3];
  auto A = [&](int x, int y) { return A0.ld<T>(clampi(x, 0, W - 1), clampi(y, 0, H - 1)); };
  auto G = [&](int x, int y) { return guide_dec(key.ld<T>(clampi(x, 0, W - 1), clampi(y, 0, H - 1))); };
  const int hsx = (W + 1) / 2, hsy = (H + 1) / 2, qsx = (W + 3) / 4, qsy = (H + 3) / 4;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      v3<T> alb = matI.ld<T>(x, y).rgb(), emi = emiI.ld<T>(x, y).rgb();
      v4<T> gp = G(x, y);
      if (gp.w < T(0)) {
        S->hist[cur].st<T>(x, y, {0, 0, 0, 0});
        S->X.st<T>(x, y, {emi.x, emi.y, emi.z, 0});
        continue;
      }
      int hx = x >> 1, hy = y >> 1;
      v4<T> A1 = filt<T>(1, 1, true, x, y, W, H, S->par1.ld<T>(hx, hy).x, S->par2.ld<T>(hx, hy).x, A, G);
      S->hist[cur].st<T>(x, y, A1);
      v3<T> f = {qf16(A1.x), qf16(A1.y), qf16(A1.z)};
      v3<T> n = gp.rgb();
      T z = gp.w;
      v4<T> pr = S->par0[cur].ld<T>(hx, hy);
      T hposx = (T(x) + T(0.5f)) / T(2) - T(0.5f), hposy = (T(y) + T(0.5f)) / T(2) - T(0.5f);
      T hbx = std::floor(hposx), hby = std::floor(hposy);
      v3<T> uB = v3s(T(0)), uA = v3s(T(0));
      T swh = 0;
      for (int j = 0; j < 4; j++) {
        int qx = (int)hbx + (j & 1), qy = (int)hby + (j >> 1);
        if (qx < 0 || qy < 0 || qx >= hsx || qy >= hsy) continue;
        v4<T> g3 = f3_g<T>(F3, qx, qy);
        if (g3.z < T(0)) continue;
        T w = jbw(hposx - hbx, hposy - hby, j, octDec(v2<T>{g3.x, g3.y}), g3.z, n, z);
        v4<T> a2 = f2_ac<T>(F2, qx, qy);
        swh += w;
        uB = uB + w * S->Bh[0].ld<T>(qx, qy).rgb();
        uA = uA + w * a2.rgb();
      }
      v3<T> ill = f;
      if (swh > T(1e-4f)) ill = uB / swh + pr.w * (f - uA / swh);
      T cposx = (T(x) + T(0.5f)) / T(4) - T(0.5f), cposy = (T(y) + T(0.5f)) / T(4) - T(0.5f);
      T cbx = std::floor(cposx), cby = std::floor(cposy);
      v3<T> uC = v3s(T(0));
      T swq = 0;
      for (int j = 0; j < 4; j++) {
        int qx = (int)cbx + (j & 1), qy = (int)cby + (j >> 1);
        if (qx < 0 || qy < 0 || qx >= qsx || qy >= qsy) continue;
        v4<T> cg = S->CG.ld<T>(qx, qy);
        if (cg.z < T(0)) continue;
        T w = jbw(cposx - cbx, cposy - cby, j, octDec(v2<T>{cg.x, cg.y}), cg.z, n, z);
        swq += w;
        uC = uC + w * S->C[0].ld<T>(qx, qy).rgb();
      }
      v3<T> up = ill;
      if (swq > T(1e-4f)) up = uC / swq;
      ill = ill + (up - ill) * pr.z;
      v3<T> o = ill * alb + emi;
      S->X.st<T>(x, y, {o.x, o.y, o.z, 0});
    }
  }
}

// ------------------------------------------------------------------------------------------------ TAA
// hush.js:625-678
template <class T> v3<T> toYCoCg(v3<T> c) {
  return {c.x * T(0.25f) + c.y * T(0.5f) + c.z * T(0.25f), c.x * T(0.5f) - c.z * T(0.5f),
          -c.x * T(0.25f) + c.y * T(0.5f) - c.z * T(0.25f)};
}
template <class T> v3<T> fromYCoCg(v3<T> c) { return {c.x + c.y - c.z, c.x + c.z, c.x - c.y - c.z}; }
template <class T> v3<T> tm(v3<T> c) { return c / (T(1) + lum(c)); }
template <class T> v3<T> itm(v3<T> c) { return c / std::max(T(1) - lum(c), T(1e-4f)); }

template <class T> void pass_taa(ho_hush *S, const ho_inputs *in) {
  const int W = S->W, H = S->H, cur = S->frame & 1, prev = cur ^ 1;
  In mvI{in->motion, W};
  const Img &Xi = S->X, &pT = S->taa[prev];
  Img &oT = S->taa[cur];
  std::vector<v3<T>> sX((size_t)W * H);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) sX[(size_t)y * W + x] = toYCoCg(tm(Xi.ld<T>(x, y).rgb()));
  auto SX = [&](int x, int y) { return sX[(size_t)clampi(y, 0, H - 1) * W + clampi(x, 0, W - 1)]; };
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      v3<T> cur_c = tm(Xi.ld<T>(x, y).rgb());
      if (S->reset) {
        v3<T> o = itm(cur_c);
        oT.st<T>(x, y, {o.x, o.y, o.z, T(1)});
        continue;
      }
      v3<T> m1 = v3s(T(0));
      for (int j = 0; j < 9; j++) m1 = m1 + SX(x + j % 3 - 1, y + j / 3 - 1);
      m1 = m1 / T(9);
      v3<T> v3_ = v3s(T(0));
      for (int j = 0; j < 9; j++) {
        v3<T> d = SX(x + j % 3 - 1, y + j / 3 - 1) - m1;
        v3_ = v3_ + d * d;
      }
      v3<T> sd = {std::sqrt(std::max(v3_.x / T(9), T(1e-12f))), std::sqrt(std::max(v3_.y / T(9), T(1e-12f))),
                  std::sqrt(std::max(v3_.z / T(9), T(1e-12f)))};
      v4<T> mv = mvI.ld<T>(x, y);
      T szx = T(W), szy = T(H);
      T uvx = (T(x) + T(0.5f) + mv.x) / szx, uvy = (T(y) + T(0.5f) + mv.y) / szy;
      v3<T> res = cur_c;
      if (uvx >= T(0) && uvy >= T(0) && uvx <= T(1) && uvy <= T(1)) {
        T ppx = uvx * szx - T(0.5f), ppy = uvy * szy - T(0.5f);
        T bx = std::floor(ppx), by = std::floor(ppy);
        T fx = ppx - bx, fy = ppy - by;
        v3<T> hist = v3s(T(0));
        for (int j = 0; j < 4; j++) {
          int ox = j & 1, oy = j >> 1;
          T wb = (ox == 1 ? fx : T(1) - fx) * (oy == 1 ? fy : T(1) - fy);
          hist = hist + wb * pT.ld<T>(clampi((int)bx + ox, 0, W - 1), clampi((int)by + oy, 0, H - 1)).rgb();
        }
        v3<T> hh = toYCoCg(tm(hist));
        v3<T> lo = m1 - T(1.25f) * sd, hi = m1 + T(1.25f) * sd;
        hh = vmin(vmax(hh, lo), hi);
        v3<T> hr = fromYCoCg(hh);
        res = hr + (cur_c - hr) * T(0.1f);
      }
      v3<T> o = itm(res);
      oT.st<T>(x, y, {o.x, o.y, o.z, T(1)});
    }
  }
}

template <class T> void run_pass(ho_hush *S, int pass, const ho_inputs *in) {
  switch (pass) {
    case HO_PASS_TEMPORAL: pass_temporal<T>(S, in); break;
    case HO_PASS_INFER: pass_infer<T>(S); break;
    case HO_PASS_MID2: pass_mid<T>(S, 2); break;
    case HO_PASS_MID3: pass_mid<T>(S, 3); break;
    case HO_PASS_COARSE1: pass_coarse1<T>(S); break;
    case HO_PASS_COARSE2: pass_coarse2<T>(S); break;
    case HO_PASS_FINE_FINAL: pass_fine_final<T>(S, in); break;
    case HO_PASS_TAA: pass_taa<T>(S, in); break;
  }
}

}  // namespace

// ================================================================================================ C API
extern "C" {

uint16_t ho_f2h_rz(float f) { return f2h_rz(f); }
float ho_h2f(uint16_t h) { return h2f(h); }
float ho_qf16(float x) { return qf16f(x); }

void ho_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n); else omp_set_num_threads(omp_get_num_procs());
#else
  (void)n;
#endif
}

// hiddenOf (hush.js:22-25)
int ho_hidden_of(long n) {
  for (long h = 1; h <= 256; h++)
    if (h * h + (20 + 12 + 2) * h + 12 == n) return (int)h;
  return 0;
}

ho_hush *ho_hush_create(int width, int height, float exposure, const uint16_t *weights, long n_weights, int fp64) {
  int hd = ho_hidden_of(n_weights);
  if (!hd || width <= 0 || height <= 0) return nullptr;
  ho_hush *S = new ho_hush();
  S->hidden = hd;
  S->fp64 = fp64;
  S->exposure = exposure;
  S->wf.resize(n_weights);
  for (long i = 0; i < n_weights; i++) S->wf[i] = h2f(weights[i]);
  // resize (hush.js:764-794)
  const int W = width, H = height, W2 = (W + 1) / 2, H2 = (H + 1) / 2, W4 = (W2 + 1) / 2, H4 = (H2 + 1) / 2;
  S->W = W; S->H = H; S->W2 = W2; S->H2 = H2; S->W4 = W4; S->H4 = H4;
  S->frame = 0;
  S->reset = true;
  S->A0.alloc(W, H); S->X.alloc(W, H);
  for (int i = 0; i < 2; i++) {
    S->Bh[i].alloc(W2, H2); S->mom[i].alloc(W, H); S->key[i].alloc(W, H); S->hist[i].alloc(W, H);
    S->taa[i].alloc(W, H); S->par0[i].alloc(W2, H2); S->C[i].alloc(W4, H4);
  }
  S->par1.alloc(W2, H2); S->par2.alloc(W2, H2);
  for (int i = 0; i < 4; i++) S->F[i].alloc(W2, H2, 8);
  S->CG.alloc(W4, H4);
  return S;
}

void ho_hush_destroy(ho_hush *h) { delete h; }
void ho_hush_reset(ho_hush *h) { h->reset = true; }
void ho_hush_set_exposure(ho_hush *h, float e) { h->exposure = e; }
int ho_hush_frame(const ho_hush *h) { return h->frame; }

int ho_hush_pass(ho_hush *h, int pass, const ho_inputs *in) {
  if (pass < 0 || pass >= HO_PASS_COUNT) return -1;
  if (h->fp64) run_pass<double>(h, pass, in); else run_pass<float>(h, pass, in);
  return 0;
}

void ho_hush_end_frame(ho_hush *h) {
  h->reset = false;
  h->frame++;
}

const uint16_t *ho_hush_denoise(ho_hush *h, const ho_inputs *in) {
  const int cur = h->frame & 1;
  for (int p = 0; p < HO_PASS_COUNT; p++) ho_hush_pass(h, p, in);
  ho_hush_end_frame(h);
  return h->taa[cur].d.data();
}

uint16_t *ho_hush_buffer(ho_hush *h, int id, int *w, int *hgt, int *channels) {
  Img *b = h->buf(id);
  if (!b) return nullptr;
  if (w) *w = b->w;
  if (hgt) *hgt = b->h;
  if (channels) *channels = b->ch;
  return b->d.data();
}

void ho_hush_set_mlp_half(ho_hush *h, int on) { h->mlp_half = on ? 1 : 0; }

void ho_mlp(const uint16_t *weights, long n_weights, const float *features, float *out, int fp64) {
  int hd = ho_hidden_of(n_weights);
  std::vector<float> wf(n_weights);
  for (long i = 0; i < n_weights; i++) wf[i] = h2f(weights[i]);
  if (fp64 == 2) {
    mlp_half(wf.data(), hd, features, out);
  } else if (fp64) {
    double f[20], o[12];
    for (int i = 0; i < 20; i++) f[i] = features[i];
    mlp<double>(wf.data(), hd, f, o);
    for (int i = 0; i < 12; i++) out[i] = (float)o[i];
  } else {
    mlp<float>(wf.data(), hd, features, out);
  }
}

}  // extern "C"

// ================================================================================================ SVGF
// The SVGF baseline of the reference (src/denoise/svgf.js:12-379), four passes per frame.
struct ho_svgf {
  int W = 0, H = 0, frame = 0;
  bool reset = true;
  int fp64 = 0;
  ho_svgf_opts o;
  Img hist[2], mom[2], tmp, atrous[2], taa[2];
};

namespace {

template <class T> bool svgf_consistent(int qx, int qy, int W, int H, const In &pnd, const In &pmv, v3<T> n, T zPrev,
                                        T obj) {  // svgf.js:31-39
  if (qx < 0 || qy < 0 || qx >= W || qy >= H) return false;
  v4<T> nd = pnd.ld<T>(qx, qy);
  if (nd.w < T(0)) return false;
  if (pmv.ld<T>(qx, qy).z != obj) return false;
  if (std::abs(nd.w - zPrev) > T(0.05f) * zPrev + T(0.01f)) return false;
  if (dot3(nd.rgb(), n) < T(0.9f)) return false;
  return true;
}

template <class T> v3<T> mix3(v3<T> a, v3<T> b, T t) { return a * (T(1) - t) + b * t; }

template <class T> void svgf_frame(ho_svgf *S, const ho_svgf_inputs *in) {
  const int W = S->W, H = S->H, cur = S->frame & 1, prev = cur ^ 1;
  const ho_svgf_opts &O = S->o;
  const bool noHistory = S->reset;
  In rad{in->radiance, W}, ndI{in->normal_depth, W}, mvI{in->motion, W}, matI{in->material, W},
      emiI{in->emission, W}, pnd{in->prev_normal_depth, W}, pmv{in->prev_motion, W};
  auto inside = [&](int x, int y) { return x >= 0 && y >= 0 && x < W && y < H; };
  // TEMPORAL (svgf.js:41-105)
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      v4<T> nd = ndI.ld<T>(x, y);
      if (nd.w < T(0)) { S->tmp.st<T>(x, y, {0, 0, 0, 0}); S->mom[cur].st<T>(x, y, {0, 0, 0, 0}); continue; }
      v4<T> mv = mvI.ld<T>(x, y);
      v3<T> alb = matI.ld<T>(x, y).rgb();
      v3<T> illum = rad.ld<T>(x, y).rgb() / vmax(alb, v3s(T(1e-3f)));
      T l = lum(illum);
      T ppx = T(x) + T(0.5f) + mv.x - T(0.5f), ppy = T(y) + T(0.5f) + mv.y - T(0.5f);
      T flx = std::floor(ppx), fly = std::floor(ppy);
      int bx = (int)flx, by = (int)fly;
      T fx = ppx - flx, fy = ppy - fly;
      T sumW = 0;
      v3<T> hc = v3s(T(0)), hm = v3s(T(0));
      T wts[4] = {(T(1) - fx) * (T(1) - fy), fx * (T(1) - fy), (T(1) - fx) * fy, fx * fy};
      if (!noHistory) {
        for (int i = 0; i < 4; i++) {
          int qx = bx + (i & 1), qy = by + (i >> 1);
          if (svgf_consistent<T>(qx, qy, W, H, pnd, pmv, nd.rgb(), mv.w, mv.z) && wts[i] > T(0)) {
            sumW += wts[i];
            hc = hc + wts[i] * S->hist[prev].ld<T>(qx, qy).rgb();
            hm = hm + wts[i] * S->mom[prev].ld<T>(qx, qy).rgb();
          }
        }
      }
      if (sumW < T(0.01f) && !noHistory) {
        int cx = (int)std::nearbyint(ppx), cy = (int)std::nearbyint(ppy);  // WGSL round(): ties to even
        for (int dy = -1; dy <= 1; dy++) {
          for (int dx = -1; dx <= 1; dx++) {
            int qx = cx + dx, qy = cy + dy;
            if (svgf_consistent<T>(qx, qy, W, H, pnd, pmv, nd.rgb(), mv.w, mv.z)) {
              sumW += T(1);
              hc = hc + S->hist[prev].ld<T>(qx, qy).rgb();
              hm = hm + S->mom[prev].ld<T>(qx, qy).rgb();
            }
          }
        }
      }
      T len = 0;
      v3<T> color = illum;
      T m0 = l, m1 = l * l;
      if (sumW >= T(0.01f)) {
        hc = hc / sumW;
        hm = hm / sumW;
        len = std::min(hm.z + T(1), T(64));
        T ac = std::max(T(O.alpha_color), T(1) / len);
        T am = std::max(T(O.alpha_moments), T(1) / len);
        color = mix3(hc, illum, ac);
        m0 = hm.x * (T(1) - am) + m0 * am;
        m1 = hm.y * (T(1) - am) + m1 * am;
      } else {
        len = 1;
      }
      S->tmp.st<T>(x, y, {color.x, color.y, color.z, 0});
      S->mom[cur].st<T>(x, y, {m0, m1, len, 0});
    }
  }
  // VARIANCE (svgf.js:114-148)
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      v4<T> nd = ndI.ld<T>(x, y);
      if (nd.w < T(0)) { S->atrous[0].st<T>(x, y, {0, 0, 0, 0}); continue; }
      v3<T> c = S->tmp.ld<T>(x, y).rgb();
      v4<T> m = S->mom[cur].ld<T>(x, y);
      if (m.z >= T(4)) {
        S->atrous[0].st<T>(x, y, {c.x, c.y, c.z, std::max(T(0), m.y - m.x * m.x)});
        continue;
      }
      T sw = 0, sm0 = 0, sm1 = 0;
      v3<T> sc = v3s(T(0));
      for (int dy = -3; dy <= 3; dy++) {
        for (int dx = -3; dx <= 3; dx++) {
          int qx = x + dx, qy = y + dy;
          if (!inside(qx, qy)) continue;
          v4<T> ndq = ndI.ld<T>(qx, qy);
          if (ndq.w < T(0)) continue;
          T dist = std::sqrt(T(dx) * T(dx) + T(dy) * T(dy));
          T wz = std::exp(-std::abs(ndq.w - nd.w) / (T(0.02f) * nd.w * dist + T(1e-3f)));
          T wn = std::pow(std::max(T(0), dot3(ndq.rgb(), nd.rgb())), T(O.sigma_n));
          T w = wz * wn;
          sw += w;
          sc = sc + w * S->tmp.ld<T>(qx, qy).rgb();
          v4<T> mq = S->mom[cur].ld<T>(qx, qy);
          sm0 += w * mq.x;
          sm1 += w * mq.y;
        }
      }
      sc = sc / std::max(sw, T(1e-6f));
      sm0 /= std::max(sw, T(1e-6f));
      sm1 /= std::max(sw, T(1e-6f));
      T v = std::max(T(0), sm1 - sm0 * sm0) * T(4) / std::max(m.z, T(1));
      S->atrous[0].st<T>(x, y, {sc.x, sc.y, sc.z, v});
    }
  }
  // ATROUS x iterations (svgf.js:151-217), iteration 0 also writes the colour history
  int src = 0;
  for (int it = 0; it < O.iterations; it++) {
    const int step = 1 << it;
    Img &inC = S->atrous[src], &outC = S->atrous[src ^ 1];
    auto ndc = [&](int qx, int qy) { return ndI.ld<T>(clampi(qx, 0, W - 1), clampi(qy, 0, H - 1)); };
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++) {
      for (int x = 0; x < W; x++) {
        v4<T> nd = ndI.ld<T>(x, y);
        if (nd.w < T(0)) {
          outC.st<T>(x, y, {0, 0, 0, 0});
          if (it == 0) S->hist[cur].st<T>(x, y, {0, 0, 0, 0});
          continue;
        }
        v4<T> center = inC.ld<T>(x, y);
        static const float k3[3] = {0.25f, 0.5f, 0.25f};
        T gv = 0;
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++)
            gv += T(k3[dx + 1]) * T(k3[dy + 1]) * inC.ld<T>(clampi(x + dx, 0, W - 1), clampi(y + dy, 0, H - 1)).w;
        T lp = lum(center.rgb());
        T denomL = T(O.sigma_l) * std::sqrt(std::max(gv, T(0))) + T(1e-6f);
        T z = nd.w;
        T zl = ndc(x - 1, y).w, zr = ndc(x + 1, y).w, zu = ndc(x, y - 1).w, zd = ndc(x, y + 1).w;
        T gx = std::min(zr > T(0) ? std::abs(zr - z) : T(1e9f), zl > T(0) ? std::abs(zl - z) : T(1e9f));
        T gy = std::min(zd > T(0) ? std::abs(zd - z) : T(1e9f), zu > T(0) ? std::abs(zu - z) : T(1e9f));
        T zg = std::min(std::max(gx, gy), z);
        static const float h[5] = {1.0f / 16, 1.0f / 4, 3.0f / 8, 1.0f / 4, 1.0f / 16};
        T sw = T(h[2]) * T(h[2]);
        v3<T> sc = center.rgb() * sw;
        T sv = center.w * sw * sw;
        for (int dy = -2; dy <= 2; dy++) {
          for (int dx = -2; dx <= 2; dx++) {
            if (dx == 0 && dy == 0) continue;
            int qx = x + dx * step, qy = y + dy * step;
            if (!inside(qx, qy)) continue;
            v4<T> ndq = ndI.ld<T>(qx, qy);
            if (ndq.w < T(0)) continue;
            v4<T> cq = inC.ld<T>(qx, qy);
            T dist = std::sqrt(T(dx) * T(dx) + T(dy) * T(dy)) * T(step);
            T wz = std::abs(ndq.w - nd.w) / (T(O.sigma_z) * zg * dist + T(1e-3f));
            T wn = std::pow(std::max(T(0), dot3(ndq.rgb(), nd.rgb())), T(O.sigma_n));
            T wl = std::abs(lum(cq.rgb()) - lp) / denomL;
            T w = T(h[dx + 2]) * T(h[dy + 2]) * wn * std::exp(-wz - wl);
            sw += w;
            sc = sc + w * cq.rgb();
            sv += w * w * cq.w;
          }
        }
        v3<T> oc = sc / sw;
        outC.st<T>(x, y, {oc.x, oc.y, oc.z, sv / (sw * sw)});
        if (it == 0) S->hist[cur].st<T>(x, y, {oc.x, oc.y, oc.z, 0});
      }
    }
    src ^= 1;
  }
  // RESOLVE: remodulate + TAA (svgf.js:219-271). The reference samples the history with a hardware bilinear
  // sampler (clamp-to-edge); this restatement uses exact f32 bilinear weights at the same texel positions.
  const Img &il = S->atrous[src], &pT = S->taa[prev];
  Img &oT = S->taa[cur];
  auto remod = [&](int qx, int qy) {
    int cx = clampi(qx, 0, W - 1), cy = clampi(qy, 0, H - 1);
    return il.ld<T>(cx, cy).rgb() * matI.ld<T>(cx, cy).rgb() + emiI.ld<T>(cx, cy).rgb();
  };
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      v3<T> curc = tm(remod(x, y));
      if (!O.taa) { v3<T> r = itm(curc); oT.st<T>(x, y, {r.x, r.y, r.z, T(1)}); continue; }
      v3<T> m1 = v3s(T(0)), m2 = v3s(T(0));
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          v3<T> c = toYCoCg(tm(remod(x + dx, y + dy)));
          m1 = m1 + c;
          m2 = m2 + c * c;
        }
      m1 = m1 / T(9);
      m2 = m2 / T(9);
      v3<T> d2 = m2 - m1 * m1;
      v3<T> sd = {std::sqrt(std::max(d2.x, T(0))), std::sqrt(std::max(d2.y, T(0))), std::sqrt(std::max(d2.z, T(0)))};
      v4<T> mv = mvI.ld<T>(x, y);
      T uvx = (T(x) + T(0.5f) + mv.x) / T(W), uvy = (T(y) + T(0.5f) + mv.y) / T(H);
      T a = T(O.taa_alpha);
      v3<T> res = curc;
      if (uvx >= T(0) && uvy >= T(0) && uvx <= T(1) && uvy <= T(1) && !S->reset) {
        T ppx = uvx * T(W) - T(0.5f), ppy = uvy * T(H) - T(0.5f);
        T bx = std::floor(ppx), by = std::floor(ppy);
        T fx = ppx - bx, fy = ppy - by;
        v3<T> hist = v3s(T(0));
        for (int j = 0; j < 4; j++) {
          int ox = j & 1, oy = j >> 1;
          T wb = (ox == 1 ? fx : T(1) - fx) * (oy == 1 ? fy : T(1) - fy);
          hist = hist + wb * pT.ld<T>(clampi((int)bx + ox, 0, W - 1), clampi((int)by + oy, 0, H - 1)).rgb();
        }
        v3<T> hh = toYCoCg(tm(hist));
        hh = vmin(vmax(hh, m1 - T(1.25f) * sd), m1 + T(1.25f) * sd);
        res = mix3(fromYCoCg(hh), curc, a);
      }
      v3<T> r = itm(res);
      oT.st<T>(x, y, {r.x, r.y, r.z, T(1)});
    }
  }
}

}  // namespace

extern "C" {

ho_svgf *ho_svgf_create(int width, int height, const ho_svgf_opts *opts, int fp64) {
  if (width <= 0 || height <= 0) return nullptr;
  ho_svgf *S = new ho_svgf();
  S->W = width; S->H = height; S->fp64 = fp64;
  S->o = ho_svgf_opts{5, 4.0f, 128.0f, 1.0f, 0.2f, 0.2f, 0.1f, 1};
  if (opts) S->o = *opts;
  for (int i = 0; i < 2; i++) {
    S->hist[i].alloc(width, height); S->mom[i].alloc(width, height); S->atrous[i].alloc(width, height);
    S->taa[i].alloc(width, height);
  }
  S->tmp.alloc(width, height);
  return S;
}
void ho_svgf_destroy(ho_svgf *s) { delete s; }
void ho_svgf_reset(ho_svgf *s) { s->reset = true; }
const uint16_t *ho_svgf_encode(ho_svgf *s, const ho_svgf_inputs *in) {
  const int cur = s->frame & 1;
  if (s->fp64) svgf_frame<double>(s, in); else svgf_frame<float>(s, in);
  s->reset = false;
  s->frame++;
  return s->taa[cur].d.data();
}

}  // extern "C"
