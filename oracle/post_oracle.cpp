// CPU oracle of the demo's display post (src/demo/post.js): TEST INFRASTRUCTURE ONLY.
//
// A scalar f32 restatement of the four render pipelines of post.js: COMPOSITE (post.js:21-39), DOWN with the Karis
// average on the first level (43-65), UP added onto the next larger level (68-81) and FINAL: bloom mix, vignette,
// AgX, sRGB and the divider line (84-133), scheduled as Post.encode does (191-210) over LEVELS = 6 (135) levels of
// max(1, size >> i) (165-167). Only the tests load it; the CUDA path (hush_b200/csrc/post.cu) never does.
//
// Parity status: the reference ships no golden outputs for post.js and its render pipelines cannot run here
// (WebGPU); parity is unpinned by reference outputs. Choices the WGSL leaves to the platform, made the same way in
// the CUDA path: a fragment at pixel (x, y) has uv = ((x + 0.5) / W, (y + 0.5) / H) (the full-screen triangle of
// post.js:10-17); the clamp-to-edge linear sampler (post.js:154) interpolates with exact f32 weights (hardware
// samplers use 8-bit fractions); rgba16float render targets are written rounded toward zero like the denoiser's
// storage writes, additive blending adds in f32 before that rounding; the 8-bit target rounds to nearest.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "hush_oracle.h"

namespace {

inline uint32_t fb(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

float h2f(uint16_t h) {
  uint32_t s = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  if (e == 0) { float v = (float)m * 5.9604644775390625e-08f; return s ? -v : v; }
  if (e == 31) return bf(s | 0x7f800000u | (m << 13));
  return bf(s | ((e + 112u) << 23) | (m << 13));
}

uint16_t f2h_rz(float f) {
  uint32_t x = fb(f);
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

struct V3 { float x, y, z; };
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 mix(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }  // WGSL mix: e1 * (1 - e3) + e2 * e3
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

struct Img {
  int w = 0, h = 0;
  uint16_t *p = nullptr;  // 4 x u16 per texel
  V3 load(int x, int y) const {
    const uint16_t *t = p + 4 * ((size_t)y * w + x);
    return {h2f(t[0]), h2f(t[1]), h2f(t[2])};
  }
  void store(int x, int y, V3 c, float a) {
    uint16_t *t = p + 4 * ((size_t)y * w + x);
    t[0] = f2h_rz(c.x); t[1] = f2h_rz(c.y); t[2] = f2h_rz(c.z); t[3] = f2h_rz(a);
  }
  // textureSampleLevel with the clamp-to-edge linear sampler
  V3 sample(float u, float v) const {
    const float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
    const float x0 = std::floor(x), y0 = std::floor(y);
    const float fx = x - x0, fy = y - y0;
    const int ix = (int)x0, iy = (int)y0;
    const int xa = std::clamp(ix, 0, w - 1), xb = std::clamp(ix + 1, 0, w - 1);
    const int ya = std::clamp(iy, 0, h - 1), yb = std::clamp(iy + 1, 0, h - 1);
    const V3 top = load(xa, ya) * (1.0f - fx) + load(xb, ya) * fx;
    const V3 bot = load(xa, yb) * (1.0f - fx) + load(xb, yb) * fx;
    return top * (1.0f - fy) + bot * fy;
  }
};

inline float kw(V3 c) { return 1.0f / (1.0f + dot(c, V3{0.2126f, 0.7152f, 0.0722f})); }

// mat3x3f(c0, c1, c2) * v with columns c0..c2 (WGSL matrices are column-major)
inline V3 mul(const float m[9], V3 v) {
  return {m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
          m[2] * v.x + m[5] * v.y + m[8] * v.z};
}

V3 agx_contrast(V3 x) {
  auto f = [](float x) {
    const float x2 = x * x, x4 = x2 * x2;
    return 15.5f * x4 * x2 - 40.14f * x4 * x + 31.96f * x4 - 6.868f * x2 * x + 0.4298f * x2 + 0.1191f * x - 0.00232f;
  };
  return {f(x.x), f(x.y), f(x.z)};
}

V3 agx(V3 c0) {
  static const float to2020[9] = {0.6274f, 0.0691f, 0.0164f, 0.3293f, 0.9195f, 0.0880f, 0.0433f, 0.0113f, 0.8956f};
  static const float toSrgb[9] = {1.6605f, -0.1246f, -0.0182f, -0.5876f, 1.1329f, -0.1006f, -0.0728f, -0.0083f, 1.1187f};
  static const float inset[9] = {0.856627153315983f, 0.137318972929847f, 0.11189821299995f,
                                 0.0951212405381588f, 0.761241990602591f, 0.0767994186031903f,
                                 0.0482516061458583f, 0.101439036467562f, 0.811302368396859f};
  static const float outset[9] = {1.1271005818144368f, -0.1413297634984383f, -0.14132976349843826f,
                                  -0.11060664309660323f, 1.157823702216272f, -0.11060664309660294f,
                                  -0.016493938717834573f, -0.016493938717834257f, 1.2519364065950405f};
  const float minEv = -12.47393f, maxEv = 4.026069f;
  V3 c = mul(inset, mul(to2020, c0));
  auto lg = [&](float v) {
    return std::min(std::max((std::log2(std::max(v, 1e-10f)) - minEv) / (maxEv - minEv), 0.0f), 1.0f);
  };
  c = {lg(c.x), lg(c.y), lg(c.z)};
  c = agx_contrast(c);
  const float l = dot(c, V3{0.2126f, 0.7152f, 0.0722f});
  c = {std::pow(std::max(c.x, 0.0f), 1.22f), std::pow(std::max(c.y, 0.0f), 1.22f), std::pow(std::max(c.z, 0.0f), 1.22f)};
  c = V3{l, l, l} + (c - V3{l, l, l}) * 1.15f;
  c = mul(outset, c);
  c = {std::pow(std::max(0.0f, c.x), 2.2f), std::pow(std::max(0.0f, c.y), 2.2f), std::pow(std::max(0.0f, c.z), 2.2f)};
  c = mul(toSrgb, c);
  return {std::min(std::max(c.x, 0.0f), 1.0f), std::min(std::max(c.y, 0.0f), 1.0f), std::min(std::max(c.z, 0.0f), 1.0f)};
}

inline float srgb1(float c) { return c <= 0.0031308f ? c * 12.92f : 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f; }

}  // namespace

extern "C" int ho_post_level_size(int width, int height, int level, int *w, int *h) {
  if (level < 1 || level > HO_POST_LEVELS) return -1;
  *w = std::max(1, width >> level);
  *h = std::max(1, height >> level);
  return 0;
}

extern "C" int ho_post(const ho_post_args *a, uint16_t *hdr_out, uint16_t *levels_out, float *out_f32,
                       uint8_t *out_rgba8) {
  const int W = a->width, H = a->height;
  if (W <= 0 || H <= 0 || !a->left || !a->right) return -1;
  const uint16_t *midp = a->mid ? a->mid : a->right;
  std::vector<uint16_t> hdr_buf(hdr_out ? 0 : (size_t)W * H * 4);
  Img hdr{W, H, hdr_out ? hdr_out : hdr_buf.data()};
  Img L{W, H, const_cast<uint16_t *>(a->left)}, R{W, H, const_cast<uint16_t *>(a->right)},
      M{W, H, const_cast<uint16_t *>(midp)};
  // COMPOSITE (post.js:27-38)
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      int px = x;
      const float u = ((float)x + 0.5f) / (float)W;
      if (a->same) px = px - (std::min(px * 3 / W, 2) - 1) * (W / 3);
      V3 c = R.load(px, y);
      if (u < a->split2) c = M.load(px, y);
      if (u < a->split) c = L.load(px, y);
      c = {std::max(c.x, 0.0f) * a->exposure, std::max(c.y, 0.0f) * a->exposure, std::max(c.z, 0.0f) * a->exposure};
      hdr.store(x, y, c, 1.0f);
    }
  // the bloom chain (post.js:197-204)
  size_t total = 0;
  int lw[HO_POST_LEVELS], lh[HO_POST_LEVELS];
  for (int i = 0; i < HO_POST_LEVELS; i++) {
    ho_post_level_size(W, H, i + 1, &lw[i], &lh[i]);
    total += (size_t)lw[i] * lh[i] * 4;
  }
  std::vector<uint16_t> lev_buf(levels_out ? 0 : total);
  uint16_t *lp = levels_out ? levels_out : lev_buf.data();
  Img lev[HO_POST_LEVELS];
  for (int i = 0; i < HO_POST_LEVELS; i++) {
    lev[i] = Img{lw[i], lh[i], lp};
    lp += (size_t)lw[i] * lh[i] * 4;
  }
  const Img *src = &hdr;
  for (int i = 0; i < HO_POST_LEVELS; i++) {  // DOWN (post.js:50-64)
    Img &d = lev[i];
    const float tx = 1.0f / (float)src->w, ty = 1.0f / (float)src->h;
    for (int y = 0; y < d.h; y++)
      for (int x = 0; x < d.w; x++) {
        const float u = ((float)x + 0.5f) / (float)d.w, v = ((float)y + 0.5f) / (float)d.h;
        auto s = [&](float ox, float oy) { return src->sample(u + ox * tx, v + oy * ty); };
        const V3 A = s(-2, -2), B = s(0, -2), C = s(2, -2), D = s(-2, 0), E = s(0, 0), F = s(2, 0), G = s(-2, 2),
                 Hh = s(0, 2), K = s(2, 2), J = s(-1, -1), Ll = s(1, -1), Mm = s(-1, 1), N = s(1, 1);
        V3 o;
        if (i == 0) {
          const V3 g0 = (A + B + D + E) * 0.25f, g1 = (B + C + E + F) * 0.25f, g2 = (D + E + G + Hh) * 0.25f,
                   g3 = (E + F + Hh + K) * 0.25f, g4 = (J + Ll + Mm + N) * 0.25f;
          const float w0 = kw(g0) * 0.125f, w1 = kw(g1) * 0.125f, w2 = kw(g2) * 0.125f, w3 = kw(g3) * 0.125f,
                      w4 = kw(g4) * 0.5f;
          o = (g0 * w0 + g1 * w1 + g2 * w2 + g3 * w3 + g4 * w4) / (w0 + w1 + w2 + w3 + w4);
        } else {
          o = E * 0.125f + (A + C + G + K) * 0.03125f + (B + D + F + Hh) * 0.0625f + (J + Ll + Mm + N) * 0.125f;
        }
        d.store(x, y, o, 1.0f);
      }
    src = &d;
  }
  for (int i = HO_POST_LEVELS - 1; i > 0; i--) {  // UP, blended with one + one (post.js:74-80, 149, 203)
    const Img &s = lev[i];
    Img &d = lev[i - 1];
    const float tx = 1.0f / (float)s.w, ty = 1.0f / (float)s.h;
    for (int y = 0; y < d.h; y++)
      for (int x = 0; x < d.w; x++) {
        const float u = ((float)x + 0.5f) / (float)d.w, v = ((float)y + 0.5f) / (float)d.h;
        auto t = [&](float ox, float oy) { return s.sample(u + ox * tx, v + oy * ty); };
        V3 o = t(0, 0) * 4.0f;
        o = o + (t(-1, 0) + t(1, 0) + t(0, -1) + t(0, 1)) * 2.0f;
        o = o + t(-1, -1) + t(1, -1) + t(-1, 1) + t(1, 1);
        o = o / 16.0f;
        const V3 dst = d.load(x, y);
        const uint16_t *dt = d.p + 4 * ((size_t)y * d.w + x);
        d.store(x, y, dst + o, h2f(dt[3]) + 1.0f);
      }
  }
  // FINAL (post.js:116-132) into the out_width x out_height target
  const Img &b = lev[0];
  const int OW = a->out_width, OH = a->out_height;
  const float tx = 1.0f / (float)b.w, ty = 1.0f / (float)b.h;
  for (int y = 0; y < OH; y++)
    for (int x = 0; x < OW; x++) {
      const float u = ((float)x + 0.5f) / (float)OW, v = ((float)y + 0.5f) / (float)OH;
      V3 c = hdr.sample(u, v);
      V3 bl = b.sample(u, v) * 4.0f;
      bl = bl + (b.sample(u - tx, v) + b.sample(u + tx, v) + b.sample(u, v - ty) + b.sample(u, v + ty)) * 2.0f;
      bl = bl + b.sample(u - tx, v - ty) + b.sample(u + tx, v + ty) + b.sample(u + tx, v - ty) + b.sample(u - tx, v + ty);
      c = mix(c, bl / 16.0f, a->bloom);
      const float qx = (u - 0.5f) * 1.0f, qy = (v - 0.5f) * 0.75f;
      c = c * mixf(1.0f, 1.0f - (qx * qx + qy * qy) * 1.6f, a->vignette);
      const V3 t = agx(c);
      V3 o = {srgb1(t.x), srgb1(t.y), srgb1(t.z)};
      if (a->line > 0.0f && std::min(std::fabs(u - a->split), std::fabs(u - a->split2)) * (float)OW < a->line)
        o = mix(o, V3{1.0f, 1.0f, 1.0f}, 0.85f);
      const size_t k = 4 * ((size_t)y * OW + x);
      if (out_f32) { out_f32[k] = o.x; out_f32[k + 1] = o.y; out_f32[k + 2] = o.z; out_f32[k + 3] = 1.0f; }
      if (out_rgba8) {
        auto q = [](float v) { return (uint8_t)std::nearbyint(std::min(std::max(v, 0.0f), 1.0f) * 255.0f); };
        out_rgba8[k] = q(o.x); out_rgba8[k + 1] = q(o.y); out_rgba8[k + 2] = q(o.z); out_rgba8[k + 3] = 255;
      }
    }
  return 0;
}
