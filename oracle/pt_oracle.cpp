// CPU oracle of the reference's path tracer: TEST INFRASTRUCTURE ONLY.
//
// A scalar restatement of src/pt/pathtracer.wgsl.js (tracePath and everything it calls, main() at 648-672), of the
// BVH builder, refit and packing of src/pt/bvh.js, of the per-triangle texture LOD of src/pt/scene.js:178-208 and of
// the environment-map preparation of src/pt/envmap.js:22-105. Only the tests load it; the CUDA path
// (hush_b200/csrc/pt_*.cu) never does.
//
// Arithmetic follows the sources: WGSL code in f32 (no FMA contraction, see the Makefile), JavaScript code in double
// with f32 storage where the JavaScript writes a Float32Array. WGSL builtins come from libm (sin, cos, acos, atan2,
// log2, pow, sqrt). Texture sampling (left to the platform by WGSL) is trilinear / bilinear with exact f32 weights,
// texel centres at (i + 0.5) / size, repeat or clamp-to-edge addressing as the reference's samplers ask.
//
// Parity status: the reference ships no golden outputs for the path tracer and cannot run here (WebGPU); the oracle
// is pinned by known-answer tests (tests/test_pt_oracle.py) only: parity unpinned by reference outputs.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "hush_oracle.h"

namespace {

constexpr float PI = 3.14159265358979f;
constexpr float INF = 1e30f;
constexpr uint32_t NONE = 0xffffffffu;
constexpr int STACK = 32;
constexpr uint32_t GW = HO_PT_ENV_GW, GH = HO_PT_ENV_GH;

inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

float h2f(uint16_t h) {
  uint32_t s = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  if (e == 0) { float v = (float)m * 5.9604644775390625e-08f; return s ? -v : v; }
  if (e == 31) return bitsf(s | 0x7f800000u | (m << 13));
  return bitsf(s | ((e + 112u) << 23) | (m << 13));
}

uint16_t f2h_rz(float f) {  // rgba16float storage write, rounded toward zero
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

// ------------------------------------------------------------------------------------------------ f32 vectors
struct V3 { float x = 0, y = 0, z = 0; };
inline V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
inline V3 operator/(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) { return a / length(a); }
inline V3 reflect(V3 d, V3 n) { return d - n * (2.0f * dot(n, d)); }
inline V3 mix(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
inline V3 mix(V3 a, V3 b, V3 t) { return a * (v3(1, 1, 1) - t) + b * t; }
inline V3 vmin(V3 a, V3 b) { return v3(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)); }
inline V3 vmax(V3 a, V3 b) { return v3(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)); }
inline float lum(V3 c) { return dot(c, v3(0.2126f, 0.7152f, 0.0722f)); }
inline float clampf(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }
inline V3 ld3(const float *p) { return v3(p[0], p[1], p[2]); }

// mat3x3f with columns c0, c1, c2
struct M3 { V3 c0, c1, c2; };
inline V3 mul(const M3 &m, V3 v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }
inline V3 mulT(const M3 &m, V3 v) { return v3(dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)); }  // transpose(m) * v

// mat4x4f (column-major elements) * vec4
inline void mul4(const float *m, const float p[4], float c[4]) {
  for (int r = 0; r < 4; r++) c[r] = m[r] * p[0] + m[4 + r] * p[1] + m[8 + r] * p[2] + m[12 + r] * p[3];
}

// ------------------------------------------------------------------------------------------------ RNG
inline uint32_t pcg(uint32_t v) {
  const uint32_t s = v * 747796405u + 2891336453u;
  const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}

struct Tracer {
  const ho_pt_scene &S;
  const ho_pt_frame &F;
  uint32_t rng = 0;

  float rnd() {
    rng = pcg(rng);
    return (float)(rng >> 8u) * (1.0f / 16777216.0f);
  }

  // ---------------------------------------------------------------------------------------- texture sampling
  static int wrap(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }
  // rgba8 texel of the texture array (layer, mip), repeat addressing
  void texel(int layer, int mip, int x, int y, float o[4]) const {
    size_t off = 0, per_layer = 0;
    for (int m = 0; m < HO_PT_TEX_MIPS; m++) {
      const size_t s = (size_t)std::max(1, HO_PT_TEX_SIZE >> m);
      if (m < mip) off += s * s * 4;
      per_layer += s * s * 4;
    }
    const int s = std::max(1, HO_PT_TEX_SIZE >> mip);
    const uint8_t *t = S.tex + per_layer * layer + off + ((size_t)wrap(y, s) * s + wrap(x, s)) * 4;
    for (int k = 0; k < 4; k++) o[k] = (float)t[k] / 255.0f;
  }
  void bilinear_tex(int layer, int mip, float u, float v, float o[4]) const {
    const int s = std::max(1, HO_PT_TEX_SIZE >> mip);
    const float x = u * (float)s - 0.5f, y = v * (float)s - 0.5f;
    const float x0 = std::floor(x), y0 = std::floor(y), fx = x - x0, fy = y - y0;
    float a[4], b[4], c[4], d[4];
    texel(layer, mip, (int)x0, (int)y0, a);
    texel(layer, mip, (int)x0 + 1, (int)y0, b);
    texel(layer, mip, (int)x0, (int)y0 + 1, c);
    texel(layer, mip, (int)x0 + 1, (int)y0 + 1, d);
    for (int k = 0; k < 4; k++) {
      const float top = a[k] * (1.0f - fx) + b[k] * fx, bot = c[k] * (1.0f - fx) + d[k] * fx;
      o[k] = top * (1.0f - fy) + bot * fy;
    }
  }
  // textureSampleLevel(texArr, samp, uv, layer, lod): trilinear, repeat (scene.js:329-331)
  void sample_tex(float u, float v, int layer, float lod, float o[4]) const {
    const float l = clampf(lod, 0.0f, (float)(HO_PT_TEX_MIPS - 1));
    const int m0 = (int)std::floor(l), m1 = std::min(m0 + 1, HO_PT_TEX_MIPS - 1);
    const float t = l - (float)m0;
    float a[4], b[4];
    bilinear_tex(layer, m0, u, v, a);
    bilinear_tex(layer, m1, u, v, b);
    for (int k = 0; k < 4; k++) o[k] = a[k] * (1.0f - t) + b[k] * t;
  }
  // textureSampleLevel(envTex, envSamp, uv, 0): bilinear, repeat in u, clamp-to-edge in v (pathtracer.js:22)
  V3 sample_env(float u, float v) const {
    const int W = S.env_w, H = S.env_h;
    const float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
    const float x0 = std::floor(x), y0 = std::floor(y), fx = x - x0, fy = y - y0;
    auto at = [&](int xi, int yi) {
      const uint16_t *t = S.env + ((size_t)std::clamp(yi, 0, H - 1) * W + wrap(xi, W)) * 4;
      return v3(h2f(t[0]), h2f(t[1]), h2f(t[2]));
    };
    const V3 top = at((int)x0, (int)y0) * (1.0f - fx) + at((int)x0 + 1, (int)y0) * fx;
    const V3 bot = at((int)x0, (int)y0 + 1) * (1.0f - fx) + at((int)x0 + 1, (int)y0 + 1) * fx;
    return top * (1.0f - fy) + bot * fy;
  }

  // ---------------------------------------------------------------------------------------- materials
  struct Mat {
    float base[4], emissive[4], pbr[4];
    int32_t tex[4];
    float uv[4];
  };
  Mat mat(uint32_t i) const {
    Mat m;
    std::memcpy(&m, S.mats + (size_t)i * 20, sizeof(Mat));
    return m;
  }
  const float *vert(uint32_t i) const { return S.verts + (size_t)i * 12; }
  const uint32_t *tri_idx(uint32_t t) const { return S.tri_idx + (size_t)t * 4; }

  // ---------------------------------------------------------------------------------------- traversal
  struct Hit { float t; uint32_t tri; float u, v; int light; };

  static float slab(V3 o, V3 inv, V3 bmin, V3 bmax, float tmax) {
    const V3 t0 = (bmin - o) * inv, t1 = (bmax - o) * inv;
    const float tn = std::max(std::max(std::min(t0.x, t1.x), std::min(t0.y, t1.y)), std::min(t0.z, t1.z));
    const float tf = std::min(std::min(std::max(t0.x, t1.x), std::max(t0.y, t1.y)), std::max(t0.z, t1.z));
    if (tn <= tf && tf > 0.0f && tn < tmax) return std::max(tn, 0.0f);
    return INF;
  }

  bool alpha_pass(uint32_t tri, float u, float v) const {
    const uint32_t *ti = tri_idx(tri);
    const Mat m = mat(ti[3] & 0xffffu);
    if (m.base[3] <= 0.0f || m.tex[0] < 0) return true;
    const float w = 1.0f - u - v;
    const float uu = vert(ti[0])[3] * w + vert(ti[1])[3] * u + vert(ti[2])[3] * v;
    const float vv = vert(ti[0])[11] * w + vert(ti[1])[11] * u + vert(ti[2])[11] * v;
    float c[4];
    sample_tex(uu * m.uv[0], vv * m.uv[1], m.tex[0], 2.0f, c);
    return c[3] >= m.base[3];
  }

  V3 intersect_tri(V3 o, V3 d, uint32_t tri, float tmax) const {
    const float *a = S.tris + (size_t)tri * 12;
    const V3 v0 = ld3(a), e1 = ld3(a + 4), e2 = ld3(a + 8);
    const V3 p = cross(d, e2);
    const float det = dot(e1, p);
    if (std::fabs(det) < 1e-12f) return v3(INF, 0, 0);
    const float inv = 1.0f / det;
    const V3 s = o - v0;
    const float u = dot(s, p) * inv;
    if (u < 0.0f || u > 1.0f) return v3(INF, 0, 0);
    const V3 q = cross(s, e1);
    const float v = dot(d, q) * inv;
    if (v < 0.0f || u + v > 1.0f) return v3(INF, 0, 0);
    const float t = dot(e2, q) * inv;
    if (t <= 1e-4f || t >= tmax) return v3(INF, 0, 0);
    if (a[3] > 0.0f && !alpha_pass(tri, u, v)) return v3(INF, 0, 0);
    return v3(t, u, v);
  }

  Hit trace_bvh(V3 o, V3 d, float tmax_in, bool shadow) const {
    Hit h{tmax_in, NONE, 0.0f, 0.0f, -1};
    auto safe = [](float x) { return std::fabs(x) < 1e-9f ? 1e-9f : x; };
    const V3 inv = v3(1.0f / safe(d.x), 1.0f / safe(d.y), 1.0f / safe(d.z));
    uint32_t stack[STACK];
    for (uint32_t b = 0; b < F.counts[0]; b++) {
      const ho_pt_blas &bl = F.blas[b];
      if (shadow && (bl.flags & 2u) != 0u) continue;
      uint32_t sp = 0, node = 0;
      for (;;) {
        const float *n = S.nodes + (size_t)(bl.node_offset + node) * 16;
        float tl = slab(o, inv, ld3(n), ld3(n + 4), h.t);
        float tr = slab(o, inv, ld3(n + 8), ld3(n + 12), h.t);
        const uint32_t lc = fbits(n[7]), rc = fbits(n[15]);
        if (lc > 0u && tl < INF) {
          const uint32_t first = bl.tri_offset + fbits(n[3]);
          for (uint32_t i = 0; i < lc; i++) {
            const V3 r = intersect_tri(o, d, first + i, h.t);
            if (r.x < h.t) {
              h.t = r.x; h.u = r.y; h.v = r.z; h.tri = first + i;
              if (shadow) return h;
            }
          }
          tl = INF;
        }
        if (rc > 0u && tr < h.t) {
          const uint32_t first = bl.tri_offset + fbits(n[11]);
          for (uint32_t i = 0; i < rc; i++) {
            const V3 r = intersect_tri(o, d, first + i, h.t);
            if (r.x < h.t) {
              h.t = r.x; h.u = r.y; h.v = r.z; h.tri = first + i;
              if (shadow) return h;
            }
          }
          tr = INF;
        }
        const uint32_t l = fbits(n[3]), r = fbits(n[11]);
        if (tl < h.t && tr < h.t) {
          if (tl <= tr) { node = l; stack[sp] = r; } else { node = r; stack[sp] = l; }
          sp = std::min(sp + 1u, (uint32_t)STACK - 1u);
        } else if (tl < h.t) {
          node = l;
        } else if (tr < h.t) {
          node = r;
        } else {
          if (sp == 0u) break;
          sp--;
          node = stack[sp];
        }
      }
    }
    return h;
  }

  static float sphere_t(V3 o, V3 d, V3 c, float r) {
    const V3 oc = o - c;
    const float b = dot(oc, d);
    const float cc = dot(oc, oc) - r * r;
    const float disc = b * b - cc;
    if (disc < 0.0f) return INF;
    const float s = std::sqrt(disc);
    float t = -b - s;
    if (t < 1e-4f) t = -b + s;
    if (t < 1e-4f) return INF;
    return t;
  }

  Hit trace_scene(V3 o, V3 d) const {
    Hit h = trace_bvh(o, d, INF, false);
    for (uint32_t i = 0; i < F.counts[1]; i++) {
      const ho_pt_light &L = F.lights[i];
      if (L.params[0] != 1.0f) continue;
      const float t = sphere_t(o, d, ld3(L.pos), L.pos[3]);
      if (t < h.t) { h.t = t; h.light = (int)i; h.tri = NONE; }
    }
    return h;
  }

  bool visible(V3 o, V3 d, float tmax) const { return trace_bvh(o, d, tmax, true).tri == NONE; }

  // ---------------------------------------------------------------------------------------- environment
  V3 env_local(V3 d) const { return v3(F.env[1] * d.x - F.env[2] * d.z, d.y, F.env[2] * d.x + F.env[1] * d.z); }
  static void env_uv(V3 l, float &u, float &v) {
    u = std::atan2(l.z, l.x) * (0.5f / PI) + 0.5f;
    v = std::acos(clampf(l.y, -1.0f, 1.0f)) / PI;
  }
  float env_pdf(V3 d) const {
    const V3 l = env_local(d);
    float u, v;
    env_uv(l, u, v);
    const float st = std::sqrt(std::max(0.0f, 1.0f - l.y * l.y));
    if (st < 1e-5f) return 0.0f;
    const uint32_t cx = std::min((uint32_t)(u * (float)GW), GW - 1u), cy = std::min((uint32_t)(v * (float)GH), GH - 1u);
    return S.env_table[(size_t)(cy * GW + cx) * 4 + 2] * (float)(GW * GH) / (2.0f * PI * PI * st);
  }
  // sampleEnv: direction and pdf (w)
  void sample_env_dir(V3 &d, float &pdf) {
    const uint32_t N = GW * GH;
    uint32_t i = std::min((uint32_t)(rnd() * (float)N), N - 1u);
    const float *a = S.env_table + (size_t)i * 4;
    if (rnd() >= a[0]) i = fbits(a[1]);
    const float r1 = rnd();
    const float u = ((float)(i % GW) + r1) / (float)GW;
    const float r2 = rnd();
    const float v = ((float)(i / GW) + r2) / (float)GH;
    const float phi = (u - 0.5f) * 2.0f * PI, th = v * PI;
    const float st = std::sin(th);
    const V3 l = v3(std::cos(phi) * st, std::cos(th), std::sin(phi) * st);
    d = v3(F.env[1] * l.x + F.env[2] * l.z, l.y, -F.env[2] * l.x + F.env[1] * l.z);
    pdf = st > 1e-5f ? S.env_table[(size_t)i * 4 + 2] * (float)N / (2.0f * PI * PI * st) : 0.0f;
  }
  V3 sky(V3 d) const {
    if (F.env[3] > 0.5f) {
      float u, v;
      env_uv(env_local(d), u, v);
      return sample_env(u, v) * F.env[0];
    }
    const float y = d.y;
    V3 c;
    if (y >= 0.0f) c = mix(ld3(F.sky_horizon), ld3(F.sky_zenith), std::pow(clampf(y, 0.0f, 1.0f), 0.6f));
    else c = mix(ld3(F.sky_horizon), ld3(F.ground), clampf(-y * 4.0f, 0.0f, 1.0f));
    return c * F.sky_horizon[3];
  }

  // ---------------------------------------------------------------------------------------- BSDF
  static M3 onb(V3 n) {
    const float s = n.z >= 0.0f ? 1.0f : -1.0f;
    const float a = -1.0f / (s + n.z);
    const float b = n.x * n.y * a;
    return M3{v3(1.0f + s * n.x * n.x * a, s * b, -s * n.x), v3(b, s + n.y * n.y * a, -n.y), n};
  }
  static float d_ggx(float nh, float a2) {
    const float d = nh * nh * (a2 - 1.0f) + 1.0f;
    return a2 / (PI * d * d);
  }
  static float g1(float nx, float a2) { return 2.0f * nx / (nx + std::sqrt(a2 + (1.0f - a2) * nx * nx)); }
  static V3 fresnel(V3 f0, float c) {
    const float k = std::pow(1.0f - clampf(c, 0.0f, 1.0f), 5.0f);
    return f0 + (v3(1, 1, 1) - f0) * k;
  }
  static V3 sample_vndf(V3 v, float a, float u1, float u2) {
    const V3 vh = normalize(v3(a * v.x, a * v.y, v.z));
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    const V3 T1 = lensq > 0.0f ? v3(-vh.y, vh.x, 0.0f) / std::sqrt(lensq) : v3(1.0f, 0.0f, 0.0f);
    const V3 T2 = cross(vh, T1);
    const float r = std::sqrt(u1);
    const float phi = 2.0f * PI * u2;
    const float t1 = r * std::cos(phi);
    float t2 = r * std::sin(phi);
    const float s = 0.5f * (1.0f + vh.z);
    t2 = (1.0f - s) * std::sqrt(1.0f - t1 * t1) + s * t2;
    const V3 nh = t1 * T1 + t2 * T2 + std::sqrt(std::max(0.0f, 1.0f - t1 * t1 - t2 * t2)) * vh;
    return normalize(v3(a * nh.x, a * nh.y, std::max(0.0f, nh.z)));
  }

  struct Surf {
    V3 p, ng, n, base, emissive;
    float rough = 0, metal = 0, transmission = 0, ior = 0;
    uint32_t obj = 0;
    bool front = false;
    V3 prev_p;
  };
  struct Eval { V3 f; float pdf; };

  static float spec_prob(const Surf &s, float nv) {
    const V3 f0 = mix(v3(0.04f, 0.04f, 0.04f), s.base, s.metal);
    const float fs = lum(fresnel(f0, nv));
    const float dw = (1.0f - s.metal) * lum(s.base) * (1.0f - fs);
    return clampf(fs / std::max(fs + dw, 1e-4f), 0.1f, 0.9f);
  }
  static Eval eval_bsdf(const Surf &s, V3 v, V3 l) {
    Eval e{v3(0, 0, 0), 0.0f};
    if (l.z <= 0.0f || v.z <= 0.0f) return e;
    const float a = std::max(s.rough * s.rough, 0.0025f);
    const float a2 = a * a;
    const V3 h = normalize(v + l);
    const float nh = h.z, vh = dot(v, h);
    const V3 f0 = mix(v3(0.04f, 0.04f, 0.04f), s.base, s.metal);
    const V3 Fr = fresnel(f0, vh);
    const float D = d_ggx(nh, a2);
    const float G = g1(v.z, a2) * g1(l.z, a2);
    const V3 spec = Fr * D * G / (4.0f * v.z);
    const V3 diff = (v3(1, 1, 1) - Fr) * (1.0f - s.metal) * s.base / PI * l.z;
    const float ps = spec_prob(s, v.z);
    const float pdf_spec = D * g1(v.z, a2) / (4.0f * v.z);
    const float pdf_diff = l.z / PI;
    e.f = spec + diff;
    e.pdf = ps * pdf_spec + (1.0f - ps) * pdf_diff;
    return e;
  }

  Surf fetch_surf(const Hit &h, V3 o, V3 d, float lod_base) const {
    Surf s;
    s.p = o + d * h.t;
    if (h.light >= 0) {
      const ho_pt_light &L = F.lights[h.light];
      s.ng = normalize(s.p - ld3(L.pos));
      s.n = s.ng;
      s.base = v3(0, 0, 0);
      s.emissive = ld3(L.radiance);
      s.obj = 1000u + (uint32_t)h.light;
      s.front = true;
      s.prev_p = ld3(L.prev_pos) + (s.p - ld3(L.pos));
      return s;
    }
    const uint32_t *ti = tri_idx(h.tri);
    const Mat m = mat(ti[3] & 0xffffu);
    const float w = 1.0f - h.u - h.v;
    const float *A = vert(ti[0]), *B = vert(ti[1]), *C = vert(ti[2]);
    const float *tr = S.tris + (size_t)h.tri * 12;
    const V3 e1 = ld3(tr + 4), e2 = ld3(tr + 8);
    V3 ng = normalize(cross(e1, e2));
    V3 n = normalize(ld3(A + 8) * w + ld3(B + 8) * h.u + ld3(C + 8) * h.v);
    s.front = dot(ng, d) < 0.0f;
    if (!s.front) ng = -ng;
    if (dot(n, ng) < 0.0f) n = -n;
    const float uv0x = A[3], uv0y = A[11], uv1x = B[3], uv1y = B[11], uv2x = C[3], uv2y = C[11];
    const float uvx = (uv0x * w + uv1x * h.u + uv2x * h.v) * m.uv[0];
    const float uvy = (uv0y * w + uv1y * h.u + uv2y * h.v) * m.uv[1];
    const float tri_lod = h2f((uint16_t)(ti[3] >> 16u));
    const float cosv = std::max(std::fabs(dot(ng, d)), 0.15f);
    const float lod = std::max(0.0f, tri_lod + std::log2(std::max(h.t * F.pixel_angle / cosv, 1e-6f) * lod_base) +
                                         std::log2(std::max(m.uv[0], 1.0f)));
    V3 base = ld3(m.base);
    if (m.tex[0] >= 0) {
      float c[4];
      sample_tex(uvx, uvy, m.tex[0], lod, c);
      base = base * v3(std::pow(c[0], 2.2f), std::pow(c[1], 2.2f), std::pow(c[2], 2.2f));
    }
    float rough = m.pbr[0], metal = m.pbr[1];
    if (m.tex[2] >= 0) {
      float arm[4];
      sample_tex(uvx, uvy, m.tex[2], lod, arm);
      rough *= arm[1];
      metal *= arm[2];
    }
    if (m.tex[1] >= 0) {
      const float d1x = (uv1x - uv0x) * m.uv[0], d1y = (uv1y - uv0y) * m.uv[1];
      const float d2x = (uv2x - uv0x) * m.uv[0], d2y = (uv2y - uv0y) * m.uv[1];
      const float det = d1x * d2y - d1y * d2x;
      if (std::fabs(det) > 1e-12f) {
        const float r = 1.0f / det;
        V3 t = (e1 * d2y - e2 * d1y) * r;
        const V3 bt = (e2 * d1x - e1 * d2x) * r;
        t = normalize(t - n * dot(n, t));
        const float handed = dot(cross(n, t), bt) >= 0.0f ? 1.0f : -1.0f;
        const V3 b = cross(n, t) * handed;
        float c[4];
        sample_tex(uvx, uvy, m.tex[1], lod, c);
        V3 tn = v3(c[0] * 2.0f - 1.0f, c[1] * 2.0f - 1.0f, c[2] * 2.0f - 1.0f);
        tn = v3(tn.x * m.uv[2], tn.y * m.uv[2], tn.z);
        const V3 nm = normalize(t * tn.x + b * tn.y + n * std::max(tn.z, 1e-3f));
        if (dot(nm, ng) > 0.05f) n = nm;
      }
    }
    s.ng = ng;
    s.n = n;
    s.base = base;
    s.emissive = ld3(m.emissive);
    s.rough = clampf(rough, 0.05f, 1.0f);
    s.metal = clampf(metal, 0.0f, 1.0f);
    s.transmission = m.pbr[2];
    s.ior = m.pbr[3];
    s.obj = ti[3] & 0xffffu;
    s.prev_p = ld3(A + 4) * w + ld3(B + 4) * h.u + ld3(C + 4) * h.v;
    return s;
  }

  // ---------------------------------------------------------------------------------------- lights
  static void cone_axis(const ho_pt_light &L, V3 p, V3 &axis, float &cos_max) {
    if (L.params[0] == 0.0f) { axis = ld3(L.pos); cos_max = L.params[1]; return; }
    const V3 to = ld3(L.pos) - p;
    const float d2 = dot(to, to), r2 = L.pos[3] * L.pos[3];
    if (d2 <= r2) { axis = v3(0, 1, 0); cos_max = -2.0f; return; }
    axis = to / std::sqrt(d2);
    cos_max = std::sqrt(1.0f - r2 / d2);
  }
  static float cone_pdf(float cos_max) { return 1.0f / (2.0f * PI * std::max(1.0f - cos_max, 1e-7f)); }
  static float mis(float a, float b) { const float a2 = a * a; return a2 / std::max(a2 + b * b, 1e-20f); }

  V3 direct_light(const Surf &s, const M3 &frame, V3 v, V3 tp, bool all) {
    V3 acc = v3(0, 0, 0);
    float w_sum = 0.0f, pick_w = 0.0f, pick_t = 0.0f;
    V3 pick_d = v3(0, 0, 0), pick_c = v3(0, 0, 0);
    for (uint32_t i = 0; i < F.counts[1]; i++) {
      const ho_pt_light &L = F.lights[i];
      V3 axis;
      float cos_max;
      cone_axis(L, s.p, axis, cos_max);
      if (cos_max < -1.0f) continue;
      const float ct = 1.0f - rnd() * (1.0f - cos_max);
      const float st = std::sqrt(std::max(0.0f, 1.0f - ct * ct));
      const float ph = 2.0f * PI * rnd();
      const M3 lf = onb(axis);
      const V3 dir = normalize(mul(lf, v3(std::cos(ph) * st, std::sin(ph) * st, ct)));
      const V3 ll = mulT(frame, dir);
      if (ll.z <= 0.0f || dot(dir, s.ng) <= 0.0f) continue;
      const Eval e = eval_bsdf(s, v, ll);
      if (e.pdf <= 0.0f && lum(e.f) <= 0.0f) continue;
      float tmax = INF;
      if (L.params[0] == 1.0f) tmax = sphere_t(s.p, dir, ld3(L.pos), L.pos[3]);
      const float lp = cone_pdf(cos_max);
      const V3 c = e.f * ld3(L.radiance) / lp * mis(lp, e.pdf);
      if (all) {
        if (!visible(s.p + s.ng * 1e-3f, dir, tmax)) continue;
        acc = acc + c;
      } else {
        const float w = lum(tp * c);
        if (w <= 0.0f) continue;
        w_sum += w;
        if (rnd() * w_sum < w) { pick_d = dir; pick_t = tmax; pick_c = c; pick_w = w; }
      }
    }
    if (!all && w_sum > 0.0f) {
      const float q = std::min(1.0f, w_sum / F.shadow_tau);
      if (rnd() < q && visible(s.p + s.ng * 1e-3f, pick_d, pick_t)) acc = pick_c * (w_sum / (pick_w * q));
    }
    if (F.env[3] > 0.5f) {
      V3 ed;
      float epdf;
      sample_env_dir(ed, epdf);
      const V3 ll = mulT(frame, ed);
      if (epdf > 0.0f && ll.z > 0.0f && dot(ed, s.ng) > 0.0f) {
        const Eval e = eval_bsdf(s, v, ll);
        if (lum(e.f) > 0.0f && visible(s.p + s.ng * 1e-3f, ed, INF)) acc = acc + e.f * sky(ed) / epdf * mis(epdf, e.pdf);
      }
    }
    return acc;
  }

  // ---------------------------------------------------------------------------------------- path
  struct GOut {
    V3 normal, albedo;
    float depth = 0, obj = 0, prev_depth = 0, rough = 0;
    float motion[2] = {0, 0};
  };

  void project_pix(const float *m, const float p[4], float out[2]) const {
    float c[4];
    mul4(m, p, c);
    const float nx = c[0] / c[3], ny = c[1] / c[3];
    out[0] = (nx * 0.5f + 0.5f) * (float)F.size[0];
    out[1] = (0.5f - ny * 0.5f) * (float)F.size[1];
  }

  void trace_path(float pix_x, float pix_y, bool write_g, V3 &radiance, V3 &primary_emission, GOut &g) {
    radiance = v3(0, 0, 0);
    primary_emission = v3(0, 0, 0);
    const float ndx = (pix_x / (float)F.size[0]) * 2.0f - 1.0f, ndy = (pix_y / (float)F.size[1]) * 2.0f - 1.0f;
    V3 o = ld3(F.cam_pos);
    V3 d = normalize(ld3(F.cam_fwd) + ld3(F.cam_right) * ndx - ld3(F.cam_up) * ndy);
    V3 tp = v3(1, 1, 1);
    float last_pdf = 0.0f, lod_base = 1.0f;
    uint32_t bounces = 0, delta_chain = 0;
    for (uint32_t depth = 0; depth < 12u; depth++) {
      const Hit h = trace_scene(o, d);
      const bool primary = depth == 0u;
      if (h.tri == NONE && h.light < 0) {
        V3 e = sky(d);
        if (F.env[3] > 0.5f && last_pdf > 0.0f) e = e * mis(last_pdf, env_pdf(d));
        for (uint32_t i = 0; i < F.counts[1]; i++) {
          const ho_pt_light &L = F.lights[i];
          if (L.params[0] == 0.0f && dot(d, ld3(L.pos)) >= L.params[1]) {
            if (last_pdf > 0.0f) e = e + ld3(L.radiance) * mis(last_pdf, cone_pdf(L.params[1]));
            else e = e + ld3(L.radiance);
          }
        }
        if (primary) {
          primary_emission = e;
          if (write_g) {
            g.normal = -d; g.depth = -1.0f; g.obj = 65535.0f; g.albedo = v3(1, 1, 1); g.rough = 1.0f;
            g.prev_depth = -1.0f;
            const float p4[4] = {d.x, d.y, d.z, 0.0f};
            float a[2], b[2];
            project_pix(F.prev_view_proj, p4, a);
            project_pix(F.view_proj, p4, b);
            g.motion[0] = a[0] - b[0];
            g.motion[1] = a[1] - b[1];
          }
        } else {
          V3 c = tp * e;
          const float lc = lum(c);
          if (lc > F.clamp_lum) c = c * (F.clamp_lum / lc);
          radiance = radiance + c;
        }
        break;
      }
      const Surf s = fetch_surf(h, o, d, lod_base);
      if (lum(s.emissive) > 0.0f) {
        V3 e = s.emissive;
        if (h.light >= 0 && last_pdf > 0.0f) {
          V3 axis;
          float cm;
          cone_axis(F.lights[h.light], o, axis, cm);
          e = e * mis(last_pdf, cone_pdf(cm));
        }
        if (primary) {
          primary_emission = e;
        } else {
          V3 c = tp * e;
          const float lc = lum(c);
          if (lc > F.clamp_lum) c = c * (F.clamp_lum / lc);
          radiance = radiance + c;
        }
      }
      const bool glass = s.transmission > 0.5f;
      if (primary && write_g) {
        g.normal = s.n;
        g.depth = dot(s.p - ld3(F.cam_pos), ld3(F.cam_fwd));
        g.obj = (float)s.obj;
        g.albedo = (glass || h.light >= 0)
                       ? v3(1, 1, 1)
                       : vmax(s.base * (1.0f - s.metal) + mix(v3(0.04f, 0.04f, 0.04f), s.base, s.metal) * s.metal,
                              v3(0.02f, 0.02f, 0.02f));
        g.rough = glass ? 0.0f : s.rough;
        const float pp[4] = {s.prev_p.x, s.prev_p.y, s.prev_p.z, 1.0f}, pc[4] = {s.p.x, s.p.y, s.p.z, 1.0f};
        float a[2], b[2];
        project_pix(F.prev_view_proj, pp, a);
        project_pix(F.view_proj, pc, b);
        g.motion[0] = a[0] - b[0];
        g.motion[1] = a[1] - b[1];
        float c4[4];
        mul4(F.prev_view_proj, pp, c4);
        g.prev_depth = c4[3];
      }
      if (h.light >= 0) break;
      if (glass) {
        delta_chain++;
        if (delta_chain > 8u) break;
        const float eta = s.front ? 1.0f / s.ior : s.ior;
        const V3 n = s.ng;
        const float c = -dot(d, n);
        const float k = 1.0f - eta * eta * (1.0f - c * c);
        float R = 1.0f;
        if (k > 0.0f) {
          const float ct = std::sqrt(k);
          const float rs = (eta * c - ct) / (eta * c + ct), rp = (c - eta * ct) / (c + eta * ct);
          R = 0.5f * (rs * rs + rp * rp);
        }
        if (rnd() < R) {
          d = reflect(d, n);
          o = s.p + n * 1e-3f;
        } else {
          d = normalize(d * eta + n * (eta * c - std::sqrt(k)));
          o = s.p - n * 1e-3f;
          tp = tp * s.base;
        }
        last_pdf = 0.0f;
        continue;
      }
      if (bounces >= F.max_bounces) break;
      bounces++;
      const M3 frame = onb(s.n);
      const V3 v = mulT(frame, -d);
      if (v.z <= 0.0f) break;
      V3 dl = tp * direct_light(s, frame, v, tp, primary || F.shadow_tau <= 0.0f);
      const float cl = primary ? (F.clamp_direct > 0.0f ? F.clamp_direct : INF) : F.clamp_lum;
      const float ld = lum(dl);
      if (ld > cl) dl = dl * (cl / ld);
      radiance = radiance + dl;
      const float ps = spec_prob(s, v.z);
      V3 l;
      if (rnd() < ps) {
        const float a = std::max(s.rough * s.rough, 0.0025f);
        const float u1 = rnd();
        const float u2 = rnd();
        l = reflect(-v, sample_vndf(v, a, u1, u2));
      } else {
        const float r = std::sqrt(rnd());
        const float ph = 2.0f * PI * rnd();
        l = v3(r * std::cos(ph), r * std::sin(ph), std::sqrt(std::max(0.0f, 1.0f - r * r)));
      }
      if (l.z <= 0.0f) break;
      const Eval e = eval_bsdf(s, v, l);
      if (e.pdf <= 0.0f) break;
      tp = tp * e.f / e.pdf;
      last_pdf = e.pdf;
      d = normalize(mul(frame, l));
      if (dot(d, s.ng) <= 0.0f) break;
      o = s.p + s.ng * 1e-3f;
      lod_base = 4.0f;
      if (bounces >= 2u) {
        const float q = clampf(std::max(tp.x, std::max(tp.y, tp.z)), 0.05f, 0.95f);
        if (rnd() > q) break;
        tp = tp / q;
      }
    }
  }
};

void pixel_mode0(const ho_pt_scene *s, const ho_pt_frame *f, int x, int y, float out[18]) {
  Tracer T{*s, *f};
  const uint32_t idx = (uint32_t)y * f->size[0] + (uint32_t)x;
  T.rng = pcg(idx ^ pcg(f->frame * 0x9E3779B9u + 17u));
  const float px = (float)x + 0.5f + f->jitter[0], py = (float)y + 0.5f + f->jitter[1];
  V3 rad, pe;
  Tracer::GOut g;
  T.trace_path(px, py, true, rad, pe, g);
  const float o[18] = {rad.x, rad.y, rad.z, pe.x, pe.y, pe.z, g.normal.x, g.normal.y, g.normal.z, g.depth,
                       g.motion[0], g.motion[1], g.obj, g.prev_depth, g.albedo.x, g.albedo.y, g.albedo.z, g.rough};
  std::memcpy(out, o, sizeof(o));
}

}  // namespace

extern "C" void ho_pt_pixel(const ho_pt_scene *s, const ho_pt_frame *f, int x, int y, float out[18]) {
  pixel_mode0(s, f, x, y, out);
}

extern "C" void ho_pt_trace(const ho_pt_scene *s, const ho_pt_frame *f, const float o[3], const float d[3],
                            float out[5]) {
  Tracer T{*s, *f};
  const Tracer::Hit h = T.trace_scene(v3(o[0], o[1], o[2]), v3(d[0], d[1], d[2]));
  out[0] = h.t;
  out[1] = h.tri == NONE ? -1.0f : (float)h.tri;
  out[2] = (float)h.light;
  out[3] = h.u;
  out[4] = h.v;
}

extern "C" int ho_pt_render(const ho_pt_scene *s, const ho_pt_frame *f, uint16_t *const gbuf[5], float *accum) {
  const int W = (int)f->size[0], H = (int)f->size[1];
  if (W <= 0 || H <= 0) return -1;
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      const size_t idx = (size_t)y * W + x;
      if (f->mode == 0u) {
        float o[18];
        pixel_mode0(s, f, x, y, o);
        const float img[5][4] = {{o[0], o[1], o[2], 1.0f}, {o[6], o[7], o[8], o[9]}, {o[10], o[11], o[12], o[13]},
                                 {o[14], o[15], o[16], o[17]}, {o[3], o[4], o[5], 0.0f}};
        for (int k = 0; k < 5; k++)
          if (gbuf[k])
            for (int c = 0; c < 4; c++) gbuf[k][idx * 4 + c] = f2h_rz(img[k][c]);
      } else {
        Tracer T{*s, *f};
        V3 sum = v3(0, 0, 0);
        for (uint32_t sp = 0; sp < f->spp; sp++) {
          T.rng = pcg((uint32_t)idx ^ pcg((f->counts[2] + sp) * 0x9E3779B9u + f->frame * 7919u + 1u));
          const float jx = T.rnd();
          const float jy = T.rnd();
          V3 rad, pe;
          Tracer::GOut g;
          T.trace_path((float)x + jx, (float)y + jy, false, rad, pe, g);
          sum = sum + rad + pe;
        }
        accum[idx * 4] += sum.x;
        accum[idx * 4 + 1] += sum.y;
        accum[idx * 4 + 2] += sum.z;
        accum[idx * 4 + 3] += (float)f->spp;
      }
    }
  }
  return 0;
}

// ------------------------------------------------------------------------------------------------ bvh.js
namespace {
constexpr int BINS = 12;
constexpr int MAX_LEAF = 4;
inline double area(double dx, double dy, double dz) { return dx < 0 ? 0 : dx * dy + dy * dz + dz * dx; }
}  // namespace

extern "C" int ho_bvh_build(const float *pos, int tri_count, float *f, uint32_t *order, int *max_depth) {
  const int n = tri_count;
  std::vector<float> cx(3 * (size_t)n), bmin(3 * (size_t)n), bmax(3 * (size_t)n);
  for (int t = 0; t < n; t++)
    for (int a = 0; a < 3; a++) {
      const double p0 = pos[t * 9 + a], p1 = pos[t * 9 + 3 + a], p2 = pos[t * 9 + 6 + a];
      const double lo = std::min(p0, std::min(p1, p2)), hi = std::max(p0, std::max(p1, p2));
      bmin[t * 3 + a] = (float)lo;
      bmax[t * 3 + a] = (float)hi;
      cx[t * 3 + a] = (float)((lo + hi) * 0.5);
    }
  for (int i = 0; i < n; i++) order[i] = (uint32_t)i;
  const int max_nodes = std::max(1, 2 * n);
  std::fill(f, f + (size_t)max_nodes * 8, 0.0f);
  auto U = [&](size_t i) -> uint32_t & { return reinterpret_cast<uint32_t *>(f)[i]; };
  int used = 1;
  const double dinf = std::numeric_limits<double>::infinity();
  struct Job { int node, first, count, depth; };
  std::vector<Job> stack{{0, 0, n, 0}};
  int maxd = 0;
  float bin_min[BINS * 3], bin_max[BINS * 3];
  uint32_t bin_cnt[BINS];
  while (!stack.empty()) {
    const Job j = stack.back();
    stack.pop_back();
    const int node = j.node, first = j.first, count = j.count, depth = j.depth;
    maxd = std::max(maxd, depth);
    {  // bounds(node, first, count)
      double x0 = dinf, y0 = dinf, z0 = dinf, x1 = -dinf, y1 = -dinf, z1 = -dinf;
      for (int i = first; i < first + count; i++) {
        const size_t t = (size_t)order[i] * 3;
        if (bmin[t] < x0) x0 = bmin[t];
        if (bmin[t + 1] < y0) y0 = bmin[t + 1];
        if (bmin[t + 2] < z0) z0 = bmin[t + 2];
        if (bmax[t] > x1) x1 = bmax[t];
        if (bmax[t + 1] > y1) y1 = bmax[t + 1];
        if (bmax[t + 2] > z1) z1 = bmax[t + 2];
      }
      const size_t o = (size_t)node * 8;
      f[o] = (float)x0; f[o + 1] = (float)y0; f[o + 2] = (float)z0;
      f[o + 4] = (float)x1; f[o + 5] = (float)y1; f[o + 6] = (float)z1;
    }
    const size_t o = (size_t)node * 8;
    if (count <= MAX_LEAF) {
      U(o + 3) = (uint32_t)first;
      U(o + 7) = (uint32_t)count;
      continue;
    }
    double c0[3] = {dinf, dinf, dinf}, c1[3] = {-dinf, -dinf, -dinf};
    for (int i = first; i < first + count; i++) {
      const size_t t = (size_t)order[i] * 3;
      for (int a = 0; a < 3; a++) {
        const double c = cx[t + a];
        if (c < c0[a]) c0[a] = c;
        if (c > c1[a]) c1[a] = c;
      }
    }
    double best_cost = dinf;
    int best_axis = -1, best_split = 0;
    for (int a = 0; a < 3; a++) {
      const double ext = c1[a] - c0[a];
      if (ext <= 1e-12) continue;
      std::fill(bin_min, bin_min + BINS * 3, std::numeric_limits<float>::infinity());
      std::fill(bin_max, bin_max + BINS * 3, -std::numeric_limits<float>::infinity());
      std::fill(bin_cnt, bin_cnt + BINS, 0u);
      const double scale = BINS / ext;
      for (int i = first; i < first + count; i++) {
        const size_t t = (size_t)order[i] * 3;
        const int b = std::min(BINS - 1, (int)((cx[t + a] - c0[a]) * scale));
        bin_cnt[b]++;
        for (int k = 0; k < 3; k++) {
          if (bmin[t + k] < bin_min[b * 3 + k]) bin_min[b * 3 + k] = bmin[t + k];
          if (bmax[t + k] > bin_max[b * 3 + k]) bin_max[b * 3 + k] = bmax[t + k];
        }
      }
      double right_area[BINS] = {0};
      uint32_t right_cnt[BINS] = {0};
      double rmin[3] = {dinf, dinf, dinf}, rmax[3] = {-dinf, -dinf, -dinf};
      uint32_t rc = 0;
      for (int b = BINS - 1; b > 0; b--) {
        rc += bin_cnt[b];
        for (int k = 0; k < 3; k++) {
          rmin[k] = std::min(rmin[k], (double)bin_min[b * 3 + k]);
          rmax[k] = std::max(rmax[k], (double)bin_max[b * 3 + k]);
        }
        right_area[b] = rc ? area(rmax[0] - rmin[0], rmax[1] - rmin[1], rmax[2] - rmin[2]) : 0;
        right_cnt[b] = rc;
      }
      double lx0 = dinf, ly0 = dinf, lz0 = dinf, lx1 = -dinf, ly1 = -dinf, lz1 = -dinf;
      uint32_t lc = 0;
      for (int b = 0; b < BINS - 1; b++) {
        lc += bin_cnt[b];
        lx0 = std::min(lx0, (double)bin_min[b * 3]); ly0 = std::min(ly0, (double)bin_min[b * 3 + 1]);
        lz0 = std::min(lz0, (double)bin_min[b * 3 + 2]);
        lx1 = std::max(lx1, (double)bin_max[b * 3]); ly1 = std::max(ly1, (double)bin_max[b * 3 + 1]);
        lz1 = std::max(lz1, (double)bin_max[b * 3 + 2]);
        if (!lc || !right_cnt[b + 1]) continue;
        const double cost = lc * area(lx1 - lx0, ly1 - ly0, lz1 - lz0) + right_cnt[b + 1] * right_area[b + 1];
        if (cost < best_cost) { best_cost = cost; best_axis = a; best_split = b + 1; }
      }
    }
    const double leaf_cost = count * area((double)f[o + 4] - f[o], (double)f[o + 5] - f[o + 1], (double)f[o + 6] - f[o + 2]);
    int mid;
    if (best_axis < 0 || (best_cost >= leaf_cost && count <= 16)) {
      if (best_axis < 0) {
        mid = first + (count >> 1);
      } else {
        U(o + 3) = (uint32_t)first;
        U(o + 7) = (uint32_t)count;
        continue;
      }
    } else {
      const int a = best_axis;
      const double scale = BINS / (c1[a] - c0[a]);
      int i = first, k = first + count - 1;
      while (i <= k) {
        const int b = std::min(BINS - 1, (int)((cx[(size_t)order[i] * 3 + a] - c0[a]) * scale));
        if (b < best_split) i++;
        else { std::swap(order[i], order[k]); k--; }
      }
      mid = i;
      if (mid == first || mid == first + count) mid = first + (count >> 1);
    }
    const int left = used;
    used += 2;
    U(o + 3) = (uint32_t)left;
    U(o + 7) = 0;
    stack.push_back({left + 1, mid, first + count - mid, depth + 1});
    stack.push_back({left, first, mid - first, depth + 1});
  }
  if (max_depth) *max_depth = maxd;
  return used;
}

extern "C" void ho_bvh_refit(float *nodes, int node_count, const float *tri_pos) {
  const uint32_t *u = reinterpret_cast<const uint32_t *>(nodes);
  const double dinf = std::numeric_limits<double>::infinity();
  for (int n = node_count - 1; n >= 0; n--) {
    const size_t o = (size_t)n * 8;
    const uint32_t count = u[o + 7];
    double x0 = dinf, y0 = dinf, z0 = dinf, x1 = -dinf, y1 = -dinf, z1 = -dinf;
    if (count > 0) {
      const uint32_t first = u[o + 3];
      for (uint32_t t = first; t < first + count; t++)
        for (int v = 0; v < 3; v++) {
          const size_t p = (size_t)t * 9 + v * 3;
          const double x = tri_pos[p], y = tri_pos[p + 1], z = tri_pos[p + 2];
          x0 = std::min(x0, x); y0 = std::min(y0, y); z0 = std::min(z0, z);
          x1 = std::max(x1, x); y1 = std::max(y1, y); z1 = std::max(z1, z);
        }
    } else {
      const size_t l = (size_t)u[o + 3] * 8, r = l + 8;
      x0 = std::min(nodes[l], nodes[r]); y0 = std::min(nodes[l + 1], nodes[r + 1]); z0 = std::min(nodes[l + 2], nodes[r + 2]);
      x1 = std::max(nodes[l + 4], nodes[r + 4]); y1 = std::max(nodes[l + 5], nodes[r + 5]);
      z1 = std::max(nodes[l + 6], nodes[r + 6]);
    }
    nodes[o] = (float)x0; nodes[o + 1] = (float)y0; nodes[o + 2] = (float)z0;
    nodes[o + 4] = (float)x1; nodes[o + 5] = (float)y1; nodes[o + 6] = (float)z1;
  }
}

extern "C" int ho_bvh_packed_count(const float *nodes, int node_count) {
  const uint32_t *u = reinterpret_cast<const uint32_t *>(nodes);
  int k = 0;
  for (int n = 0; n < node_count; n++)
    if (u[(size_t)n * 8 + 7] == 0) k++;
  return std::max(k, 1);
}

extern "C" void ho_bvh_pack(const float *nodes, int node_count, float *out) {
  const uint32_t *u = reinterpret_cast<const uint32_t *>(nodes);
  uint32_t *ou = reinterpret_cast<uint32_t *>(out);
  std::vector<int> id(node_count);
  int k = 0;
  for (int n = 0; n < node_count; n++) id[n] = u[(size_t)n * 8 + 7] == 0 ? k++ : -1;
  auto child = [&](size_t o, size_t c) {
    const size_t s = c * 8;
    for (int a = 0; a < 3; a++) { out[o + a] = nodes[s + a]; out[o + 4 + a] = nodes[s + 4 + a]; }
    const uint32_t count = u[s + 7];
    ou[o + 3] = count > 0 ? u[s + 3] : (uint32_t)id[c];
    ou[o + 7] = count;
  };
  if (k == 0) {
    child(0, 0);
    child(8, 0);
    return;
  }
  for (int n = 0; n < node_count; n++) {
    if (id[n] < 0) continue;
    const size_t o = (size_t)id[n] * 16, l = u[(size_t)n * 8 + 3];
    child(o, l);
    child(o + 8, l + 1);
  }
}

// scene.js computeTriLod (178-208), including its f16 conversion (truncating, flushes subnormals to zero)
extern "C" uint16_t ho_tri_lod(const float *va, const float *vb, const float *vc, int tex_size) {
  const double e1[3] = {(double)vb[0] - va[0], (double)vb[1] - va[1], (double)vb[2] - va[2]};
  const double e2[3] = {(double)vc[0] - va[0], (double)vc[1] - va[1], (double)vc[2] - va[2]};
  const double cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  const double wa = std::hypot(cr[0], cr[1], cr[2]) * 0.5;
  const double u1[2] = {(double)vb[3] - va[3], (double)vb[11] - va[11]};
  const double u2[2] = {(double)vc[3] - va[3], (double)vc[11] - va[11]};
  const double ua = std::fabs(u1[0] * u2[1] - u1[1] * u2[0]) * 0.5;
  const double lod = wa > 1e-12 && ua > 1e-14 ? std::log2(std::sqrt(ua / wa) * tex_size) : 0.0;
  const uint32_t x = fbits((float)lod);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const int e = (int)((x >> 23) & 0xffu) - 127 + 15;
  const uint32_t m = (x >> 13) & 0x3ffu;
  if (e <= 0) return (uint16_t)sign;
  if (e >= 31) return (uint16_t)(sign | 0x7c00u);
  return (uint16_t)(sign | ((uint32_t)e << 10) | m);
}

// ------------------------------------------------------------------------------------------------ envmap.js
namespace {
inline double lumd(double r, double g, double b) { return 0.2126 * r + 0.7152 * g + 0.0722 * b; }
void dir_of(double u, double v, double d[3]) {
  const double phi = (u - 0.5) * 2 * M_PI, th = v * M_PI;
  d[0] = std::cos(phi) * std::sin(th);
  d[1] = std::cos(th);
  d[2] = std::sin(phi) * std::sin(th);
}
}  // namespace

extern "C" int ho_env_prepare(float *rgba, int W, int H, int sun, double cone_deg, uint16_t *half_out,
                              float *table, double sun_dir[3], double sun_irr[3]) {
  int has_sun = 0;
  if (sun) {  // cutSun (envmap.js:22-61)
    double best = 0;
    int bi = 0;
    for (int i = 0; i < W * H; i++) {
      const double l = lumd(rgba[i * 4], rgba[i * 4 + 1], rgba[i * 4 + 2]);
      if (l > best) { best = l; bi = i; }
    }
    double s[3];
    dir_of(((bi % W) + 0.5) / W, (std::floor((double)bi / W) + 0.5) / H, s);
    const double cos_in = std::cos(cone_deg * M_PI / 180), cos_out = std::cos(cone_deg * 1.6 * M_PI / 180);
    const int row = bi / W, span = (int)std::ceil(cone_deg * 1.7 * H / 180);
    const int r0 = std::max(0, row - span), r1 = std::min(H - 1, row + span);
    double ring[3] = {0, 0, 0};
    int n = 0;
    struct In { int i; double d[3]; int y; };
    std::vector<In> inner;
    for (int y = r0; y <= r1; y++)
      for (int x = 0; x < W; x++) {
        In e;
        dir_of((x + 0.5) / W, (y + 0.5) / H, e.d);
        const double c = e.d[0] * s[0] + e.d[1] * s[1] + e.d[2] * s[2];
        e.i = (y * W + x) * 4;
        e.y = y;
        if (c >= cos_in) inner.push_back(e);
        else if (c >= cos_out) { ring[0] += rgba[e.i]; ring[1] += rgba[e.i + 1]; ring[2] += rgba[e.i + 2]; n++; }
      }
    if (n) {
      for (int k = 0; k < 3; k++) ring[k] /= n;
      const double ring_l = lumd(ring[0], ring[1], ring[2]);
      if (best >= 50 * ring_l) {
        double E[3] = {0, 0, 0}, c[3] = {0, 0, 0};
        const double dA = (2 * M_PI / W) * (M_PI / H);
        for (const In &e : inner) {
          const int i = e.i;
          if (lumd(rgba[i], rgba[i + 1], rgba[i + 2]) < 3 * ring_l) continue;
          const double w = dA * std::sin(((e.y + 0.5) / H) * M_PI);
          double ex[3];
          for (int k = 0; k < 3; k++) ex[k] = std::max(0.0, rgba[i + k] - ring[k]) * w;
          for (int k = 0; k < 3; k++) { E[k] += ex[k]; rgba[i + k] = (float)ring[k]; }
          const double wl = lumd(ex[0], ex[1], ex[2]);
          for (int k = 0; k < 3; k++) c[k] += e.d[k] * wl;
        }
        double cl = std::hypot(std::hypot(c[0], c[1]), c[2]);
        if (cl == 0) cl = 1;
        for (int k = 0; k < 3; k++) { sun_dir[k] = c[k] / cl; sun_irr[k] = E[k]; }
        has_sun = 1;
      }
    }
  }
  std::vector<double> weights((size_t)GW * GH, 0.0);
  for (int y = 0; y < H; y++) {
    const int gy = std::min((int)GH - 1, (int)std::floor((double)y * GH / H));
    for (int x = 0; x < W; x++) {
      const size_t i = ((size_t)y * W + x) * 4;
      weights[(size_t)gy * GW + std::min((int)GW - 1, (int)std::floor((double)x * GW / W))] +=
          lumd(rgba[i], rgba[i + 1], rgba[i + 2]);
    }
  }
  for (uint32_t gy = 0; gy < GH; gy++) {
    const double st = std::sin(((gy + 0.5) / GH) * M_PI);
    for (uint32_t gx = 0; gx < GW; gx++) weights[gy * GW + gx] = weights[gy * GW + gx] * st + 1e-6;
  }
  for (size_t i = 0; i < (size_t)W * H * 4; i++) {  // three.js toHalfFloat truncates the mantissa
    const float v = std::min(rgba[i], 65000.0f);
    half_out[i] = f2h_rz(v);
  }
  // aliasTable (envmap.js:64-82), Vose
  const size_t N = weights.size();
  double sum = 0;
  for (double w : weights) sum += w;
  std::vector<double> p(N);
  for (size_t i = 0; i < N; i++) p[i] = (weights[i] / sum) * N;
  std::vector<uint32_t> small, large;
  for (size_t i = 0; i < N; i++) (p[i] < 1 ? small : large).push_back((uint32_t)i);
  uint32_t *tu = reinterpret_cast<uint32_t *>(table);
  std::fill(table, table + N * 4, 0.0f);
  while (!small.empty() && !large.empty()) {
    const uint32_t s = small.back();
    small.pop_back();
    const uint32_t l = large.back();
    table[s * 4] = (float)p[s];
    tu[s * 4 + 1] = l;
    p[l] -= 1 - p[s];
    if (p[l] < 1) { large.pop_back(); small.push_back(l); }
  }
  for (uint32_t i : small) { table[i * 4] = 1; tu[i * 4 + 1] = i; }
  for (uint32_t i : large) { table[i * 4] = 1; tu[i * 4 + 1] = i; }
  for (size_t i = 0; i < N; i++) table[i * 4 + 2] = (float)(weights[i] / sum);
  return has_sun;
}

extern "C" void ho_pt_jitter(float out[32]) {
  auto halton = [](int i, int b) {
    double f = 1, r = 0;
    while (i > 0) { f /= b; r += f * (i % b); i = i / b; }
    return r;
  };
  for (int i = 0; i < 16; i++) {
    out[2 * i] = (float)(halton(i + 1, 2) - 0.5);
    out[2 * i + 1] = (float)(halton(i + 1, 3) - 0.5);
  }
}
