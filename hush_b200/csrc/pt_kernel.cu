// The path tracer's kernel and the PathTracer instance (src/pt/pathtracer.js, pathtracer.wgsl.js).
//
// One thread per pixel, 8 x 8 pixel blocks (each warp covers an 8 x 4 patch, so primary rays of a warp stay
// coherent); each thread walks the packed BVH2 with its traversal stack in shared memory, laid out stack-slot-major
// (slot k of thread t at k * 64 + t) so that the warp's pushes and pops hit 32 distinct banks. Scene records are read
// as float4 / uint4 through the read-only path. The arithmetic and the order of random draws follow the WGSL
// (pathtracer.wgsl.js:75-672): PCG hash per pixel and frame, Moller-Trumbore triangles, GGX with VNDF sampling, smooth
// glass, next-event estimation with MIS on cone lights and the importance-sampled environment map, Russian roulette
// after two bounces. Texture and environment lookups are explicit trilinear / bilinear filters with f32 weights.
// Mode 0 writes the five rgba16float G-buffer images (storage rounding toward zero), mode 1 accumulates.
#include <cuda_runtime.h>

#include <string>

#include "common.cuh"
#include "hush.h"
#include "pt_internal.h"

using hush::f4_to_h4;
using hush::h4_to_f4;

namespace {

constexpr float PI = 3.14159265358979f;
constexpr float INF = 1e30f;
constexpr uint32_t NONE = 0xffffffffu;
constexpr int STACK = 32;  // >= BVH depth, checked by the scene build
constexpr int BW = 8, BH = 8, NT = BW * BH;
constexpr uint32_t GW = HUSH_PT_ENV_GW, GH = HUSH_PT_ENV_GH;
constexpr int TEX_S = HUSH_PT_TEX_SIZE, TEX_M = HUSH_PT_TEX_MIPS;

#define DI __device__ __forceinline__

DI float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
DI float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
DI float3 f3(const float *p) { return make_float3(p[0], p[1], p[2]); }
DI float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
DI float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
DI float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
DI float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
DI float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
DI float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
DI float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DI float3 cross(float3 a, float3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
DI float3 normalize(float3 a) { return a / sqrtf(dot(a, a)); }
DI float3 reflect(float3 d, float3 n) { return d - n * (2.0f * dot(n, d)); }
DI float3 lerp3(float3 a, float3 b, float t) { return a * (1.0f - t) + b * t; }
DI float lum(float3 c) { return dot(c, f3(0.2126f, 0.7152f, 0.0722f)); }
DI float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

struct Basis { float3 t, b, n; };  // columns of onb()
DI float3 to_world(const Basis &m, float3 v) { return m.t * v.x + m.b * v.y + m.n * v.z; }
DI float3 to_local(const Basis &m, float3 v) { return f3(dot(m.t, v), dot(m.b, v), dot(m.n, v)); }

DI Basis onb(float3 n) {  // Duff et al. 2017 orthonormal basis
  const float s = n.z >= 0.0f ? 1.0f : -1.0f;
  const float a = -1.0f / (s + n.z);
  const float b = n.x * n.y * a;
  return Basis{f3(1.0f + s * n.x * n.x * a, s * b, -s * n.x), f3(b, s + n.y * n.y * a, -n.y), n};
}

DI uint32_t pcg(uint32_t v) {
  const uint32_t s = v * 747796405u + 2891336453u;
  const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}

struct Hit { float t; uint32_t tri; float u, v; int light; };

struct Surf {
  float3 p, ng, n, base, emissive, prev_p;
  float rough, metal, transmission, ior;
  uint32_t obj;
  bool front;
};

struct GBuf { uint2 *rad, *nd, *mv, *mat, *emi; };

struct Tracer {
  const hush_pt_frame &F;
  const pt::SceneView &S;
  const pt::EnvView &E;
  uint32_t *stk;  // this thread's column of the shared traversal stacks
  uint32_t rng;

  DI float rnd() {
    rng = pcg(rng);
    return (float)(rng >> 8u) * (1.0f / 16777216.0f);
  }

  // -------------------------------------------------------------------------------------- texture lookups
  DI static int wrapi(int i, int n) { const int r = i % n; return r < 0 ? r + n : r; }
  DI float4 texel(int layer, int mip, int x, int y) const {
    size_t off = 0, per = 0;
#pragma unroll
    for (int m = 0; m < TEX_M; m++) {
      const size_t s = (size_t)max(1, TEX_S >> m);
      off += m < mip ? s * s * 4 : 0;
      per += s * s * 4;
    }
    const int s = max(1, TEX_S >> mip);
    const uchar4 t = __ldg(reinterpret_cast<const uchar4 *>(S.tex + per * layer + off) + (size_t)wrapi(y, s) * s + wrapi(x, s));
    return make_float4(t.x / 255.0f, t.y / 255.0f, t.z / 255.0f, t.w / 255.0f);
  }
  DI float4 bilinear(int layer, int mip, float u, float v) const {
    const int s = max(1, TEX_S >> mip);
    const float x = u * (float)s - 0.5f, y = v * (float)s - 0.5f;
    const float x0 = floorf(x), y0 = floorf(y), fx = x - x0, fy = y - y0;
    const int ix = (int)x0, iy = (int)y0;
    const float4 a = texel(layer, mip, ix, iy), b = texel(layer, mip, ix + 1, iy);
    const float4 c = texel(layer, mip, ix, iy + 1), d = texel(layer, mip, ix + 1, iy + 1);
    auto mix1 = [&](float p, float q, float r, float w) {
      return (p * (1.0f - fx) + q * fx) * (1.0f - fy) + (r * (1.0f - fx) + w * fx) * fy;
    };
    return make_float4(mix1(a.x, b.x, c.x, d.x), mix1(a.y, b.y, c.y, d.y), mix1(a.z, b.z, c.z, d.z),
                       mix1(a.w, b.w, c.w, d.w));
  }
  DI float4 sample_tex(float u, float v, int layer, float lod) const {  // trilinear, repeat
    const float l = clampf(lod, 0.0f, (float)(TEX_M - 1));
    const int m0 = (int)floorf(l), m1 = min(m0 + 1, TEX_M - 1);
    const float t = l - (float)m0;
    const float4 a = bilinear(layer, m0, u, v), b = bilinear(layer, m1, u, v);
    return make_float4(a.x * (1.0f - t) + b.x * t, a.y * (1.0f - t) + b.y * t, a.z * (1.0f - t) + b.z * t,
                       a.w * (1.0f - t) + b.w * t);
  }
  DI float3 sample_env(float u, float v) const {  // bilinear, repeat in u, clamp-to-edge in v
    const float x = u * (float)E.w - 0.5f, y = v * (float)E.h - 0.5f;
    const float x0 = floorf(x), y0 = floorf(y), fx = x - x0, fy = y - y0;
    auto at = [&](int xi, int yi) {
      return f3(h4_to_f4(__ldg(E.texels + (size_t)min(max(yi, 0), E.h - 1) * E.w + wrapi(xi, E.w))));
    };
    const int ix = (int)x0, iy = (int)y0;
    const float3 top = at(ix, iy) * (1.0f - fx) + at(ix + 1, iy) * fx;
    const float3 bot = at(ix, iy + 1) * (1.0f - fx) + at(ix + 1, iy + 1) * fx;
    return top * (1.0f - fy) + bot * fy;
  }

  // -------------------------------------------------------------------------------------- geometry
  DI static float slab(float3 o, float3 inv, float4 bmin, float4 bmax, float tmax) {
    const float t0x = (bmin.x - o.x) * inv.x, t1x = (bmax.x - o.x) * inv.x;
    const float t0y = (bmin.y - o.y) * inv.y, t1y = (bmax.y - o.y) * inv.y;
    const float t0z = (bmin.z - o.z) * inv.z, t1z = (bmax.z - o.z) * inv.z;
    const float tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
    const float tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
    return (tn <= tf && tf > 0.0f && tn < tmax) ? fmaxf(tn, 0.0f) : INF;
  }

  DI bool alpha_pass(uint32_t tri, float u, float v) const {
    const uint4 ti = __ldg(S.tri_idx + tri);
    const float4 base = __ldg(S.mats + (size_t)(ti.w & 0xffffu) * 5);
    const float4 tex = __ldg(S.mats + (size_t)(ti.w & 0xffffu) * 5 + 3);
    const int tex0 = __float_as_int(tex.x);
    if (base.w <= 0.0f || tex0 < 0) return true;
    const float4 uvs = __ldg(S.mats + (size_t)(ti.w & 0xffffu) * 5 + 4);
    const float w = 1.0f - u - v;
    const float4 A = __ldg(S.verts + (size_t)ti.x * 3), B = __ldg(S.verts + (size_t)ti.y * 3),
                 C = __ldg(S.verts + (size_t)ti.z * 3);
    const float4 An = __ldg(S.verts + (size_t)ti.x * 3 + 2), Bn = __ldg(S.verts + (size_t)ti.y * 3 + 2),
                 Cn = __ldg(S.verts + (size_t)ti.z * 3 + 2);
    const float uu = A.w * w + B.w * u + C.w * v, vv = An.w * w + Bn.w * u + Cn.w * v;
    return sample_tex(uu * uvs.x, vv * uvs.y, tex0, 2.0f).w >= base.w;
  }

  // Moller-Trumbore; returns (t, u, v) or t = INF
  DI float3 hit_tri(float3 o, float3 d, uint32_t tri, float tmax) const {
    const float4 a = __ldg(S.tris + (size_t)tri * 3);
    const float3 e1 = f3(__ldg(S.tris + (size_t)tri * 3 + 1)), e2 = f3(__ldg(S.tris + (size_t)tri * 3 + 2));
    const float3 p = cross(d, e2);
    const float det = dot(e1, p);
    if (fabsf(det) < 1e-12f) return f3(INF, 0.f, 0.f);
    const float inv = 1.0f / det;
    const float3 s = o - f3(a);
    const float u = dot(s, p) * inv;
    if (u < 0.0f || u > 1.0f) return f3(INF, 0.f, 0.f);
    const float3 q = cross(s, e1);
    const float v = dot(d, q) * inv;
    if (v < 0.0f || u + v > 1.0f) return f3(INF, 0.f, 0.f);
    const float t = dot(e2, q) * inv;
    if (t <= 1e-4f || t >= tmax) return f3(INF, 0.f, 0.f);
    if (a.w > 0.0f && !alpha_pass(tri, u, v)) return f3(INF, 0.f, 0.f);
    return f3(t, u, v);
  }

  // closest (or, for shadow rays, any) hit over the BLAS list; packed BVH2 (both child boxes per 64-byte node)
  DI Hit trace_bvh(float3 o, float3 d, float tmax_in, bool shadow) const {
    Hit h{tmax_in, NONE, 0.0f, 0.0f, -1};
    const float3 inv = f3(1.0f / (fabsf(d.x) < 1e-9f ? 1e-9f : d.x), 1.0f / (fabsf(d.y) < 1e-9f ? 1e-9f : d.y),
                          1.0f / (fabsf(d.z) < 1e-9f ? 1e-9f : d.z));
    for (uint32_t b = 0; b < F.counts[0]; b++) {
      const hush_pt_blas bl = F.blas[b];
      if (shadow && (bl.flags & 2u)) continue;
      uint32_t sp = 0, node = 0;
      // a BVH built by the scene visits each node at most once per ray; the cap only bounds a corrupted one
      for (uint32_t guard = 0; guard < (1u << 24); guard++) {
        const float4 *nd = S.nodes + (size_t)(bl.node_offset + node) * 4;
        const float4 lmin = __ldg(nd), lmax = __ldg(nd + 1), rmin = __ldg(nd + 2), rmax = __ldg(nd + 3);
        float tl = slab(o, inv, lmin, lmax, h.t);
        float tr = slab(o, inv, rmin, rmax, h.t);
        const uint32_t lc = __float_as_uint(lmax.w), rc = __float_as_uint(rmax.w);
        if (lc > 0u && tl < INF) {
          const uint32_t first = bl.tri_offset + __float_as_uint(lmin.w);
          for (uint32_t i = 0; i < lc; i++) {
            const float3 r = hit_tri(o, d, first + i, h.t);
            if (r.x < h.t) {
              h.t = r.x; h.u = r.y; h.v = r.z; h.tri = first + i;
              if (shadow) return h;
            }
          }
          tl = INF;
        }
        if (rc > 0u && tr < h.t) {
          const uint32_t first = bl.tri_offset + __float_as_uint(rmin.w);
          for (uint32_t i = 0; i < rc; i++) {
            const float3 r = hit_tri(o, d, first + i, h.t);
            if (r.x < h.t) {
              h.t = r.x; h.u = r.y; h.v = r.z; h.tri = first + i;
              if (shadow) return h;
            }
          }
          tr = INF;
        }
        const uint32_t l = __float_as_uint(lmin.w), r = __float_as_uint(rmin.w);
        if (tl < h.t && tr < h.t) {
          const bool near_left = tl <= tr;
          node = near_left ? l : r;
          stk[sp * NT] = near_left ? r : l;
          sp = min(sp + 1u, (uint32_t)STACK - 1u);
        } else if (tl < h.t) {
          node = l;
        } else if (tr < h.t) {
          node = r;
        } else {
          if (sp == 0u) break;
          node = stk[--sp * NT];
        }
      }
    }
    return h;
  }

  DI static float sphere_t(float3 o, float3 d, float3 c, float r) {
    const float3 oc = o - c;
    const float b = dot(oc, d), cc = dot(oc, oc) - r * r;
    const float disc = b * b - cc;
    if (disc < 0.0f) return INF;
    const float s = sqrtf(disc);
    float t = -b - s;
    if (t < 1e-4f) t = -b + s;
    return t < 1e-4f ? INF : t;
  }

  DI Hit trace_scene(float3 o, float3 d) const {
    Hit h = trace_bvh(o, d, INF, false);
    for (uint32_t i = 0; i < F.counts[1]; i++) {
      const hush_pt_light &L = F.lights[i];
      if (L.params[0] != 1.0f) continue;
      const float t = sphere_t(o, d, f3(L.pos), L.pos[3]);
      if (t < h.t) { h.t = t; h.light = (int)i; h.tri = NONE; }
    }
    return h;
  }

  DI bool visible(float3 o, float3 d, float tmax) const { return trace_bvh(o, d, tmax, true).tri == NONE; }

  // -------------------------------------------------------------------------------------- environment
  DI float3 env_local(float3 d) const { return f3(F.env[1] * d.x - F.env[2] * d.z, d.y, F.env[2] * d.x + F.env[1] * d.z); }
  DI static float2 env_uv(float3 l) {
    return make_float2(atan2f(l.z, l.x) * (0.5f / PI) + 0.5f, acosf(clampf(l.y, -1.0f, 1.0f)) / PI);
  }
  DI float env_pdf(float3 d) const {
    const float3 l = env_local(d);
    const float2 uv = env_uv(l);
    const float st = sqrtf(fmaxf(0.0f, 1.0f - l.y * l.y));
    if (st < 1e-5f) return 0.0f;
    const uint32_t cx = min((uint32_t)(uv.x * (float)GW), GW - 1u), cy = min((uint32_t)(uv.y * (float)GH), GH - 1u);
    return __ldg(E.table + cy * GW + cx).z * (float)(GW * GH) / (2.0f * PI * PI * st);
  }
  DI float4 sample_env_dir() {  // direction (xyz) and solid-angle pdf (w)
    const uint32_t N = GW * GH;
    uint32_t i = min((uint32_t)(rnd() * (float)N), N - 1u);
    const float4 a = __ldg(E.table + i);
    if (rnd() >= a.x) i = __float_as_uint(a.y);
    const float r1 = rnd();
    const float u = ((float)(i % GW) + r1) / (float)GW;
    const float r2 = rnd();
    const float v = ((float)(i / GW) + r2) / (float)GH;
    const float phi = (u - 0.5f) * 2.0f * PI, th = v * PI;
    const float st = sinf(th);
    const float3 l = f3(cosf(phi) * st, cosf(th), sinf(phi) * st);
    const float pdf = st > 1e-5f ? __ldg(E.table + i).z * (float)N / (2.0f * PI * PI * st) : 0.0f;
    return make_float4(F.env[1] * l.x + F.env[2] * l.z, l.y, -F.env[2] * l.x + F.env[1] * l.z, pdf);
  }
  DI float3 sky(float3 d) const {
    if (F.env[3] > 0.5f) {
      const float2 uv = env_uv(env_local(d));
      return sample_env(uv.x, uv.y) * F.env[0];
    }
    float3 c;
    if (d.y >= 0.0f) c = lerp3(f3(F.sky_horizon), f3(F.sky_zenith), powf(clampf(d.y, 0.0f, 1.0f), 0.6f));
    else c = lerp3(f3(F.sky_horizon), f3(F.ground), clampf(-d.y * 4.0f, 0.0f, 1.0f));
    return c * F.sky_horizon[3];
  }

  // -------------------------------------------------------------------------------------- BSDF
  DI static float d_ggx(float nh, float a2) {
    const float d = nh * nh * (a2 - 1.0f) + 1.0f;
    return a2 / (PI * d * d);
  }
  DI static float g1(float nx, float a2) { return 2.0f * nx / (nx + sqrtf(a2 + (1.0f - a2) * nx * nx)); }
  DI static float3 fresnel(float3 f0, float c) {
    const float k = powf(1.0f - clampf(c, 0.0f, 1.0f), 5.0f);
    return f0 + (f3(1.f, 1.f, 1.f) - f0) * k;
  }
  DI static float3 sample_vndf(float3 v, float a, float u1, float u2) {  // Heitz 2018
    const float3 vh = normalize(f3(a * v.x, a * v.y, v.z));
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    const float3 T1 = lensq > 0.0f ? f3(-vh.y, vh.x, 0.0f) / sqrtf(lensq) : f3(1.f, 0.f, 0.f);
    const float3 T2 = cross(vh, T1);
    const float r = sqrtf(u1), phi = 2.0f * PI * u2;
    const float t1 = r * cosf(phi);
    float t2 = r * sinf(phi);
    const float s = 0.5f * (1.0f + vh.z);
    t2 = (1.0f - s) * sqrtf(1.0f - t1 * t1) + s * t2;
    const float3 nh = T1 * t1 + T2 * t2 + vh * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1 - t2 * t2));
    return normalize(f3(a * nh.x, a * nh.y, fmaxf(0.0f, nh.z)));
  }
  DI static float spec_prob(const Surf &s, float nv) {
    const float3 f0 = lerp3(f3(0.04f, 0.04f, 0.04f), s.base, s.metal);
    const float fs = lum(fresnel(f0, nv));
    const float dw = (1.0f - s.metal) * lum(s.base) * (1.0f - fs);
    return clampf(fs / fmaxf(fs + dw, 1e-4f), 0.1f, 0.9f);
  }
  // f * cos and the combined pdf of the diffuse + GGX lobes (local frame)
  DI static float4 eval_bsdf(const Surf &s, float3 v, float3 l, float3 &f) {
    f = f3(0.f, 0.f, 0.f);
    if (l.z <= 0.0f || v.z <= 0.0f) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float a = fmaxf(s.rough * s.rough, 0.0025f), a2 = a * a;
    const float3 h = normalize(v + l);
    const float3 f0 = lerp3(f3(0.04f, 0.04f, 0.04f), s.base, s.metal);
    const float3 Fr = fresnel(f0, dot(v, h));
    const float D = d_ggx(h.z, a2);
    const float G = g1(v.z, a2) * g1(l.z, a2);
    const float3 spec = Fr * D * G / (4.0f * v.z);
    const float3 diff = (f3(1.f, 1.f, 1.f) - Fr) * (1.0f - s.metal) * s.base / PI * l.z;
    const float ps = spec_prob(s, v.z);
    f = spec + diff;
    const float pdf = ps * (D * g1(v.z, a2) / (4.0f * v.z)) + (1.0f - ps) * (l.z / PI);
    return make_float4(f.x, f.y, f.z, pdf);
  }

  DI Surf fetch_surf(const Hit &h, float3 o, float3 d, float lod_base) const {
    Surf s;
    s.p = o + d * h.t;
    s.rough = s.metal = s.transmission = s.ior = 0.0f;
    if (h.light >= 0) {
      const hush_pt_light &L = F.lights[h.light];
      s.ng = normalize(s.p - f3(L.pos));
      s.n = s.ng;
      s.base = f3(0.f, 0.f, 0.f);
      s.emissive = f3(L.radiance);
      s.obj = 1000u + (uint32_t)h.light;
      s.front = true;
      s.prev_p = f3(L.prev_pos) + (s.p - f3(L.pos));
      return s;
    }
    const uint4 ti = __ldg(S.tri_idx + h.tri);
    const float4 *M = S.mats + (size_t)(ti.w & 0xffffu) * 5;
    const float4 mb = __ldg(M), me = __ldg(M + 1), mp = __ldg(M + 2), mt = __ldg(M + 3), mu = __ldg(M + 4);
    const int tex_base = __float_as_int(mt.x), tex_nrm = __float_as_int(mt.y), tex_arm = __float_as_int(mt.z);
    const float w = 1.0f - h.u - h.v;
    const float4 A0 = __ldg(S.verts + (size_t)ti.x * 3), A2 = __ldg(S.verts + (size_t)ti.x * 3 + 2);
    const float4 B0 = __ldg(S.verts + (size_t)ti.y * 3), B2 = __ldg(S.verts + (size_t)ti.y * 3 + 2);
    const float4 C0 = __ldg(S.verts + (size_t)ti.z * 3), C2 = __ldg(S.verts + (size_t)ti.z * 3 + 2);
    const float3 e1 = f3(__ldg(S.tris + (size_t)h.tri * 3 + 1)), e2 = f3(__ldg(S.tris + (size_t)h.tri * 3 + 2));
    float3 ng = normalize(cross(e1, e2));
    float3 n = normalize(f3(A2) * w + f3(B2) * h.u + f3(C2) * h.v);
    s.front = dot(ng, d) < 0.0f;
    if (!s.front) ng = -ng;
    if (dot(n, ng) < 0.0f) n = -n;
    const float uvx = (A0.w * w + B0.w * h.u + C0.w * h.v) * mu.x;
    const float uvy = (A2.w * w + B2.w * h.u + C2.w * h.v) * mu.y;
    const float tri_lod = __half2float(__ushort_as_half((unsigned short)(ti.w >> 16u)));
    const float cosv = fmaxf(fabsf(dot(ng, d)), 0.15f);
    const float lod = fmaxf(0.0f, tri_lod + log2f(fmaxf(h.t * F.pixel_angle / cosv, 1e-6f) * lod_base) +
                                      log2f(fmaxf(mu.x, 1.0f)));
    float3 base = f3(mb);
    if (tex_base >= 0) {
      const float4 c = sample_tex(uvx, uvy, tex_base, lod);
      base = base * f3(powf(c.x, 2.2f), powf(c.y, 2.2f), powf(c.z, 2.2f));
    }
    float rough = mp.x, metal = mp.y;
    if (tex_arm >= 0) {
      const float4 arm = sample_tex(uvx, uvy, tex_arm, lod);
      rough *= arm.y;
      metal *= arm.z;
    }
    if (tex_nrm >= 0) {  // tangent frame from dP / dUV of the triangle
      const float d1x = (B0.w - A0.w) * mu.x, d1y = (B2.w - A2.w) * mu.y;
      const float d2x = (C0.w - A0.w) * mu.x, d2y = (C2.w - A2.w) * mu.y;
      const float det = d1x * d2y - d1y * d2x;
      if (fabsf(det) > 1e-12f) {
        const float r = 1.0f / det;
        float3 t = (e1 * d2y - e2 * d1y) * r;
        const float3 bt = (e2 * d1x - e1 * d2x) * r;
        t = normalize(t - n * dot(n, t));
        const float3 b = cross(n, t) * (dot(cross(n, t), bt) >= 0.0f ? 1.0f : -1.0f);
        const float4 c = sample_tex(uvx, uvy, tex_nrm, lod);
        const float3 tn = f3((c.x * 2.0f - 1.0f) * mu.z, (c.y * 2.0f - 1.0f) * mu.z, c.z * 2.0f - 1.0f);
        const float3 nm = normalize(t * tn.x + b * tn.y + n * fmaxf(tn.z, 1e-3f));
        if (dot(nm, ng) > 0.05f) n = nm;
      }
    }
    s.ng = ng;
    s.n = n;
    s.base = base;
    s.emissive = f3(me);
    s.rough = clampf(rough, 0.05f, 1.0f);
    s.metal = clampf(metal, 0.0f, 1.0f);
    s.transmission = mp.z;
    s.ior = mp.w;
    s.obj = ti.w & 0xffffu;
    s.prev_p = f3(__ldg(S.verts + (size_t)ti.x * 3 + 1)) * w + f3(__ldg(S.verts + (size_t)ti.y * 3 + 1)) * h.u +
               f3(__ldg(S.verts + (size_t)ti.z * 3 + 1)) * h.v;
    return s;
  }

  // -------------------------------------------------------------------------------------- lights
  DI static float4 cone_axis(const hush_pt_light &L, float3 p) {  // axis, cos of the half angle (-2: inside)
    if (L.params[0] == 0.0f) return make_float4(L.pos[0], L.pos[1], L.pos[2], L.params[1]);
    const float3 to = f3(L.pos) - p;
    const float d2 = dot(to, to), r2 = L.pos[3] * L.pos[3];
    if (d2 <= r2) return make_float4(0.f, 1.f, 0.f, -2.0f);
    const float3 a = to / sqrtf(d2);
    return make_float4(a.x, a.y, a.z, sqrtf(1.0f - r2 / d2));
  }
  DI static float cone_pdf(float cos_max) { return 1.0f / (2.0f * PI * fmaxf(1.0f - cos_max, 1e-7f)); }
  DI static float mis(float a, float b) { const float a2 = a * a; return a2 / fmaxf(a2 + b * b, 1e-20f); }

  DI float3 direct_light(const Surf &s, const Basis &frame, float3 v, float3 tp, bool all) {
    float3 acc = f3(0.f, 0.f, 0.f), pick_c = acc, pick_d = acc;
    float w_sum = 0.0f, pick_w = 0.0f, pick_t = 0.0f;
    for (uint32_t i = 0; i < F.counts[1]; i++) {
      const hush_pt_light &L = F.lights[i];
      const float4 ax = cone_axis(L, s.p);
      if (ax.w < -1.0f) continue;
      const float ct = 1.0f - rnd() * (1.0f - ax.w);
      const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
      const float ph = 2.0f * PI * rnd();
      const float3 dir = normalize(to_world(onb(f3(ax)), f3(cosf(ph) * st, sinf(ph) * st, ct)));
      const float3 ll = to_local(frame, dir);
      if (ll.z <= 0.0f || dot(dir, s.ng) <= 0.0f) continue;
      float3 f;
      const float pdf = eval_bsdf(s, v, ll, f).w;
      if (pdf <= 0.0f && lum(f) <= 0.0f) continue;
      const float tmax = L.params[0] == 1.0f ? sphere_t(s.p, dir, f3(L.pos), L.pos[3]) : INF;
      const float lp = cone_pdf(ax.w);
      const float3 c = f * f3(L.radiance) / lp * mis(lp, pdf);
      if (all) {
        if (!visible(s.p + s.ng * 1e-3f, dir, tmax)) continue;
        acc = acc + c;
      } else {
        const float wl = lum(tp * c);
        if (wl <= 0.0f) continue;
        w_sum += wl;
        if (rnd() * w_sum < wl) { pick_d = dir; pick_t = tmax; pick_c = c; pick_w = wl; }
      }
    }
    if (!all && w_sum > 0.0f) {
      const float q = fminf(1.0f, w_sum / F.shadow_tau);
      if (rnd() < q && visible(s.p + s.ng * 1e-3f, pick_d, pick_t)) acc = pick_c * (w_sum / (pick_w * q));
    }
    if (F.env[3] > 0.5f) {
      const float4 es = sample_env_dir();
      const float3 ed = f3(es);
      const float3 ll = to_local(frame, ed);
      if (es.w > 0.0f && ll.z > 0.0f && dot(ed, s.ng) > 0.0f) {
        float3 f;
        const float pdf = eval_bsdf(s, v, ll, f).w;
        if (lum(f) > 0.0f && visible(s.p + s.ng * 1e-3f, ed, INF)) acc = acc + f * sky(ed) / es.w * mis(es.w, pdf);
      }
    }
    return acc;
  }

  DI float2 project_pix(const float *m, float px, float py, float pz, float pw) const {
    const float cx = m[0] * px + m[4] * py + m[8] * pz + m[12] * pw;
    const float cy = m[1] * px + m[5] * py + m[9] * pz + m[13] * pw;
    const float cw = m[3] * px + m[7] * py + m[11] * pz + m[15] * pw;
    const float nx = cx / cw, ny = cy / cw;
    return make_float2((nx * 0.5f + 0.5f) * (float)F.size[0], (0.5f - ny * 0.5f) * (float)F.size[1]);
  }

  // tracePath (pathtracer.wgsl.js:511-646); with write_g the primary hit's G-buffer values go to g[0..11]
  DI void trace_path(float pix_x, float pix_y, bool write_g, float3 &radiance, float3 &prim_emission, float *g) {
    radiance = f3(0.f, 0.f, 0.f);
    prim_emission = radiance;
    const float ndx = (pix_x / (float)F.size[0]) * 2.0f - 1.0f, ndy = (pix_y / (float)F.size[1]) * 2.0f - 1.0f;
    float3 o = f3(F.cam_pos);
    float3 d = normalize(f3(F.cam_fwd) + f3(F.cam_right) * ndx - f3(F.cam_up) * ndy);
    float3 tp = f3(1.f, 1.f, 1.f);
    float last_pdf = 0.0f, lod_base = 1.0f;
    uint32_t bounces = 0, delta_chain = 0;
    for (uint32_t depth = 0; depth < 12u; depth++) {
      const Hit h = trace_scene(o, d);
      const bool primary = depth == 0u;
      if (h.tri == NONE && h.light < 0) {  // sky
        float3 e = sky(d);
        if (F.env[3] > 0.5f && last_pdf > 0.0f) e = e * mis(last_pdf, env_pdf(d));
        for (uint32_t i = 0; i < F.counts[1]; i++) {  // sun disks reached by BSDF sampling
          const hush_pt_light &L = F.lights[i];
          if (L.params[0] == 0.0f && dot(d, f3(L.pos)) >= L.params[1])
            e = e + f3(L.radiance) * (last_pdf > 0.0f ? mis(last_pdf, cone_pdf(L.params[1])) : 1.0f);
        }
        if (primary) {
          prim_emission = e;
          if (write_g) {
            const float2 a = project_pix(F.prev_view_proj, d.x, d.y, d.z, 0.0f);
            const float2 b = project_pix(F.view_proj, d.x, d.y, d.z, 0.0f);
            const float gv[12] = {-d.x, -d.y, -d.z, -1.0f, a.x - b.x, a.y - b.y, 65535.0f, -1.0f, 1.f, 1.f, 1.f, 1.f};
#pragma unroll
            for (int k = 0; k < 12; k++) g[k] = gv[k];
          }
        } else {
          float3 c = tp * e;
          const float lc = lum(c);
          if (lc > F.clamp_lum) c = c * (F.clamp_lum / lc);
          radiance = radiance + c;
        }
        break;
      }
      const Surf s = fetch_surf(h, o, d, lod_base);
      if (lum(s.emissive) > 0.0f) {
        float3 e = s.emissive;
        if (h.light >= 0 && last_pdf > 0.0f) e = e * mis(last_pdf, cone_pdf(cone_axis(F.lights[h.light], o).w));
        if (primary) {
          prim_emission = e;
        } else {
          float3 c = tp * e;
          const float lc = lum(c);
          if (lc > F.clamp_lum) c = c * (F.clamp_lum / lc);
          radiance = radiance + c;
        }
      }
      const bool glass = s.transmission > 0.5f;
      if (primary && write_g) {
        const bool white = glass || h.light >= 0;
        const float3 alb = s.base * (1.0f - s.metal) + lerp3(f3(0.04f, 0.04f, 0.04f), s.base, s.metal) * s.metal;
        const float2 a = project_pix(F.prev_view_proj, s.prev_p.x, s.prev_p.y, s.prev_p.z, 1.0f);
        const float2 b = project_pix(F.view_proj, s.p.x, s.p.y, s.p.z, 1.0f);
        const float *pm = F.prev_view_proj;
        const float prev_w = pm[3] * s.prev_p.x + pm[7] * s.prev_p.y + pm[11] * s.prev_p.z + pm[15];
        g[0] = s.n.x; g[1] = s.n.y; g[2] = s.n.z;
        g[3] = dot(s.p - f3(F.cam_pos), f3(F.cam_fwd));
        g[4] = a.x - b.x; g[5] = a.y - b.y;
        g[6] = (float)s.obj;
        g[7] = prev_w;
        g[8] = white ? 1.0f : fmaxf(alb.x, 0.02f);
        g[9] = white ? 1.0f : fmaxf(alb.y, 0.02f);
        g[10] = white ? 1.0f : fmaxf(alb.z, 0.02f);
        g[11] = glass ? 0.0f : s.rough;
      }
      if (h.light >= 0) break;
      if (glass) {  // smooth dielectric: Fresnel-weighted reflect / refract
        if (++delta_chain > 8u) break;
        const float eta = s.front ? 1.0f / s.ior : s.ior;
        const float3 n = s.ng;
        const float c = -dot(d, n);
        const float k = 1.0f - eta * eta * (1.0f - c * c);
        float R = 1.0f;
        if (k > 0.0f) {
          const float ct = sqrtf(k);
          const float rs = (eta * c - ct) / (eta * c + ct), rp = (c - eta * ct) / (c + eta * ct);
          R = 0.5f * (rs * rs + rp * rp);
        }
        if (rnd() < R) {
          d = reflect(d, n);
          o = s.p + n * 1e-3f;
        } else {
          d = normalize(d * eta + n * (eta * c - sqrtf(k)));
          o = s.p - n * 1e-3f;
          tp = tp * s.base;
        }
        last_pdf = 0.0f;
        continue;
      }
      if (bounces >= F.max_bounces) break;
      bounces++;
      const Basis frame = onb(s.n);
      const float3 v = to_local(frame, -d);
      if (v.z <= 0.0f) break;
      float3 dl = tp * direct_light(s, frame, v, tp, primary || F.shadow_tau <= 0.0f);
      const float cl = primary ? (F.clamp_direct > 0.0f ? F.clamp_direct : INF) : F.clamp_lum;
      const float ld = lum(dl);
      if (ld > cl) dl = dl * (cl / ld);
      radiance = radiance + dl;
      const float ps = spec_prob(s, v.z);
      float3 l;
      if (rnd() < ps) {
        const float a = fmaxf(s.rough * s.rough, 0.0025f);
        const float u1 = rnd();
        const float u2 = rnd();
        l = reflect(-v, sample_vndf(v, a, u1, u2));
      } else {
        const float r = sqrtf(rnd());
        const float ph = 2.0f * PI * rnd();
        l = f3(r * cosf(ph), r * sinf(ph), sqrtf(fmaxf(0.0f, 1.0f - r * r)));
      }
      if (l.z <= 0.0f) break;
      float3 f;
      const float pdf = eval_bsdf(s, v, l, f).w;
      if (pdf <= 0.0f) break;
      tp = tp * f / pdf;
      last_pdf = pdf;
      d = normalize(to_world(frame, l));
      if (dot(d, s.ng) <= 0.0f) break;
      o = s.p + s.ng * 1e-3f;
      lod_base = 4.0f;
      if (bounces >= 2u) {  // Russian roulette
        const float q = clampf(fmaxf(tp.x, fmaxf(tp.y, tp.z)), 0.05f, 0.95f);
        if (rnd() > q) break;
        tp = tp / q;
      }
    }
  }
};

// main() of pathtracer.wgsl.js:648-672
__global__ void __launch_bounds__(NT, 8) k_pathtrace(const __grid_constant__ hush_pt_frame F, const pt::SceneView S,
                                                   const pt::EnvView E, const GBuf G, float4 *__restrict__ accum) {
  __shared__ uint32_t stacks[STACK * NT];
  const uint32_t t = threadIdx.y * BW + threadIdx.x;
  const uint32_t x = blockIdx.x * BW + threadIdx.x, y = blockIdx.y * BH + threadIdx.y;
  if (x >= F.size[0] || y >= F.size[1]) return;  // no block-wide barrier below
  Tracer T{F, S, E, stacks + t, 0u};
  const uint32_t idx = y * F.size[0] + x;
  if (F.mode == 0u) {
    T.rng = pcg(idx ^ pcg(F.frame * 0x9E3779B9u + 17u));
    float3 rad, pe;
    float g[12];
    T.trace_path((float)x + 0.5f + F.jitter[0], (float)y + 0.5f + F.jitter[1], true, rad, pe, g);
    G.rad[idx] = f4_to_h4(make_float4(rad.x, rad.y, rad.z, 1.0f));
    G.nd[idx] = f4_to_h4(make_float4(g[0], g[1], g[2], g[3]));
    G.mv[idx] = f4_to_h4(make_float4(g[4], g[5], g[6], g[7]));
    G.mat[idx] = f4_to_h4(make_float4(g[8], g[9], g[10], g[11]));
    G.emi[idx] = f4_to_h4(make_float4(pe.x, pe.y, pe.z, 0.0f));
  } else {
    float3 sum = f3(0.f, 0.f, 0.f);
    for (uint32_t sp = 0; sp < F.spp; sp++) {
      T.rng = pcg(idx ^ pcg((F.counts[2] + sp) * 0x9E3779B9u + F.frame * 7919u + 1u));
      const float jx = T.rnd();
      const float jy = T.rnd();
      float3 rad, pe;
      T.trace_path((float)x + jx, (float)y + jy, false, rad, pe, nullptr);
      sum = sum + rad + pe;
    }
    const float4 a = accum[idx];
    accum[idx] = make_float4(a.x + sum.x, a.y + sum.y, a.z + sum.z, a.w + (float)F.spp);
  }
}

}  // namespace

struct hush_pt_s {
  hush_pt_scene_t *scene = nullptr;
  int dev = 0, W = 0, H = 0;
  void *pool = nullptr;
  uint2 *gbuf[2][5] = {};
  float4 *accum = nullptr;
  void *env_pool = nullptr;
  pt::EnvView env{};
};

static int pt_alloc(hush_pt_t *p, int W, int H) {
  cudaSetDevice(p->dev);
  if (p->pool) cudaFree(p->pool);
  p->pool = nullptr;
  const size_t img = ((size_t)W * H * 8 + 255) & ~(size_t)255, acc = (size_t)W * H * 16;
  cudaError_t e = cudaMalloc(&p->pool, img * 10 + acc);
  if (e != cudaSuccess) {
    p->pool = nullptr;
    return pt::fail(HUSH_ERR_CUDA, std::string("PathTracer.resize: cudaMalloc: ") + cudaGetErrorString(e));
  }
  char *b = static_cast<char *>(p->pool);
  for (int s = 0; s < 2; s++)
    for (int k = 0; k < 5; k++) p->gbuf[s][k] = reinterpret_cast<uint2 *>(b + img * (s * 5 + k));
  p->accum = reinterpret_cast<float4 *>(b + img * 10);
  e = cudaMemset(p->pool, 0, img * 10 + acc);
  if (e != cudaSuccess) return pt::fail(HUSH_ERR_CUDA, std::string("PathTracer.resize: ") + cudaGetErrorString(e));
  p->W = W;
  p->H = H;
  return HUSH_OK;
}

extern "C" int hush_pt_create(hush_pt_scene_t *scene, int W, int H, hush_pt_t **out) {
  if (!out) return pt::fail(HUSH_ERR_ARG, "hush_pt_create: out is NULL");
  *out = nullptr;
  if (!pt::scene_built(scene)) return pt::fail(HUSH_ERR_ARG, "PathTracer: the scene is not built");
  if (W <= 0 || H <= 0) return pt::fail(HUSH_ERR_ARG, "PathTracer: bad size");
  hush_pt_t *p = new hush_pt_t();
  p->scene = scene;
  p->dev = pt::scene_device(scene);
  if (int rc = pt_alloc(p, W, H)) {
    delete p;
    return rc;
  }
  *out = p;
  return HUSH_OK;
}

extern "C" void hush_pt_destroy(hush_pt_t *p) {
  if (!p) return;
  cudaSetDevice(p->dev);
  if (p->pool) cudaFree(p->pool);
  if (p->env_pool) cudaFree(p->env_pool);
  delete p;
}

extern "C" int hush_pt_resize(hush_pt_t *p, int W, int H) {
  if (!p) return pt::fail(HUSH_ERR_ARG, "PathTracer.resize: NULL tracer");
  if (W <= 0 || H <= 0) return pt::fail(HUSH_ERR_ARG, "PathTracer: bad size");
  if (W == p->W && H == p->H) return HUSH_OK;
  return pt_alloc(p, W, H);
}

extern "C" int hush_pt_set_envmap(hush_pt_t *p, const uint16_t *half, int w, int h, const float *table) {
  if (!p) return pt::fail(HUSH_ERR_ARG, "PathTracer.setEnvMap: NULL tracer");
  cudaSetDevice(p->dev);
  if (p->env_pool) cudaFree(p->env_pool);
  p->env_pool = nullptr;
  p->env = pt::EnvView{};
  if (!half) return HUSH_OK;
  if (!table || w <= 0 || h <= 0) return pt::fail(HUSH_ERR_ARG, "PathTracer.setEnvMap: bad map");
  const size_t tex = ((size_t)w * h * 8 + 255) & ~(size_t)255, tab = (size_t)GW * GH * 16;
  cudaError_t e = cudaMalloc(&p->env_pool, tex + tab);
  if (e == cudaSuccess) e = cudaMemcpy(p->env_pool, half, (size_t)w * h * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(static_cast<char *>(p->env_pool) + tex, table, tab, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return pt::fail(HUSH_ERR_CUDA, std::string("PathTracer.setEnvMap: ") + cudaGetErrorString(e));
  p->env.texels = static_cast<const uint2 *>(p->env_pool);
  p->env.w = w;
  p->env.h = h;
  p->env.table = reinterpret_cast<const float4 *>(static_cast<char *>(p->env_pool) + tex);
  return HUSH_OK;
}

extern "C" int hush_pt_encode(hush_pt_t *p, const hush_pt_frame *f, int slot, void *stream) {
  if (!p || !f) return pt::fail(HUSH_ERR_ARG, "PathTracer.encode: NULL argument");
  if (slot < 0 || slot > 1) return pt::fail(HUSH_ERR_ARG, "PathTracer.encode: slot must be 0 or 1");
  if ((int)f->size[0] != p->W || (int)f->size[1] != p->H)
    return pt::fail(HUSH_ERR_ARG, "PathTracer.encode: frame size " + std::to_string(f->size[0]) + "x" +
                                      std::to_string(f->size[1]) + " differs from the tracer's " +
                                      std::to_string(p->W) + "x" + std::to_string(p->H));
  if (f->counts[0] > HUSH_PT_MAX_BLAS || f->counts[1] > HUSH_PT_MAX_LIGHTS)
    return pt::fail(HUSH_ERR_ARG, "PathTracer.encode: too many BLAS or lights");
  const int ngroups = hush_pt_scene_blas(p->scene, nullptr, HUSH_PT_MAX_BLAS);
  hush_pt_blas tab[HUSH_PT_MAX_BLAS];
  hush_pt_scene_blas(p->scene, tab, HUSH_PT_MAX_BLAS);
  for (uint32_t b = 0; b < f->counts[0]; b++) {  // every BLAS must lie inside the scene's buffers
    bool ok = false;
    for (int g = 0; g < ngroups; g++)
      ok |= f->blas[b].node_offset == tab[g].node_offset && f->blas[b].tri_offset == tab[g].tri_offset &&
            f->blas[b].node_count == tab[g].node_count;
    if (!ok) return pt::fail(HUSH_ERR_ARG, "PathTracer.encode: BLAS " + std::to_string(b) + " is not one of the scene's");
  }
  if (f->env[3] > 0.5f && !p->env.texels)
    return pt::fail(HUSH_ERR_ARG, "PathTracer.encode: env.w = 1 but no environment map is bound");
  cudaSetDevice(p->dev);
  const GBuf G{p->gbuf[slot][0], p->gbuf[slot][1], p->gbuf[slot][2], p->gbuf[slot][3], p->gbuf[slot][4]};
  const dim3 grid((p->W + BW - 1) / BW, (p->H + BH - 1) / BH), blk(BW, BH);
  k_pathtrace<<<grid, blk, 0, (cudaStream_t)stream>>>(*f, pt::scene_view(p->scene), p->env, G, p->accum);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HUSH_OK : pt::fail(HUSH_ERR_CUDA, std::string("PathTracer.encode: ") + cudaGetErrorString(e));
}

extern "C" const void *hush_pt_gbuffer(const hush_pt_t *p, int slot, int which) {
  if (!p || slot < 0 || slot > 1 || which < 0 || which > 4) return nullptr;
  return p->gbuf[slot][which];
}

extern "C" float *hush_pt_accum(const hush_pt_t *p) { return p ? reinterpret_cast<float *>(p->accum) : nullptr; }

extern "C" int hush_pt_clear_accum(hush_pt_t *p, void *stream) {
  if (!p) return pt::fail(HUSH_ERR_ARG, "PathTracer.clearAccum: NULL tracer");
  cudaSetDevice(p->dev);
  const cudaError_t e = cudaMemsetAsync(p->accum, 0, (size_t)p->W * p->H * 16, (cudaStream_t)stream);
  return e == cudaSuccess ? HUSH_OK : pt::fail(HUSH_ERR_CUDA, std::string("PathTracer.clearAccum: ") + cudaGetErrorString(e));
}
