// Host side of the path tracer: the scene (SceneGPU of src/pt/scene.js without three.js), the binned-SAH BVH
// (src/pt/bvh.js), the environment-map preparation (src/pt/envmap.js) and the Halton jitter (src/pt/pathtracer.js).
//
// The scene arrives as world-space meshes grouped into BLAS (at most 8). Building produces the reference's GPU
// layouts, so the device kernel reads exactly what the WGSL reads:
//   nodes   16 floats per packed BVH node: [lmin, lData] [lmax, lCount] [rmin, rData] [rmax, rCount]
//   tris    12 floats per triangle in BVH order: [v0, alpha-tested] [v1 - v0, 0] [v2 - v0, 0]
//   triIdx  4 u32: vertex ids a b c, material | f16 texture LOD << 16
//   verts   12 floats: pos.xyz, u, prev.xyz, 0, normal.xyz, v
//   mats    80 bytes (hush_pt_material)
//   tex     rgba8 layers of 11 mips (1024^2 .. 1^2), mip-major inside a layer
// The BVH builder makes the same decisions as bvh.js (JavaScript doubles over f32 storage), so the trees match the
// reference's bit for bit; binning evaluates the three axes in one pass over the triangles.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "hush.h"
#include "pt_internal.h"

namespace {

thread_local std::string g_pt_err;

constexpr int BINS = 12;     // bvh.js:9
constexpr int MAX_LEAF = 4;  // bvh.js:10

inline uint32_t f_as_u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float u_as_f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// ------------------------------------------------------------------------------------------------ BVH (bvh.js)
// Build layout: 8 floats per node, [min.xyz, leftOrFirst bits] [max.xyz, count bits]; interior nodes have count 0
// and children at leftOrFirst, leftOrFirst + 1 (allocated after the parent).
struct SahBuilder {
  int n;
  std::vector<float> cen, lo, hi;  // per triangle and axis: centroid, bounds (Float32Array in bvh.js)
  float *nodes;
  uint32_t *order;
  int used = 1, max_depth = 0;

  static double area(double dx, double dy, double dz) { return dx < 0 ? 0 : dx * dy + dy * dz + dz * dx; }
  uint32_t &word(size_t i) { return reinterpret_cast<uint32_t *>(nodes)[i]; }

  SahBuilder(const float *pos, int count, float *out_nodes, uint32_t *out_order)
      : n(count), cen(3 * (size_t)count), lo(3 * (size_t)count), hi(3 * (size_t)count), nodes(out_nodes),
        order(out_order) {
    for (int t = 0; t < n; t++) {
      for (int a = 0; a < 3; a++) {
        const double p0 = pos[t * 9 + a], p1 = pos[t * 9 + 3 + a], p2 = pos[t * 9 + 6 + a];
        const double mn = std::min({p0, p1, p2}), mx = std::max({p0, p1, p2});
        lo[t * 3 + a] = (float)mn;
        hi[t * 3 + a] = (float)mx;
        cen[t * 3 + a] = (float)((mn + mx) * 0.5);
      }
      order[t] = (uint32_t)t;
    }
    std::fill(nodes, nodes + (size_t)std::max(1, 2 * n) * 8, 0.0f);
  }

  void set_bounds(int node, int first, int count) {
    const double inf = std::numeric_limits<double>::infinity();
    double b[6] = {inf, inf, inf, -inf, -inf, -inf};
    for (int i = first; i < first + count; i++) {
      const size_t t = (size_t)order[i] * 3;
      for (int a = 0; a < 3; a++) {
        if (lo[t + a] < b[a]) b[a] = lo[t + a];
        if (hi[t + a] > b[3 + a]) b[3 + a] = hi[t + a];
      }
    }
    float *o = nodes + (size_t)node * 8;
    o[0] = (float)b[0]; o[1] = (float)b[1]; o[2] = (float)b[2];
    o[4] = (float)b[3]; o[5] = (float)b[4]; o[6] = (float)b[5];
  }

  void make_leaf(int node, int first, int count) {
    word((size_t)node * 8 + 3) = (uint32_t)first;
    word((size_t)node * 8 + 7) = (uint32_t)count;
  }

  int bin_of(size_t t, int a, double c0, double scale) const {
    return std::min(BINS - 1, (int)((cen[t * 3 + a] - c0) * scale));
  }

  void build() {
    struct Job { int node, first, count, depth; };
    std::vector<Job> todo{{0, 0, n, 0}};
    const double inf = std::numeric_limits<double>::infinity();
    const float finf = std::numeric_limits<float>::infinity();
    while (!todo.empty()) {
      const Job j = todo.back();
      todo.pop_back();
      max_depth = std::max(max_depth, j.depth);
      set_bounds(j.node, j.first, j.count);
      if (j.count <= MAX_LEAF) { make_leaf(j.node, j.first, j.count); continue; }
      double c0[3] = {inf, inf, inf}, c1[3] = {-inf, -inf, -inf};
      for (int i = j.first; i < j.first + j.count; i++)
        for (int a = 0; a < 3; a++) {
          const double c = cen[(size_t)order[i] * 3 + a];
          c0[a] = c < c0[a] ? c : c0[a];
          c1[a] = c > c1[a] ? c : c1[a];
        }
      // bins of all three axes in one pass
      float bmin[3][BINS][3], bmax[3][BINS][3];
      uint32_t bcnt[3][BINS] = {};
      double scale[3];
      bool live[3];
      for (int a = 0; a < 3; a++) {
        live[a] = c1[a] - c0[a] > 1e-12;
        scale[a] = live[a] ? BINS / (c1[a] - c0[a]) : 0.0;
        for (int b = 0; b < BINS; b++)
          for (int k = 0; k < 3; k++) { bmin[a][b][k] = finf; bmax[a][b][k] = -finf; }
      }
      for (int i = j.first; i < j.first + j.count; i++) {
        const size_t t = order[i];
        for (int a = 0; a < 3; a++) {
          if (!live[a]) continue;
          const int b = bin_of(t, a, c0[a], scale[a]);
          bcnt[a][b]++;
          for (int k = 0; k < 3; k++) {
            bmin[a][b][k] = std::min(bmin[a][b][k], lo[t * 3 + k]);
            bmax[a][b][k] = std::max(bmax[a][b][k], hi[t * 3 + k]);
          }
        }
      }
      double best = inf;
      int best_axis = -1, best_split = 0;
      for (int a = 0; a < 3; a++) {
        if (!live[a]) continue;
        double r_area[BINS] = {}, rb[6] = {inf, inf, inf, -inf, -inf, -inf};
        uint32_t r_cnt[BINS] = {}, rc = 0;
        for (int b = BINS - 1; b > 0; b--) {  // sweep from the right
          rc += bcnt[a][b];
          for (int k = 0; k < 3; k++) {
            rb[k] = std::min(rb[k], (double)bmin[a][b][k]);
            rb[3 + k] = std::max(rb[3 + k], (double)bmax[a][b][k]);
          }
          r_area[b] = rc ? area(rb[3] - rb[0], rb[4] - rb[1], rb[5] - rb[2]) : 0;
          r_cnt[b] = rc;
        }
        double lb[6] = {inf, inf, inf, -inf, -inf, -inf};
        uint32_t lc = 0;
        for (int b = 0; b < BINS - 1; b++) {
          lc += bcnt[a][b];
          for (int k = 0; k < 3; k++) {
            lb[k] = std::min(lb[k], (double)bmin[a][b][k]);
            lb[3 + k] = std::max(lb[3 + k], (double)bmax[a][b][k]);
          }
          if (!lc || !r_cnt[b + 1]) continue;
          const double cost = lc * area(lb[3] - lb[0], lb[4] - lb[1], lb[5] - lb[2]) + r_cnt[b + 1] * r_area[b + 1];
          if (cost < best) { best = cost; best_axis = a; best_split = b + 1; }
        }
      }
      const float *o = nodes + (size_t)j.node * 8;
      const double leaf_cost = j.count * area((double)o[4] - o[0], (double)o[5] - o[1], (double)o[6] - o[2]);
      int mid;
      if (best_axis < 0) {
        mid = j.first + (j.count >> 1);  // all centroids coincide: split by index
      } else if (best >= leaf_cost && j.count <= 16) {
        make_leaf(j.node, j.first, j.count);
        continue;
      } else {
        int i = j.first, k = j.first + j.count - 1;
        while (i <= k) {
          if (bin_of(order[i], best_axis, c0[best_axis], scale[best_axis]) < best_split) i++;
          else std::swap(order[i], order[k--]);
        }
        mid = i;
        if (mid == j.first || mid == j.first + j.count) mid = j.first + (j.count >> 1);
      }
      const int left = used;
      used += 2;
      word((size_t)j.node * 8 + 3) = (uint32_t)left;
      word((size_t)j.node * 8 + 7) = 0;
      todo.push_back({left + 1, mid, j.first + j.count - mid, j.depth + 1});
      todo.push_back({left, j.first, mid - j.first, j.depth + 1});
    }
  }
};

// refitBVH (bvh.js:147-171): reverse walk = bottom-up; tri_pos 9 floats per triangle in BVH order
void refit(float *nodes, int node_count, const float *tri_pos) {
  const uint32_t *w = reinterpret_cast<const uint32_t *>(nodes);
  const double inf = std::numeric_limits<double>::infinity();
  for (int nd = node_count - 1; nd >= 0; nd--) {
    float *o = nodes + (size_t)nd * 8;
    const uint32_t count = w[(size_t)nd * 8 + 7];
    double b[6] = {inf, inf, inf, -inf, -inf, -inf};
    if (count > 0) {
      const uint32_t first = w[(size_t)nd * 8 + 3];
      for (uint32_t t = first; t < first + count; t++)
        for (int v = 0; v < 3; v++)
          for (int a = 0; a < 3; a++) {
            const double x = tri_pos[(size_t)t * 9 + v * 3 + a];
            b[a] = x < b[a] ? x : b[a];
            b[3 + a] = x > b[3 + a] ? x : b[3 + a];
          }
    } else {
      const float *l = nodes + (size_t)w[(size_t)nd * 8 + 3] * 8, *r = l + 8;
      for (int a = 0; a < 3; a++) {
        b[a] = std::min(l[a], r[a]);
        b[3 + a] = std::max(l[4 + a], r[4 + a]);
      }
    }
    for (int a = 0; a < 3; a++) { o[a] = (float)b[a]; o[4 + a] = (float)b[3 + a]; }
  }
}

int packed_count(const float *nodes, int node_count) {
  const uint32_t *w = reinterpret_cast<const uint32_t *>(nodes);
  int k = 0;
  for (int nd = 0; nd < node_count; nd++) k += w[(size_t)nd * 8 + 7] == 0;
  return std::max(k, 1);
}

// packBVH (bvh.js:186-210): one 64-byte record per interior node holding both children's boxes
void pack(const float *nodes, int node_count, float *out) {
  const uint32_t *w = reinterpret_cast<const uint32_t *>(nodes);
  uint32_t *ow = reinterpret_cast<uint32_t *>(out);
  std::vector<int> id(node_count, -1);
  int k = 0;
  for (int nd = 0; nd < node_count; nd++)
    if (w[(size_t)nd * 8 + 7] == 0) id[nd] = k++;
  auto put = [&](size_t o, size_t c) {
    const float *s = nodes + c * 8;
    for (int a = 0; a < 3; a++) { out[o + a] = s[a]; out[o + 4 + a] = s[4 + a]; }
    const uint32_t count = w[c * 8 + 7];
    ow[o + 3] = count > 0 ? w[c * 8 + 3] : (uint32_t)id[c];
    ow[o + 7] = count;
  };
  if (k == 0) {  // a single leaf: one packed node with the leaf on both sides
    put(0, 0);
    put(8, 0);
    return;
  }
  for (int nd = 0; nd < node_count; nd++) {
    if (id[nd] < 0) continue;
    const size_t l = w[(size_t)nd * 8 + 3];
    put((size_t)id[nd] * 16, l);
    put((size_t)id[nd] * 16 + 8, l + 1);
  }
}

// f16 bits of log2(texels per world unit) of a triangle (scene.js computeTriLod 178-208, with its truncating
// float -> half conversion that flushes f16 subnormals to zero)
uint16_t tri_lod(const float *va, const float *vb, const float *vc) {
  const double e1[3] = {(double)vb[0] - va[0], (double)vb[1] - va[1], (double)vb[2] - va[2]};
  const double e2[3] = {(double)vc[0] - va[0], (double)vc[1] - va[1], (double)vc[2] - va[2]};
  const double wa = std::hypot(e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                               e1[0] * e2[1] - e1[1] * e2[0]) * 0.5;
  const double ua = std::fabs(((double)vb[3] - va[3]) * ((double)vc[11] - va[11]) -
                              ((double)vb[11] - va[11]) * ((double)vc[3] - va[3])) * 0.5;
  const double lod = wa > 1e-12 && ua > 1e-14 ? std::log2(std::sqrt(ua / wa) * HUSH_PT_TEX_SIZE) : 0.0;
  const uint32_t x = f_as_u((float)lod);
  const int e = (int)((x >> 23) & 0xffu) - 112;
  const uint32_t sign = (x >> 16) & 0x8000u;
  if (e <= 0) return (uint16_t)sign;
  if (e >= 31) return (uint16_t)(sign | 0x7c00u);
  return (uint16_t)(sign | ((uint32_t)e << 10) | ((x >> 13) & 0x3ffu));
}

// rgba8 image -> 1024^2 level (bilinear, clamp to edge, texel centres) + 2x2 box mips
std::vector<uint8_t> make_mip_chain(const uint8_t *rgba, int w, int h) {
  const int S = HUSH_PT_TEX_SIZE;
  std::vector<uint8_t> out(pt::tex_layer_bytes());
  uint8_t *l0 = out.data();
  for (int y = 0; y < S; y++)
    for (int x = 0; x < S; x++) {
      const float sx = ((float)x + 0.5f) * (float)w / (float)S - 0.5f, sy = ((float)y + 0.5f) * (float)h / (float)S - 0.5f;
      const int x0 = (int)std::floor(sx), y0 = (int)std::floor(sy);
      const float fx = sx - (float)x0, fy = sy - (float)y0;
      auto at = [&](int xi, int yi, int c) {
        return (float)rgba[((size_t)std::clamp(yi, 0, h - 1) * w + std::clamp(xi, 0, w - 1)) * 4 + c];
      };
      for (int c = 0; c < 4; c++) {
        const float v = (at(x0, y0, c) * (1 - fx) + at(x0 + 1, y0, c) * fx) * (1 - fy) +
                        (at(x0, y0 + 1, c) * (1 - fx) + at(x0 + 1, y0 + 1, c) * fx) * fy;
        l0[((size_t)y * S + x) * 4 + c] = (uint8_t)std::lround(std::clamp(v, 0.0f, 255.0f));
      }
    }
  size_t off = (size_t)S * S * 4;
  const uint8_t *prev = l0;
  for (int m = 1; m < HUSH_PT_TEX_MIPS; m++) {
    const int ps = std::max(1, S >> (m - 1)), s = std::max(1, S >> m);
    uint8_t *cur = out.data() + off;
    for (int y = 0; y < s; y++)
      for (int x = 0; x < s; x++)
        for (int c = 0; c < 4; c++) {
          const int x0 = std::min(2 * x, ps - 1), x1 = std::min(2 * x + 1, ps - 1);
          const int y0 = std::min(2 * y, ps - 1), y1 = std::min(2 * y + 1, ps - 1);
          const int sum = prev[((size_t)y0 * ps + x0) * 4 + c] + prev[((size_t)y0 * ps + x1) * 4 + c] +
                          prev[((size_t)y1 * ps + x0) * 4 + c] + prev[((size_t)y1 * ps + x1) * 4 + c];
          cur[((size_t)y * s + x) * 4 + c] = (uint8_t)((sum + 2) / 4);
        }
    prev = cur;
    off += (size_t)s * s * 4;
  }
  return out;
}

}  // namespace

namespace pt {

size_t tex_layer_bytes() {
  size_t b = 0;
  for (int m = 0; m < HUSH_PT_TEX_MIPS; m++) {
    const size_t s = (size_t)std::max(1, HUSH_PT_TEX_SIZE >> m);
    b += s * s * 4;
  }
  return b;
}

int fail(int code, const std::string &msg) {
  g_pt_err = msg;
  return code;
}

}  // namespace pt

struct PtGroup {
  int flags = 0;
  int vert_offset = 0, vert_count = 0, tri_offset = 0, tri_count = 0;
  std::vector<uint32_t> local_idx;  // 4 per triangle (global vertex ids, material), build order
  std::vector<uint32_t> order;      // BVH order -> build order
  std::vector<float> nodes;         // build layout
  int node_count = 0, pack_offset = 0, pack_count = 0;
};

struct hush_pt_scene_s {
  int dev = 0;
  bool built = false;
  std::vector<hush_pt_material> mats;
  std::vector<std::vector<uint8_t>> tex;
  std::vector<PtGroup> groups;
  std::vector<float> verts, tri_pos, tris, nodes;
  std::vector<uint32_t> tri_idx;
  int max_depth = 0;
  // device copies
  void *pool = nullptr;
  float *d_nodes = nullptr, *d_tris = nullptr, *d_verts = nullptr, *d_mats = nullptr;
  uint32_t *d_tri_idx = nullptr;
  uint8_t *d_tex = nullptr;
};

extern "C" const char *hush_pt_last_error(void) { return g_pt_err.c_str(); }

extern "C" hush_pt_material hush_pt_material_default(void) {
  hush_pt_material m;
  const float base[4] = {1, 1, 1, 0}, em[4] = {0, 0, 0, 0}, pbr[4] = {1, 0, 0, 1.5f}, uv[4] = {1, 1, 1, 0};
  std::memcpy(m.base, base, 16);
  std::memcpy(m.emissive, em, 16);
  std::memcpy(m.pbr, pbr, 16);
  std::memcpy(m.uv, uv, 16);
  for (int k = 0; k < 3; k++) m.tex[k] = -1;
  m.tex[3] = 0;
  return m;
}

extern "C" int hush_pt_scene_create(int device, hush_pt_scene_t **out) {
  if (!out) return pt::fail(HUSH_ERR_ARG, "hush_pt_scene_create: out is NULL");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
    return pt::fail(HUSH_ERR_DEVICE, "SceneGPU: no CUDA device " + std::to_string(device));
  *out = new hush_pt_scene_t();
  (*out)->dev = device;
  return HUSH_OK;
}

extern "C" void hush_pt_scene_destroy(hush_pt_scene_t *s) {
  if (!s) return;
  if (s->pool) {
    cudaSetDevice(s->dev);
    cudaFree(s->pool);
  }
  delete s;
}

extern "C" int hush_pt_scene_add_material(hush_pt_scene_t *s, const hush_pt_material *m) {
  if (!s || !m) return pt::fail(-1, "SceneGPU.material: NULL argument"), -1;
  if (s->mats.size() >= 0xffffu) return pt::fail(-1, "SceneGPU.material: more than 65535 materials"), -1;
  s->mats.push_back(*m);
  return (int)s->mats.size() - 1;
}

extern "C" int hush_pt_scene_add_texture(hush_pt_scene_t *s, const uint8_t *rgba, int w, int h) {
  if (!s || !rgba || w <= 0 || h <= 0) return pt::fail(-1, "SceneGPU.texture: bad image"), -1;
  s->tex.push_back(make_mip_chain(rgba, w, h));
  return (int)s->tex.size() - 1;
}

extern "C" int hush_pt_scene_add_group(hush_pt_scene_t *s, int flags, const float *pos, const float *nrm,
                                       const float *uv, int n_verts, const uint32_t *idx, const uint32_t *mat,
                                       int n_tris) {
  if (!s || !pos || !idx || !mat || n_verts <= 0 || n_tris <= 0)
    return pt::fail(-1, "SceneGPU.group: missing vertices or triangles"), -1;
  if (s->built) return pt::fail(-1, "SceneGPU.group: the scene is already built"), -1;
  if ((int)s->groups.size() >= HUSH_PT_MAX_BLAS) return pt::fail(-1, "too many dynamic groups"), -1;  // scene.js:82
  for (int t = 0; t < n_tris; t++) {
    for (int k = 0; k < 3; k++)
      if (idx[t * 3 + k] >= (uint32_t)n_verts)
        return pt::fail(-1, "SceneGPU.group: triangle " + std::to_string(t) + " indexes vertex " +
                                std::to_string(idx[t * 3 + k]) + " of " + std::to_string(n_verts)), -1;
    if (mat[t] >= s->mats.size())
      return pt::fail(-1, "SceneGPU.group: triangle " + std::to_string(t) + " uses unknown material " +
                              std::to_string(mat[t])), -1;
  }
  PtGroup g;
  g.flags = flags & (HUSH_PT_GROUP_DYNAMIC | HUSH_PT_GROUP_NO_SHADOW);
  g.vert_offset = (int)(s->verts.size() / 12);
  g.vert_count = n_verts;
  s->verts.resize(s->verts.size() + (size_t)n_verts * 12, 0.0f);
  for (int i = 0; i < n_verts; i++) {
    float *o = s->verts.data() + (size_t)(g.vert_offset + i) * 12;
    for (int a = 0; a < 3; a++) o[a] = o[4 + a] = pos[i * 3 + a];
    o[3] = uv ? uv[i * 2] : 0.0f;
    o[11] = uv ? uv[i * 2 + 1] : 0.0f;
    float n[3] = {0, 1, 0};
    if (nrm) {
      const double l = std::hypot((double)nrm[i * 3], (double)nrm[i * 3 + 1], (double)nrm[i * 3 + 2]);
      for (int a = 0; a < 3; a++) n[a] = l > 0 ? (float)(nrm[i * 3 + a] / l) : 0.0f;
    }
    o[8] = n[0]; o[9] = n[1]; o[10] = n[2];
  }
  g.tri_count = n_tris;
  g.local_idx.resize((size_t)n_tris * 4);
  for (int t = 0; t < n_tris; t++) {
    for (int k = 0; k < 3; k++) g.local_idx[t * 4 + k] = (uint32_t)g.vert_offset + idx[t * 3 + k];
    g.local_idx[t * 4 + 3] = mat[t];
  }
  s->groups.push_back(std::move(g));
  return (int)s->groups.size() - 1;
}

static void pack_tris(hush_pt_scene_t *s, int first, int count) {
  for (int t = first; t < first + count; t++) {
    const float *p = s->tri_pos.data() + (size_t)t * 9;
    float *o = s->tris.data() + (size_t)t * 12;
    const hush_pt_material &m = s->mats[s->tri_idx[(size_t)t * 4 + 3] & 0xffffu];
    o[0] = p[0]; o[1] = p[1]; o[2] = p[2];
    o[3] = m.base[3] > 0 && m.tex[0] >= 0 ? 1.0f : 0.0f;
    for (int k = 1; k < 3; k++) {
      for (int a = 0; a < 3; a++) o[k * 4 + a] = p[k * 3 + a] - p[a];
      o[k * 4 + 3] = 0.0f;
    }
  }
}

// triangle positions of a group in BVH order from the current vertices
static void gather_tri_pos(hush_pt_scene_t *s, const PtGroup &g) {
  for (int i = 0; i < g.tri_count; i++) {
    const uint32_t src = g.order[i];
    float *dst = s->tri_pos.data() + (size_t)(g.tri_offset + i) * 9;
    for (int k = 0; k < 3; k++) {
      const float *v = s->verts.data() + (size_t)g.local_idx[src * 4 + k] * 12;
      dst[k * 3] = v[0]; dst[k * 3 + 1] = v[1]; dst[k * 3 + 2] = v[2];
    }
  }
}

static int upload(hush_pt_scene_t *s) {
  cudaSetDevice(s->dev);
  if (s->pool) cudaFree(s->pool);
  s->pool = nullptr;
  size_t mats_bytes = std::max<size_t>(1, s->mats.size()) * sizeof(hush_pt_material);
  const size_t tex_bytes = std::max<size_t>(1, s->tex.size()) * pt::tex_layer_bytes();
  const size_t parts[6] = {s->nodes.size() * 4, s->tris.size() * 4, s->tri_idx.size() * 4, s->verts.size() * 4,
                           mats_bytes, tex_bytes};
  size_t off[6], total = 0;
  for (int k = 0; k < 6; k++) {
    off[k] = total;
    total += (parts[k] + 255) & ~(size_t)255;
  }
  cudaError_t e = cudaMalloc(&s->pool, total);
  if (e != cudaSuccess) {
    s->pool = nullptr;
    return pt::fail(HUSH_ERR_CUDA, std::string("SceneGPU.upload: cudaMalloc: ") + cudaGetErrorString(e));
  }
  char *b = static_cast<char *>(s->pool);
  s->d_nodes = reinterpret_cast<float *>(b + off[0]);
  s->d_tris = reinterpret_cast<float *>(b + off[1]);
  s->d_tri_idx = reinterpret_cast<uint32_t *>(b + off[2]);
  s->d_verts = reinterpret_cast<float *>(b + off[3]);
  s->d_mats = reinterpret_cast<float *>(b + off[4]);
  s->d_tex = reinterpret_cast<uint8_t *>(b + off[5]);
  const void *src[5] = {s->nodes.data(), s->tris.data(), s->tri_idx.data(), s->verts.data(), s->mats.data()};
  void *dst[5] = {s->d_nodes, s->d_tris, s->d_tri_idx, s->d_verts, s->d_mats};
  for (int k = 0; k < 5 && e == cudaSuccess; k++)
    if (parts[k] && (k != 4 || !s->mats.empty())) e = cudaMemcpy(dst[k], src[k], parts[k], cudaMemcpyHostToDevice);
  for (size_t l = 0; l < s->tex.size() && e == cudaSuccess; l++)
    e = cudaMemcpy(s->d_tex + l * pt::tex_layer_bytes(), s->tex[l].data(), pt::tex_layer_bytes(),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return pt::fail(HUSH_ERR_CUDA, std::string("SceneGPU.upload: ") + cudaGetErrorString(e));
  return HUSH_OK;
}

// SceneGPU.build (scene.js:64-176) from the added groups
extern "C" int hush_pt_scene_build(hush_pt_scene_t *s) {
  if (!s) return pt::fail(HUSH_ERR_ARG, "SceneGPU.build: NULL scene");
  if (s->built) return pt::fail(HUSH_ERR_ARG, "SceneGPU.build: already built");
  if (s->groups.empty()) return pt::fail(HUSH_ERR_ARG, "SceneGPU.build: the scene has no triangles");
  for (size_t m = 0; m < s->mats.size(); m++)
    for (int k = 0; k < 3; k++)
      if (s->mats[m].tex[k] >= (int32_t)s->tex.size())
        return pt::fail(HUSH_ERR_ARG, "SceneGPU.build: material " + std::to_string(m) + " uses texture layer " +
                                          std::to_string(s->mats[m].tex[k]) + " of " + std::to_string(s->tex.size()));
  int tri_total = 0;
  for (auto &g : s->groups) {
    g.tri_offset = tri_total;
    tri_total += g.tri_count;
  }
  s->tri_pos.assign((size_t)tri_total * 9, 0.0f);
  s->tri_idx.assign((size_t)tri_total * 4, 0u);
  s->tris.assign((size_t)tri_total * 12, 0.0f);
  int node_off = 0;
  s->max_depth = 0;
  std::vector<float> local;
  for (auto &g : s->groups) {
    local.assign((size_t)g.tri_count * 9, 0.0f);  // build-order triangle positions
    for (int t = 0; t < g.tri_count; t++)
      for (int k = 0; k < 3; k++) {
        const float *v = s->verts.data() + (size_t)g.local_idx[t * 4 + k] * 12;
        for (int a = 0; a < 3; a++) local[(size_t)t * 9 + k * 3 + a] = v[a];
      }
    g.order.assign(g.tri_count, 0u);
    g.nodes.assign((size_t)std::max(1, 2 * g.tri_count) * 8, 0.0f);
    SahBuilder b(local.data(), g.tri_count, g.nodes.data(), g.order.data());
    b.build();
    g.node_count = b.used;
    g.nodes.resize((size_t)b.used * 8);
    s->max_depth = std::max(s->max_depth, b.max_depth);
    g.pack_count = packed_count(g.nodes.data(), g.node_count);
    g.pack_offset = node_off;
    node_off += g.pack_count;
    for (int i = 0; i < g.tri_count; i++) {
      const uint32_t src = g.order[i];
      std::memcpy(&s->tri_pos[(size_t)(g.tri_offset + i) * 9], &local[(size_t)src * 9], 36);
      std::memcpy(&s->tri_idx[(size_t)(g.tri_offset + i) * 4], &g.local_idx[(size_t)src * 4], 16);
    }
  }
  if (s->max_depth > 32)
    return pt::fail(HUSH_ERR_ARG, "SceneGPU.build: BVH depth " + std::to_string(s->max_depth) +
                                      " exceeds the traversal stack (32)");
  s->nodes.assign((size_t)node_off * 16, 0.0f);
  for (auto &g : s->groups) pack(g.nodes.data(), g.node_count, s->nodes.data() + (size_t)g.pack_offset * 16);
  for (int t = 0; t < tri_total; t++) {
    uint32_t *ti = &s->tri_idx[(size_t)t * 4];
    const uint16_t lod = tri_lod(&s->verts[(size_t)ti[0] * 12], &s->verts[(size_t)ti[1] * 12],
                                 &s->verts[(size_t)ti[2] * 12]);
    ti[3] = (ti[3] & 0xffffu) | ((uint32_t)lod << 16);
  }
  pack_tris(s, 0, tri_total);
  if (int rc = upload(s)) return rc;
  s->built = true;
  return HUSH_OK;
}

// SceneGPU.update for one dynamic group (scene.js:225-270)
extern "C" int hush_pt_scene_update(hush_pt_scene_t *s, int group, const float *pos, const float *nrm, void *stream) {
  if (!s || !pos) return pt::fail(HUSH_ERR_ARG, "SceneGPU.update: NULL argument");
  if (!s->built) return pt::fail(HUSH_ERR_ARG, "SceneGPU.update: build the scene first");
  if (group < 0 || group >= (int)s->groups.size() || !(s->groups[group].flags & HUSH_PT_GROUP_DYNAMIC))
    return pt::fail(HUSH_ERR_ARG, "SceneGPU.update: group " + std::to_string(group) + " is not dynamic");
  PtGroup &g = s->groups[group];
  for (int i = 0; i < g.vert_count; i++) {
    float *o = s->verts.data() + (size_t)(g.vert_offset + i) * 12;
    for (int a = 0; a < 3; a++) {
      o[4 + a] = o[a];
      o[a] = pos[i * 3 + a];
    }
    if (nrm) {
      const double l = std::hypot((double)nrm[i * 3], (double)nrm[i * 3 + 1], (double)nrm[i * 3 + 2]);
      for (int a = 0; a < 3; a++) o[8 + a] = l > 0 ? (float)(nrm[i * 3 + a] / l) : 0.0f;
    }
  }
  if (!nrm) {  // area-weighted smooth normals (scene.js skinnedNormals 272-291)
    for (int i = 0; i < g.vert_count; i++) {
      float *o = s->verts.data() + (size_t)(g.vert_offset + i) * 12;
      o[8] = o[9] = o[10] = 0.0f;
    }
    for (int t = 0; t < g.tri_count; t++) {
      float *v[3];
      for (int k = 0; k < 3; k++) v[k] = s->verts.data() + (size_t)g.local_idx[t * 4 + k] * 12;
      const double e1[3] = {(double)v[1][0] - v[0][0], (double)v[1][1] - v[0][1], (double)v[1][2] - v[0][2]};
      const double e2[3] = {(double)v[2][0] - v[0][0], (double)v[2][1] - v[0][1], (double)v[2][2] - v[0][2]};
      const double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      for (int k = 0; k < 3; k++)
        for (int a = 0; a < 3; a++) v[k][8 + a] = (float)(v[k][8 + a] + n[a]);
    }
    for (int i = 0; i < g.vert_count; i++) {
      float *o = s->verts.data() + (size_t)(g.vert_offset + i) * 12;
      double l = std::hypot((double)o[8], (double)o[9], (double)o[10]);
      if (l == 0) l = 1;
      for (int a = 0; a < 3; a++) o[8 + a] = (float)(o[8 + a] / l);
    }
  }
  gather_tri_pos(s, g);
  refit(g.nodes.data(), g.node_count, s->tri_pos.data() + (size_t)g.tri_offset * 9);
  pack(g.nodes.data(), g.node_count, s->nodes.data() + (size_t)g.pack_offset * 16);
  pack_tris(s, g.tri_offset, g.tri_count);
  cudaSetDevice(s->dev);
  cudaStream_t st = (cudaStream_t)stream;
  // pageable sources: the copies are staged before cudaMemcpyAsync returns, so the host arrays may change after
  cudaError_t e = cudaMemcpyAsync(s->d_nodes + (size_t)g.pack_offset * 16, s->nodes.data() + (size_t)g.pack_offset * 16,
                                  (size_t)g.pack_count * 64, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_tris + (size_t)g.tri_offset * 12, s->tris.data() + (size_t)g.tri_offset * 12,
                        (size_t)g.tri_count * 48, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_verts + (size_t)g.vert_offset * 12, s->verts.data() + (size_t)g.vert_offset * 12,
                        (size_t)g.vert_count * 48, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return pt::fail(HUSH_ERR_CUDA, std::string("SceneGPU.update: ") + cudaGetErrorString(e));
  return HUSH_OK;
}

extern "C" int hush_pt_scene_blas(const hush_pt_scene_t *s, hush_pt_blas *out, int max) {
  if (!s || !s->built) return 0;
  const int n = std::min((int)s->groups.size(), max);
  for (int i = 0; i < n && out; i++) {
    const PtGroup &g = s->groups[i];
    out[i] = hush_pt_blas{(uint32_t)g.pack_offset, (uint32_t)g.tri_offset, (uint32_t)g.pack_count, (uint32_t)g.flags};
  }
  return n;
}

extern "C" int hush_pt_scene_info(const hush_pt_scene_t *s, int *tri_total, int *node_total, int *vert_total,
                                  int *max_depth) {
  if (!s) return pt::fail(HUSH_ERR_ARG, "SceneGPU.info: NULL scene");
  if (tri_total) *tri_total = (int)(s->tri_idx.size() / 4);
  if (node_total) *node_total = (int)(s->nodes.size() / 16);
  if (vert_total) *vert_total = (int)(s->verts.size() / 12);
  if (max_depth) *max_depth = s->max_depth;
  return HUSH_OK;
}

extern "C" int hush_pt_scene_device(const hush_pt_scene_t *s, const void **nodes, const void **tris,
                                    const void **tri_idx, const void **verts, const void **mats, const void **tex) {
  if (!s || !s->built) return pt::fail(HUSH_ERR_ARG, "SceneGPU: not built");
  if (nodes) *nodes = s->d_nodes;
  if (tris) *tris = s->d_tris;
  if (tri_idx) *tri_idx = s->d_tri_idx;
  if (verts) *verts = s->d_verts;
  if (mats) *mats = s->d_mats;
  if (tex) *tex = s->d_tex;
  return HUSH_OK;
}

namespace pt {
SceneView scene_view(const hush_pt_scene_t *s) {
  SceneView v{};
  v.nodes = reinterpret_cast<const float4 *>(s->d_nodes);
  v.tris = reinterpret_cast<const float4 *>(s->d_tris);
  v.tri_idx = reinterpret_cast<const uint4 *>(s->d_tri_idx);
  v.verts = reinterpret_cast<const float4 *>(s->d_verts);
  v.mats = reinterpret_cast<const float4 *>(s->d_mats);
  v.tex = s->d_tex;
  v.tex_layers = (int)s->tex.size();
  return v;
}
int scene_device(const hush_pt_scene_t *s) { return s->dev; }
bool scene_built(const hush_pt_scene_t *s) { return s && s->built; }
}  // namespace pt

extern "C" int hush_pt_bvh_build(const float *pos, int tri_count, float *nodes, uint32_t *order, int *max_depth) {
  if (!pos || !nodes || !order || tri_count < 0) return pt::fail(-1, "hush_pt_bvh_build: bad argument"), -1;
  SahBuilder b(pos, tri_count, nodes, order);
  b.build();
  if (max_depth) *max_depth = b.max_depth;
  return b.used;
}

// ------------------------------------------------------------------------------------------------ envmap.js
namespace {
inline double lum709(double r, double g, double b) { return 0.2126 * r + 0.7152 * g + 0.0722 * b; }
inline void equirect_dir(double u, double v, double d[3]) {  // dirOf (envmap.js:15-18), row 0 = up
  const double phi = (u - 0.5) * 2 * M_PI, th = v * M_PI;
  d[0] = std::cos(phi) * std::sin(th);
  d[1] = std::cos(th);
  d[2] = std::sin(phi) * std::sin(th);
}
uint16_t half_rz(float f) {
  const uint32_t x = f_as_u(f), ax = x & 0x7fffffffu;
  const uint16_t s = (uint16_t)((x >> 16) & 0x8000u);
  if (ax > 0x7f800000u) return s | 0x7fffu;
  if (ax >= 0x477fe000u) return s | 0x7bffu;  // finite values saturate, as the clamp to 65504 does
  if (ax >= 0x38800000u) return (uint16_t)(s | (((ax >> 23) - 112u) << 10) | ((ax >> 13) & 0x3ffu));
  const uint32_t e = ax >> 23;
  if (e <= 102u) return s;
  return (uint16_t)(s | (((ax & 0x7fffffu) | 0x800000u) >> (126u - e)));
}
}  // namespace

extern "C" int hush_pt_env_prepare(float *rgba, int W, int H, int sun, double cone_deg, uint16_t *half_out,
                                   float *table, double sun_dir[3], double sun_irr[3]) {
  if (!rgba || W <= 0 || H <= 0 || !half_out || !table) return pt::fail(-1, "prepareEnvMap: bad image"), -1;
  int has_sun = 0;
  if (sun) {  // cutSun (envmap.js:22-61): the brightest texel's neighbourhood, if much brighter than its ring
    size_t bi = 0;
    double best = 0;
    for (size_t i = 0; i < (size_t)W * H; i++) {
      const double l = lum709(rgba[i * 4], rgba[i * 4 + 1], rgba[i * 4 + 2]);
      if (l > best) { best = l; bi = i; }
    }
    const int by = (int)(bi / W);
    double s[3];
    equirect_dir(((double)(bi % W) + 0.5) / W, (by + 0.5) / H, s);
    const double cin = std::cos(cone_deg * M_PI / 180), cout = std::cos(cone_deg * 1.6 * M_PI / 180);
    const int rows = (int)std::ceil(cone_deg * 1.7 * H / 180);
    double ring[3] = {0, 0, 0};
    long nring = 0;
    std::vector<std::pair<size_t, int>> inner;  // texel, row
    std::vector<double> inner_dir;
    for (int y = std::max(0, by - rows); y <= std::min(H - 1, by + rows); y++)
      for (int x = 0; x < W; x++) {
        double d[3];
        equirect_dir((x + 0.5) / W, (y + 0.5) / H, d);
        const double c = d[0] * s[0] + d[1] * s[1] + d[2] * s[2];
        const size_t i = ((size_t)y * W + x) * 4;
        if (c >= cin) {
          inner.push_back({i, y});
          inner_dir.insert(inner_dir.end(), d, d + 3);
        } else if (c >= cout) {
          for (int k = 0; k < 3; k++) ring[k] += rgba[i + k];
          nring++;
        }
      }
    if (nring) {
      for (double &r : ring) r /= nring;
      const double ring_l = lum709(ring[0], ring[1], ring[2]);
      if (best >= 50 * ring_l) {
        double E[3] = {0, 0, 0}, c[3] = {0, 0, 0};
        const double dA = (2 * M_PI / W) * (M_PI / H);
        for (size_t q = 0; q < inner.size(); q++) {
          const size_t i = inner[q].first;
          if (lum709(rgba[i], rgba[i + 1], rgba[i + 2]) < 3 * ring_l) continue;
          const double w = dA * std::sin(((inner[q].second + 0.5) / H) * M_PI);
          double ex[3];
          for (int k = 0; k < 3; k++) {
            ex[k] = std::max(0.0, rgba[i + k] - ring[k]) * w;
            E[k] += ex[k];
            rgba[i + k] = (float)ring[k];
          }
          const double wl = lum709(ex[0], ex[1], ex[2]);
          for (int k = 0; k < 3; k++) c[k] += inner_dir[q * 3 + k] * wl;
        }
        double cl = std::hypot(c[0], c[1], c[2]);
        if (cl == 0) cl = 1;
        for (int k = 0; k < 3; k++) {
          if (sun_dir) sun_dir[k] = c[k] / cl;
          if (sun_irr) sun_irr[k] = E[k];
        }
        has_sun = 1;
      }
    }
  }
  const int GW = HUSH_PT_ENV_GW, GH = HUSH_PT_ENV_GH;
  std::vector<double> wgt((size_t)GW * GH, 0.0);
  for (int y = 0; y < H; y++) {
    const int gy = std::min(GH - 1, (int)std::floor((double)y * GH / H));
    for (int x = 0; x < W; x++) {
      const size_t i = ((size_t)y * W + x) * 4;
      wgt[(size_t)gy * GW + std::min(GW - 1, (int)std::floor((double)x * GW / W))] +=
          lum709(rgba[i], rgba[i + 1], rgba[i + 2]);
    }
  }
  for (int gy = 0; gy < GH; gy++) {
    const double st = std::sin(((gy + 0.5) / GH) * M_PI);
    for (int gx = 0; gx < GW; gx++) wgt[(size_t)gy * GW + gx] = wgt[(size_t)gy * GW + gx] * st + 1e-6;
  }
  for (size_t i = 0; i < (size_t)W * H * 4; i++) half_out[i] = half_rz(std::min(rgba[i], 65000.0f));
  // Vose alias table (envmap.js:64-82): [threshold, alias bits, pmf, 0]
  const size_t N = wgt.size();
  double sum = 0;
  for (double w : wgt) sum += w;
  std::vector<double> p(N);
  std::vector<uint32_t> small, large;
  for (size_t i = 0; i < N; i++) {
    p[i] = wgt[i] / sum * N;
    (p[i] < 1 ? small : large).push_back((uint32_t)i);
  }
  std::fill(table, table + N * 4, 0.0f);
  auto alias_of = [&](size_t i, uint32_t a) { table[i * 4 + 1] = u_as_f(a); };
  while (!small.empty() && !large.empty()) {
    const uint32_t sm = small.back(), lg = large.back();
    small.pop_back();
    table[(size_t)sm * 4] = (float)p[sm];
    alias_of(sm, lg);
    p[lg] -= 1 - p[sm];
    if (p[lg] < 1) {
      large.pop_back();
      small.push_back(lg);
    }
  }
  for (uint32_t i : small) { table[(size_t)i * 4] = 1; alias_of(i, i); }
  for (uint32_t i : large) { table[(size_t)i * 4] = 1; alias_of(i, i); }
  for (size_t i = 0; i < N; i++) table[i * 4 + 2] = (float)(wgt[i] / sum);
  return has_sun;
}

extern "C" void hush_pt_jitter(float out[32]) {
  for (int i = 1; i <= 16; i++) {
    double v[2];
    const int bases[2] = {2, 3};
    for (int k = 0; k < 2; k++) {  // radical inverse of i in base 2 / 3
      double f = 1, r = 0;
      for (int j = i; j > 0; j /= bases[k]) {
        f /= bases[k];
        r += f * (j % bases[k]);
      }
      v[k] = r - 0.5;
    }
    out[2 * (i - 1)] = (float)v[0];
    out[2 * (i - 1) + 1] = (float)v[1];
  }
}
