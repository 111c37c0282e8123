// Display post of the demo (src/demo/post.js) as CUDA kernels writing a headless target buffer: split-screen
// composite of up to three linear HDR images, a six-level bloom pyramid (13-tap downsample with a Karis average on
// the first level, 3x3 tent upsample added onto the next larger level), then bloom mix, vignette, AgX tone mapping,
// sRGB and the divider line. The reference draws these as full-screen render passes into a canvas; here every pass
// is a compute kernel over one image, with the fragment position, the clamp-to-edge bilinear sampler and the
// additive blend written out explicitly:
//   * fragment (x, y) of a W x H target sits at uv = ((x + 0.5) / W, (y + 0.5) / H) (full-screen triangle,
//     post.js:10-17);
//   * the sampler (post.js:154) interpolates at uv * size - 0.5 with f32 weights, texel indices clamped to the edge;
//   * rgba16float targets are written rounded toward zero (the denoiser's storage rounding); the one + one blend of
//     the upsample (post.js:149) adds in f32 before that rounding;
//   * the final target is rgba8 / bgra8 unorm (rounded to nearest) or rgba32f (the colour before quantisation).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "common.cuh"
#include "hush.h"
#include "hush_internal.h"

using namespace hush;

namespace {

constexpr int LEVELS = HUSH_POST_LEVELS;  // post.js:135
constexpr int BX = 32, BY = 8;

HD_INL float3 ld3(const uint2 *__restrict__ img, int w, int x, int y) {
  const float4 t = h4_to_f4(__ldg(img + y * w + x));
  return make_float3(t.x, t.y, t.z);
}
HD_INL float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
HD_INL float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
HD_INL float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
HD_INL float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
HD_INL float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HD_INL float3 mix3(float3 a, float3 b, float t) { return a * (1.0f - t) + b * t; }  // WGSL mix

// textureSampleLevel(tex, clamp-to-edge linear sampler, uv, 0)
HD_INL float3 sample(const uint2 *__restrict__ img, int w, int h, float u, float v) {
  const float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
  const float x0 = floorf(x), y0 = floorf(y);
  const float fx = x - x0, fy = y - y0;
  const int ix = (int)x0, iy = (int)y0;
  const int xa = clampi(ix, 0, w - 1), xb = clampi(ix + 1, 0, w - 1);
  const int ya = clampi(iy, 0, h - 1), yb = clampi(iy + 1, 0, h - 1);
  const float3 top = ld3(img, w, xa, ya) * (1.0f - fx) + ld3(img, w, xb, ya) * fx;
  const float3 bot = ld3(img, w, xa, yb) * (1.0f - fx) + ld3(img, w, xb, yb) * fx;
  return top * (1.0f - fy) + bot * fy;
}

HD_INL uint2 pack_rgb1(float3 c, float a) { return f4_to_h4(make_float4(c.x, c.y, c.z, a)); }

// COMPOSITE (post.js:27-38): left | mid | right at split / split2, times exposure; same = each third shows the
// middle third of its image.
__global__ void k_post_composite(const uint2 *__restrict__ left, const uint2 *__restrict__ right,
                                 const uint2 *__restrict__ mid, int W, int H, float split, float split2, float exposure,
                                 int same, uint2 *__restrict__ hdr) {
  const int x = blockIdx.x * BX + threadIdx.x, y = blockIdx.y * BY + threadIdx.y;
  if (x >= W || y >= H) return;
  const float u = __fdiv_rn((float)x + 0.5f, (float)W);  // IEEE: compared against the split positions
  int px = x;
  if (same) px = px - (min(px * 3 / W, 2) - 1) * (W / 3);
  const uint2 *src = u < split ? left : (u < split2 ? mid : right);
  float3 c = ld3(src, W, px, y);
  c = make_float3(fmaxf(c.x, 0.0f) * exposure, fmaxf(c.y, 0.0f) * exposure, fmaxf(c.z, 0.0f) * exposure);
  hdr[y * W + x] = pack_rgb1(c, 1.0f);
}

HD_INL float karis_w(float3 c) { return 1.0f / (1.0f + (c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f)); }

// DOWN (post.js:50-64): 13 bilinear taps of src around the destination fragment (x, y), Karis-weighted on the first
// level.
template <bool KARIS>
HD_INL void down_texel(const uint2 *__restrict__ src, int sw, int sh, uint2 *__restrict__ dst, int dw, int dh, int x,
                       int y) {
  const float u = ((float)x + 0.5f) / (float)dw, v = ((float)y + 0.5f) / (float)dh;
  const float tx = 1.0f / (float)sw, ty = 1.0f / (float)sh;
  auto s = [&](float ox, float oy) { return sample(src, sw, sh, u + ox * tx, v + oy * ty); };
  const float3 a = s(-2.f, -2.f), b = s(0.f, -2.f), c = s(2.f, -2.f), d = s(-2.f, 0.f), e = s(0.f, 0.f),
               f = s(2.f, 0.f), g = s(-2.f, 2.f), h = s(0.f, 2.f), k = s(2.f, 2.f), j = s(-1.f, -1.f),
               l = s(1.f, -1.f), m = s(-1.f, 1.f), n = s(1.f, 1.f);
  float3 o;
  if constexpr (KARIS) {
    const float3 g0 = (a + b + d + e) * 0.25f, g1 = (b + c + e + f) * 0.25f, g2 = (d + e + g + h) * 0.25f,
                 g3 = (e + f + h + k) * 0.25f, g4 = (j + l + m + n) * 0.25f;
    const float w0 = karis_w(g0) * 0.125f, w1 = karis_w(g1) * 0.125f, w2 = karis_w(g2) * 0.125f,
                w3 = karis_w(g3) * 0.125f, w4 = karis_w(g4) * 0.5f;
    o = (g0 * w0 + g1 * w1 + g2 * w2 + g3 * w3 + g4 * w4) / (w0 + w1 + w2 + w3 + w4);
  } else {
    o = e * 0.125f + (a + c + g + k) * 0.03125f + (b + d + f + h) * 0.0625f + (j + l + m + n) * 0.125f;
  }
  dst[y * dw + x] = pack_rgb1(o, 1.0f);
}

// UP (post.js:74-80) at destination texel (x, y), added onto it (the one + one blend of post.js:149).
HD_INL void up_texel(const uint2 *__restrict__ src, int sw, int sh, uint2 *__restrict__ dst, int dw, int dh, int x,
                     int y) {
  const float u = ((float)x + 0.5f) / (float)dw, v = ((float)y + 0.5f) / (float)dh;
  const float tx = 1.0f / (float)sw, ty = 1.0f / (float)sh;
  auto t = [&](float ox, float oy) { return sample(src, sw, sh, u + ox * tx, v + oy * ty); };
  float3 o = t(0.f, 0.f) * 4.0f;
  o = o + (t(-1.f, 0.f) + t(1.f, 0.f) + t(0.f, -1.f) + t(0.f, 1.f)) * 2.0f;
  o = o + t(-1.f, -1.f) + t(1.f, -1.f) + t(-1.f, 1.f) + t(1.f, 1.f);
  o = o / 16.0f;
  const float4 d = h4_to_f4(dst[y * dw + x]);
  dst[y * dw + x] = f4_to_h4(make_float4(d.x + o.x, d.y + o.y, d.z + o.z, d.w + 1.0f));
}

template <bool KARIS>
__global__ void k_post_down(const uint2 *__restrict__ src, int sw, int sh, uint2 *__restrict__ dst, int dw, int dh) {
  const int x = blockIdx.x * BX + threadIdx.x, y = blockIdx.y * BY + threadIdx.y;
  if (x < dw && y < dh) down_texel<KARIS>(src, sw, sh, dst, dw, dh, x, y);
}

__global__ void k_post_up(const uint2 *__restrict__ src, int sw, int sh, uint2 *__restrict__ dst, int dw, int dh) {
  const int x = blockIdx.x * BX + threadIdx.x, y = blockIdx.y * BY + threadIdx.y;
  if (x < dw && y < dh) up_texel(src, sw, sh, dst, dw, dh, x, y);
}

// mat3x3f(c0, c1, c2) * v, columns c0..c2 (WGSL matrices are column-major)
HD_INL float3 mul3(const float *m, float3 v) {
  return make_float3(m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
                     m[2] * v.x + m[5] * v.y + m[8] * v.z);
}

__constant__ float c_to2020[9] = {0.6274f, 0.0691f, 0.0164f, 0.3293f, 0.9195f, 0.0880f, 0.0433f, 0.0113f, 0.8956f};
__constant__ float c_toSrgb[9] = {1.6605f, -0.1246f, -0.0182f, -0.5876f, 1.1329f, -0.1006f, -0.0728f, -0.0083f, 1.1187f};
__constant__ float c_inset[9] = {0.856627153315983f, 0.137318972929847f, 0.11189821299995f,
                                 0.0951212405381588f, 0.761241990602591f, 0.0767994186031903f,
                                 0.0482516061458583f, 0.101439036467562f, 0.811302368396859f};
__constant__ float c_outset[9] = {1.1271005818144368f, -0.1413297634984383f, -0.14132976349843826f,
                                  -0.11060664309660323f, 1.157823702216272f, -0.11060664309660294f,
                                  -0.016493938717834573f, -0.016493938717834257f, 1.2519364065950405f};

HD_INL float agx_contrast(float x) {  // post.js:90-94
  const float x2 = x * x, x4 = x2 * x2;
  return 15.5f * x4 * x2 - 40.14f * x4 * x + 31.96f * x4 - 6.868f * x2 * x + 0.4298f * x2 + 0.1191f * x - 0.00232f;
}

// agx (post.js:95-114): inset of the Rec.2020 colour, log2 encoding over [minEv, maxEv], the contrast polynomial,
// the look (pow 1.22, saturation 1.15), outset, pow 2.2, back to sRGB primaries.
HD_INL float3 agx(float3 c0) {
  const float minEv = -12.47393f, maxEv = 4.026069f;
  float3 c = mul3(c_inset, mul3(c_to2020, c0));
  auto lg = [&](float v) { return fminf(fmaxf((log2f(fmaxf(v, 1e-10f)) - minEv) / (maxEv - minEv), 0.0f), 1.0f); };
  c = make_float3(agx_contrast(lg(c.x)), agx_contrast(lg(c.y)), agx_contrast(lg(c.z)));
  const float l = c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f;
  c = make_float3(powf(fmaxf(c.x, 0.0f), 1.22f), powf(fmaxf(c.y, 0.0f), 1.22f), powf(fmaxf(c.z, 0.0f), 1.22f));
  c = make_float3(l, l, l) + (c - make_float3(l, l, l)) * 1.15f;
  c = mul3(c_outset, c);
  c = make_float3(powf(fmaxf(0.0f, c.x), 2.2f), powf(fmaxf(0.0f, c.y), 2.2f), powf(fmaxf(0.0f, c.z), 2.2f));
  c = mul3(c_toSrgb, c);
  return make_float3(fminf(fmaxf(c.x, 0.0f), 1.0f), fminf(fmaxf(c.y, 0.0f), 1.0f), fminf(fmaxf(c.z, 0.0f), 1.0f));
}

HD_INL float srgb1(float c) { return c <= 0.0031308f ? c * 12.92f : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f; }

HD_INL uint8_t unorm8(float v) { return (uint8_t)__float2uint_rn(fminf(fmaxf(v, 0.0f), 1.0f) * 255.0f); }

struct FinalArgs {
  float split, split2, line, bloom, vignette;
  int format;
};

// FINAL (post.js:116-132) into the OW x OH target. EXACT2: the target has the HDR image's size and the bloom level is
// exactly half of it (even sizes), the usual case. Then the HDR sample falls on the pixel's own texel and the nine
// bilinear bloom samples, which share one sub-texel phase, collapse into a separable 4 x 4 kernel over bloom texels
// (per axis [0.25, 1.25, 1.75, 0.75] from texel m - 2 for even pixels, mirrored from m - 1 for odd ones; sum 4):
// 16 texel reads instead of 36. The weights are the bilinear and tent weights multiplied out exactly.
template <bool EXACT2>
__global__ void k_post_final(const uint2 *__restrict__ hdr, int W, int H, const uint2 *__restrict__ bl, int bw, int bh,
                             void *__restrict__ target, int OW, int OH, size_t pitch, FinalArgs a) {
  const int x = blockIdx.x * BX + threadIdx.x, y = blockIdx.y * BY + threadIdx.y;
  if (x >= OW || y >= OH) return;
  // the fragment position with IEEE division: the divider line compares it against a pixel threshold
  const float u = __fdiv_rn((float)x + 0.5f, (float)OW), v = __fdiv_rn((float)y + 0.5f, (float)OH);
  float3 c, b;
  if constexpr (EXACT2) {
    c = ld3(hdr, W, x, y);
    const int mx = x >> 1, my = y >> 1;
    const int x0 = (x & 1) ? mx - 1 : mx - 2, y0 = (y & 1) ? my - 1 : my - 2;
    const float we[4] = {0.25f, 1.25f, 1.75f, 0.75f}, wo[4] = {0.75f, 1.75f, 1.25f, 0.25f};
    b = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int yy = clampi(y0 + j, 0, bh - 1);
      const float wy = (y & 1) ? wo[j] : we[j];
      float3 r = make_float3(0.f, 0.f, 0.f);
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const float wx = (x & 1) ? wo[i] : we[i];
        r = r + ld3(bl, bw, clampi(x0 + i, 0, bw - 1), yy) * wx;
      }
      b = b + r * wy;
    }
  } else {
    const float tx = 1.0f / (float)bw, ty = 1.0f / (float)bh;
    c = sample(hdr, W, H, u, v);
    b = sample(bl, bw, bh, u, v) * 4.0f;
    b = b + (sample(bl, bw, bh, u - tx, v) + sample(bl, bw, bh, u + tx, v) + sample(bl, bw, bh, u, v - ty) +
             sample(bl, bw, bh, u, v + ty)) * 2.0f;
    b = b + sample(bl, bw, bh, u - tx, v - ty) + sample(bl, bw, bh, u + tx, v + ty) +
        sample(bl, bw, bh, u + tx, v - ty) + sample(bl, bw, bh, u - tx, v + ty);
  }
  c = mix3(c, b / 16.0f, a.bloom);
  const float qx = (u - 0.5f) * 1.0f, qy = (v - 0.5f) * 0.75f;
  const float vig = 1.0f * (1.0f - a.vignette) + (1.0f - (qx * qx + qy * qy) * 1.6f) * a.vignette;
  c = c * vig;
  const float3 t = agx(c);
  float3 o = make_float3(srgb1(t.x), srgb1(t.y), srgb1(t.z));
  if (a.line > 0.0f && fminf(fabsf(u - a.split), fabsf(u - a.split2)) * (float)OW < a.line)
    o = mix3(o, make_float3(1.0f, 1.0f, 1.0f), 0.85f);
  char *row = reinterpret_cast<char *>(target) + (size_t)y * pitch;
  if (a.format == HUSH_POST_RGBA32F) {
    reinterpret_cast<float4 *>(row)[x] = make_float4(o.x, o.y, o.z, 1.0f);
  } else {
    const uint8_t r = unorm8(o.x), g = unorm8(o.y), bb = unorm8(o.z);
    reinterpret_cast<uchar4 *>(row)[x] =
        a.format == HUSH_POST_BGRA8 ? make_uchar4(bb, g, r, 255) : make_uchar4(r, g, bb, 255);
  }
}

dim3 grid_for(int w, int h) { return dim3((w + BX - 1) / BX, (h + BY - 1) / BY); }

std::string g_post_err;

}  // namespace

struct hush_post_s {
  int dev = 0;
  hush_post_desc d{};
  int W = 0, H = 0;
  char *pool = nullptr;
  uint2 *hdr = nullptr, *lev[LEVELS] = {};
  int lw[LEVELS] = {}, lh[LEVELS] = {};
  std::string last_error;
};

static int post_fail(hush_post_t *p, int code, const std::string &m) {
  (p ? p->last_error : g_post_err) = m;
  return code;
}

extern "C" hush_post_desc hush_post_desc_default(void) {
  hush_post_desc d;
  d.device = 0;
  d.format = HUSH_POST_RGBA8;
  d.bloom = 0.03f;
  d.vignette = 0.35f;
  return d;
}

extern "C" hush_post_inputs hush_post_inputs_default(void) {
  hush_post_inputs in{};
  in.split = 0.5f;
  in.split2 = 0.5f;
  in.exposure = 1.0f;
  in.line = 1.5f;
  return in;
}

extern "C" int hush_post_create(const hush_post_desc *desc, hush_post_t **out) {
  if (!out) return post_fail(nullptr, HUSH_ERR_ARG, "hush_post_create: out is NULL");
  *out = nullptr;
  const hush_post_desc d = desc ? *desc : hush_post_desc_default();
  if (d.format < HUSH_POST_RGBA8 || d.format > HUSH_POST_RGBA32F)
    return post_fail(nullptr, HUSH_ERR_ARG, "Post: unknown target format " + std::to_string(d.format));
  hush_post_t *p = new hush_post_t();
  p->dev = d.device;
  p->d = d;
  *out = p;
  return HUSH_OK;
}

extern "C" void hush_post_destroy(hush_post_t *p) {
  if (!p) return;
  if (p->pool) {
    cudaSetDevice(p->dev);
    cudaFree(p->pool);
  }
  delete p;
}

// Post.resize (post.js:158-169): the HDR target and the six levels of max(1, size >> i).
static int post_resize(hush_post_t *p, int W, int H) {
  if (W == p->W && H == p->H && p->pool) return HUSH_OK;
  cudaSetDevice(p->dev);
  if (p->pool) cudaFree(p->pool);
  p->pool = nullptr;
  p->W = p->H = 0;
  size_t off[LEVELS + 1], total = (size_t)W * H * 8;
  for (int i = 0; i < LEVELS; i++) {
    p->lw[i] = std::max(1, W >> (i + 1));
    p->lh[i] = std::max(1, H >> (i + 1));
    total = (total + 255) & ~(size_t)255;
    off[i] = total;
    total += (size_t)p->lw[i] * p->lh[i] * 8;
  }
  cudaError_t e = cudaMalloc(&p->pool, total);
  if (e != cudaSuccess) {
    p->pool = nullptr;
    return post_fail(p, HUSH_ERR_CUDA, std::string("Post.resize: cudaMalloc: ") + cudaGetErrorString(e));
  }
  p->hdr = reinterpret_cast<uint2 *>(p->pool);
  for (int i = 0; i < LEVELS; i++) p->lev[i] = reinterpret_cast<uint2 *>(p->pool + off[i]);
  p->W = W;
  p->H = H;
  return HUSH_OK;
}

// Post.encode (post.js:191-210).
extern "C" int hush_post_encode(hush_post_t *p, const hush_post_inputs *in, void *target, int target_width,
                                int target_height, size_t target_pitch, void *stream) {
  if (!p || !in) return post_fail(p, HUSH_ERR_ARG, "Post.encode: NULL argument");
  if (!in->left || !in->right) return post_fail(p, HUSH_ERR_ARG, "Post.encode: missing left or right image");
  if (!target) return post_fail(p, HUSH_ERR_ARG, "Post.encode: missing target");
  if (in->width <= 0 || in->height <= 0 || target_width <= 0 || target_height <= 0)
    return post_fail(p, HUSH_ERR_ARG, "Post.encode: bad size");
  const size_t px = p->d.format == HUSH_POST_RGBA32F ? 16 : 4;
  if ((uintptr_t)in->left % 8 || (uintptr_t)in->right % 8 || (uintptr_t)in->mid % 8)
    return post_fail(p, HUSH_ERR_ARG, "Post.encode: input images must be 8-byte aligned (rgba16float texels)");
  if ((uintptr_t)target % px)
    return post_fail(p, HUSH_ERR_ARG, "Post.encode: target must be " + std::to_string(px) + "-byte aligned");
  const size_t pitch = target_pitch ? target_pitch : (size_t)target_width * px;
  if (pitch < (size_t)target_width * px || pitch % px != 0)
    return post_fail(p, HUSH_ERR_ARG, "Post.encode: target pitch " + std::to_string(pitch) + " is too small or misaligned");
  if (int rc = post_resize(p, in->width, in->height)) return rc;
  cudaSetDevice(p->dev);
  cudaStream_t st = (cudaStream_t)stream;
  const int W = in->width, H = in->height;
  const uint2 *L = (const uint2 *)in->left, *R = (const uint2 *)in->right;
  const uint2 *M = in->mid ? (const uint2 *)in->mid : R;
  const dim3 blk(BX, BY);
  k_post_composite<<<grid_for(W, H), blk, 0, st>>>(L, R, M, W, H, in->split, in->split2, in->exposure, in->same,
                                                   p->hdr);
  k_post_down<true><<<grid_for(p->lw[0], p->lh[0]), blk, 0, st>>>(p->hdr, W, H, p->lev[0], p->lw[0], p->lh[0]);
  for (int i = 1; i < LEVELS; i++)
    k_post_down<false><<<grid_for(p->lw[i], p->lh[i]), blk, 0, st>>>(p->lev[i - 1], p->lw[i - 1], p->lh[i - 1],
                                                                     p->lev[i], p->lw[i], p->lh[i]);
  for (int i = LEVELS - 1; i > 0; i--)
    k_post_up<<<grid_for(p->lw[i - 1], p->lh[i - 1]), blk, 0, st>>>(p->lev[i], p->lw[i], p->lh[i], p->lev[i - 1],
                                                                    p->lw[i - 1], p->lh[i - 1]);
  FinalArgs fa{in->split, in->split2, in->line, p->d.bloom, p->d.vignette, p->d.format};
  const bool exact2 = target_width == W && target_height == H && W == 2 * p->lw[0] && H == 2 * p->lh[0];
  if (exact2)
    k_post_final<true><<<grid_for(W, H), blk, 0, st>>>(p->hdr, W, H, p->lev[0], p->lw[0], p->lh[0], target, W, H,
                                                       pitch, fa);
  else
    k_post_final<false><<<grid_for(target_width, target_height), blk, 0, st>>>(
        p->hdr, W, H, p->lev[0], p->lw[0], p->lh[0], target, target_width, target_height, pitch, fa);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HUSH_OK : post_fail(p, HUSH_ERR_CUDA, std::string("Post.encode: ") + cudaGetErrorString(e));
}

extern "C" int hush_post_set(hush_post_t *p, float bloom, float vignette) {
  if (!p) return post_fail(nullptr, HUSH_ERR_ARG, "hush_post_set: NULL post");
  p->d.bloom = bloom;
  p->d.vignette = vignette;
  return HUSH_OK;
}

// level 0: the composited HDR image; 1..6: the bloom levels (after the upsample chain of the last encode).
extern "C" const void *hush_post_buffer(const hush_post_t *p, int level, int *width, int *height) {
  if (!p || !p->pool || level < 0 || level > LEVELS) return nullptr;
  if (level == 0) {
    if (width) *width = p->W;
    if (height) *height = p->H;
    return p->hdr;
  }
  if (width) *width = p->lw[level - 1];
  if (height) *height = p->lh[level - 1];
  return p->lev[level - 1];
}

extern "C" const char *hush_post_last_error(const hush_post_t *p) { return p ? p->last_error.c_str() : g_post_err.c_str(); }
