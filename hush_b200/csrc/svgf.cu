// SVGF baseline (Schied et al. 2017) + TAA resolve: the reference's SVGF class (src/denoise/svgf.js) as CUDA
// kernels over rgba16float device buffers. Kept beside Hush as its fallback and as the judge of its error.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "common.cuh"
#include "hush.h"
#include "hush_device.cuh"

using namespace hush;

namespace {

struct SvgfFrame {
  int W, H;
  int reset, use_taa;
  float sigma_l, sigma_n, sigma_z, alpha_color, alpha_moments, taa_alpha;
  const uint2 *rad, *nd, *mv, *mat, *emi, *pnd, *pmv;
  int p_rad, p_nd, p_mv, p_mat, p_emi, p_pnd, p_pmv;
  const uint2 *hist_prev, *mom_prev, *taa_prev;
  uint2 *tmp, *mom, *hist, *taa;
};

HD_INL bool svgf_consistent(const SvgfFrame &f, int qx, int qy, float4 n, float zPrev, float obj) {  // svgf.js:31-39
  if (qx < 0 || qy < 0 || qx >= f.W || qy >= f.H) return false;
  const float4 nd = ldh(f.pnd, qy * f.p_pnd + qx);
  if (nd.w < 0.0f) return false;
  if (ldh(f.pmv, qy * f.p_pmv + qx).z != obj) return false;
  if (fabsf(nd.w - zPrev) > 0.05f * zPrev + 0.01f) return false;
  if (dot3(nd, n) < 0.9f) return false;
  return true;
}

// TEMPORAL (svgf.js:41-105)
__global__ void k_svgf_temporal(const SvgfFrame f) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= f.W || y >= f.H) return;
  const int o = y * f.W + x;
  const float4 nd = ldh(f.nd, y * f.p_nd + x);
  if (nd.w < 0.0f) {
    sth(f.tmp, o, make_float4(0.f, 0.f, 0.f, 0.f));
    sth(f.mom, o, make_float4(0.f, 0.f, 0.f, 0.f));
    return;
  }
  const float4 mv = ldh(f.mv, y * f.p_mv + x);
  const float4 alb = ldh(f.mat, y * f.p_mat + x);
  const float4 r = ldh(f.rad, y * f.p_rad + x);
  const float ix = r.x / fmaxf(alb.x, 1e-3f), iy = r.y / fmaxf(alb.y, 1e-3f), iz = r.z / fmaxf(alb.z, 1e-3f);
  const float l = __fadd_rn(__fadd_rn(__fmul_rn(ix, 0.2126f), __fmul_rn(iy, 0.7152f)), __fmul_rn(iz, 0.0722f));
  const float ppx = (float)x + 0.5f + mv.x - 0.5f, ppy = (float)y + 0.5f + mv.y - 0.5f;
  const float flx = floorf(ppx), fly = floorf(ppy);
  const int bx = (int)flx, by = (int)fly;
  const float fx = ppx - flx, fy = ppy - fly;
  // the history length it blends into decides the spatial / temporal variance branch (m.z >= 4), so the weighted
  // sums are rounded product by product like an unfused shader (no FMA contraction)
  float sumW = 0.f, hcx = 0.f, hcy = 0.f, hcz = 0.f, hm0 = 0.f, hm1 = 0.f, hm2 = 0.f;
  const float wts[4] = {__fmul_rn(1.0f - fx, 1.0f - fy), __fmul_rn(fx, 1.0f - fy), __fmul_rn(1.0f - fx, fy),
                        __fmul_rn(fx, fy)};
  const bool noHistory = f.reset != 0;
  if (!noHistory) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int qx = bx + (i & 1), qy = by + (i >> 1);
      if (svgf_consistent(f, qx, qy, nd, mv.w, mv.z) && wts[i] > 0.0f) {
        const float4 c = ldh(f.hist_prev, qy * f.W + qx), m = ldh(f.mom_prev, qy * f.W + qx);
        sumW += wts[i];
        hcx = __fadd_rn(hcx, __fmul_rn(wts[i], c.x)); hcy = __fadd_rn(hcy, __fmul_rn(wts[i], c.y));
        hcz = __fadd_rn(hcz, __fmul_rn(wts[i], c.z));
        hm0 = __fadd_rn(hm0, __fmul_rn(wts[i], m.x)); hm1 = __fadd_rn(hm1, __fmul_rn(wts[i], m.y));
        hm2 = __fadd_rn(hm2, __fmul_rn(wts[i], m.z));
      }
    }
  }
  if (sumW < 0.01f && !noHistory) {
    const int cx = (int)rintf(ppx), cy = (int)rintf(ppy);  // WGSL round(): ties to even
    for (int dy = -1; dy <= 1; dy++) {
      for (int dx = -1; dx <= 1; dx++) {
        const int qx = cx + dx, qy = cy + dy;
        if (svgf_consistent(f, qx, qy, nd, mv.w, mv.z)) {
          const float4 c = ldh(f.hist_prev, qy * f.W + qx), m = ldh(f.mom_prev, qy * f.W + qx);
          sumW += 1.0f;
          hcx += c.x; hcy += c.y; hcz += c.z;
          hm0 += m.x; hm1 += m.y; hm2 += m.z;
        }
      }
    }
  }
  float len, cx = ix, cy = iy, cz = iz, m0 = l, m1 = __fmul_rn(l, l);
  if (sumW >= 0.01f) {
    hcx /= sumW; hcy /= sumW; hcz /= sumW;
    hm0 /= sumW; hm1 /= sumW; hm2 /= sumW;
    len = fminf(hm2 + 1.0f, 64.0f);
    const float ac = fmaxf(f.alpha_color, 1.0f / len), am = fmaxf(f.alpha_moments, 1.0f / len);
    cx = __fadd_rn(__fmul_rn(hcx, 1.0f - ac), __fmul_rn(ix, ac));
    cy = __fadd_rn(__fmul_rn(hcy, 1.0f - ac), __fmul_rn(iy, ac));
    cz = __fadd_rn(__fmul_rn(hcz, 1.0f - ac), __fmul_rn(iz, ac));
    m0 = __fadd_rn(__fmul_rn(hm0, 1.0f - am), __fmul_rn(m0, am));
    m1 = __fadd_rn(__fmul_rn(hm1, 1.0f - am), __fmul_rn(m1, am));
  } else {
    len = 1.0f;
  }
  sth(f.tmp, o, make_float4(cx, cy, cz, 0.f));
  sth(f.mom, o, make_float4(m0, m1, len, 0.f));
}

// VARIANCE (svgf.js:114-148)
__global__ void k_svgf_variance(const SvgfFrame f, uint2 *out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= f.W || y >= f.H) return;
  const int o = y * f.W + x;
  const float4 nd = ldh(f.nd, y * f.p_nd + x);
  if (nd.w < 0.0f) { sth(out, o, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  const float4 c = ldh(f.tmp, o), m = ldh(f.mom, o);
  if (m.z >= 4.0f) {
    sth(out, o, make_float4(c.x, c.y, c.z, fmaxf(0.0f, m.y - m.x * m.x)));
    return;
  }
  float sw = 0.f, scx = 0.f, scy = 0.f, scz = 0.f, sm0 = 0.f, sm1 = 0.f;
  for (int dy = -3; dy <= 3; dy++) {
    for (int dx = -3; dx <= 3; dx++) {
      const int qx = x + dx, qy = y + dy;
      if (qx < 0 || qy < 0 || qx >= f.W || qy >= f.H) continue;
      const float4 ndq = ldh(f.nd, qy * f.p_nd + qx);
      if (ndq.w < 0.0f) continue;
      const float dist = sqrtf((float)dx * (float)dx + (float)dy * (float)dy);
      const float wz = expf(-fabsf(ndq.w - nd.w) / (0.02f * nd.w * dist + 1e-3f));
      const float wn = powf(fmaxf(0.0f, dot3(ndq, nd)), f.sigma_n);
      const float w = wz * wn;
      const float4 cq = ldh(f.tmp, qy * f.W + qx), mq = ldh(f.mom, qy * f.W + qx);
      sw += w;
      scx += w * cq.x; scy += w * cq.y; scz += w * cq.z;
      sm0 += w * mq.x; sm1 += w * mq.y;
    }
  }
  const float d = fmaxf(sw, 1e-6f);
  scx /= d; scy /= d; scz /= d; sm0 /= d; sm1 /= d;
  const float v = fmaxf(0.0f, sm1 - sm0 * sm0) * 4.0f / fmaxf(m.z, 1.0f);
  sth(out, o, make_float4(scx, scy, scz, v));
}

// The normal weight pow(max(n . n_q, 0), sigma_n): by seven squarings for the default sigma_n = 128 (no special-function
// unit), else as the hardware exp2(sigma_n log2 x); pow(x, 0) = 1.
HD_INL float svgf_wn(float x, float sigma_n) {
  if (sigma_n == 128.0f) {
#pragma unroll
    for (int i = 0; i < 7; i++) x *= x;
    return x;
  }
  return sigma_n != 0.0f ? __powf(x, sigma_n) : 1.0f;
}

// ATROUS iteration (svgf.js:157-216); iteration 0 also writes the colour history.
__global__ void k_svgf_atrous(const SvgfFrame f, const uint2 *in, uint2 *out, int iter, int step) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= f.W || y >= f.H) return;
  const int o = y * f.W + x;
  const float4 nd = ldh(f.nd, y * f.p_nd + x);
  if (nd.w < 0.0f) {
    sth(out, o, make_float4(0.f, 0.f, 0.f, 0.f));
    if (iter == 0) sth(f.hist, o, make_float4(0.f, 0.f, 0.f, 0.f));
    return;
  }
  const float4 center = ldh(in, o);
  const float k3[3] = {0.25f, 0.5f, 0.25f};
  float gv = 0.f;
#pragma unroll
  for (int dy = -1; dy <= 1; dy++)
#pragma unroll
    for (int dx = -1; dx <= 1; dx++)
      gv += k3[dx + 1] * k3[dy + 1] * ldh(in, clampi(y + dy, 0, f.H - 1) * f.W + clampi(x + dx, 0, f.W - 1)).w;
  const float lp = lum(center);
  const float denomL = f.sigma_l * sqrtf(fmaxf(gv, 0.0f)) + 1e-6f;
  const float z = nd.w;
  const float zl = ldh(f.nd, y * f.p_nd + clampi(x - 1, 0, f.W - 1)).w;
  const float zr = ldh(f.nd, y * f.p_nd + clampi(x + 1, 0, f.W - 1)).w;
  const float zu = ldh(f.nd, clampi(y - 1, 0, f.H - 1) * f.p_nd + x).w;
  const float zd = ldh(f.nd, clampi(y + 1, 0, f.H - 1) * f.p_nd + x).w;
  const float gx = fminf(zr > 0.0f ? fabsf(zr - z) : 1e9f, zl > 0.0f ? fabsf(zl - z) : 1e9f);
  const float gy = fminf(zd > 0.0f ? fabsf(zd - z) : 1e9f, zu > 0.0f ? fabsf(zu - z) : 1e9f);
  const float zg = fminf(fmaxf(gx, gy), z);
  const float h[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
  // the tap distances sqrt(dx^2 + dy^2) (correctly rounded: 1, sqrt 2, 2, sqrt 5, sqrt 8) and one reciprocal per
  // distance class and for the luminance scale instead of a division per tap; the weights' exp and pow run as the
  // hardware approximations, which WGSL's own accuracy rules allow (exp: 3 + 2|x| ULP; pow via exp2(y log2 x)). The
  // temporal pass, whose history-length test flips on an ulp, keeps IEEE arithmetic.
  const float dcls[5] = {1.0f, 1.41421356237f, 2.0f, 2.2360679775f, 2.82842712475f};
  float izd[5];
#pragma unroll
  for (int c = 0; c < 5; c++) izd[c] = 1.0f / (f.sigma_z * zg * (dcls[c] * (float)step) + 1e-3f);
  const float ilum = 1.0f / denomL;
  float sw = h[2] * h[2];
  float scx = center.x * sw, scy = center.y * sw, scz = center.z * sw;
  float sv = center.w * sw * sw;
#pragma unroll
  for (int dy = -2; dy <= 2; dy++) {
#pragma unroll
    for (int dx = -2; dx <= 2; dx++) {
      if (dx == 0 && dy == 0) continue;
      const int qx = x + dx * step, qy = y + dy * step;
      if (qx < 0 || qy < 0 || qx >= f.W || qy >= f.H) continue;
      const float4 ndq = ldh(f.nd, qy * f.p_nd + qx);
      if (ndq.w < 0.0f) continue;
      const float4 cq = ldh(in, qy * f.W + qx);
      const int d2 = dx * dx + dy * dy;  // 1, 2, 4, 5, 8
      const int cls = d2 == 1 ? 0 : (d2 == 2 ? 1 : (d2 == 4 ? 2 : (d2 == 5 ? 3 : 4)));
      const float wz = fabsf(ndq.w - nd.w) * izd[cls];
      const float wn = svgf_wn(fmaxf(0.0f, dot3(ndq, nd)), f.sigma_n);
      const float wl = fabsf(lum(cq) - lp) * ilum;
      const float w = h[dx + 2] * h[dy + 2] * wn * __expf(-wz - wl);
      sw += w;
      scx += w * cq.x; scy += w * cq.y; scz += w * cq.z;
      sv += w * w * cq.w;
    }
  }
  const float4 r = make_float4(scx / sw, scy / sw, scz / sw, sv / (sw * sw));
  sth(out, o, r);
  if (iter == 0) sth(f.hist, o, make_float4(r.x, r.y, r.z, 0.f));
}

// The same iteration for steps 1, 2 and 4 with the 5 x 5 footprint staged in shared memory: a 16 x 16 tile with an
// apron of 2 step texels (clamped to the image, as the centre's 3 x 3 variance blur and depth gradient read them),
// each texel converted once and its luminance formed once. The arithmetic per tap is the kernel's above.
template <int STEP>
__global__ void __launch_bounds__(256) k_svgf_atrous_tile(const SvgfFrame f, const uint2 *in, uint2 *out, int iter) {
  constexpr int TS = 16, A = 2 * STEP, T = TS + 2 * A;
  __shared__ float4 sC[T * T], sN[T * T];
  __shared__ float sL[T * T];
  const int li = threadIdx.y * TS + threadIdx.x;
  const int bx = blockIdx.x * TS, by = blockIdx.y * TS;
  for (int i = li; i < T * T; i += TS * TS) {
    const int gx = clampi(bx - A + i % T, 0, f.W - 1), gy = clampi(by - A + i / T, 0, f.H - 1);
    const float4 c = ldh(in, gy * f.W + gx);
    sC[i] = c;
    sN[i] = ldh(f.nd, gy * f.p_nd + gx);
    sL[i] = lum(c);
  }
  __syncthreads();
  const int x = bx + threadIdx.x, y = by + threadIdx.y;
  if (x >= f.W || y >= f.H) return;
  const int o = y * f.W + x;
  const int lx = threadIdx.x + A, ly = threadIdx.y + A, tc = ly * T + lx;
  const float4 nd = sN[tc];
  if (nd.w < 0.0f) {
    sth(out, o, make_float4(0.f, 0.f, 0.f, 0.f));
    if (iter == 0) sth(f.hist, o, make_float4(0.f, 0.f, 0.f, 0.f));
    return;
  }
  const float4 center = sC[tc];
  const float k3[3] = {0.25f, 0.5f, 0.25f};
  float gv = 0.f;
#pragma unroll
  for (int dy = -1; dy <= 1; dy++)
#pragma unroll
    for (int dx = -1; dx <= 1; dx++) gv += k3[dx + 1] * k3[dy + 1] * sC[tc + dy * T + dx].w;
  const float lp = sL[tc];
  const float denomL = f.sigma_l * sqrtf(fmaxf(gv, 0.0f)) + 1e-6f;
  const float z = nd.w;
  const float zl = sN[tc - 1].w, zr = sN[tc + 1].w, zu = sN[tc - T].w, zd = sN[tc + T].w;
  const float gx = fminf(zr > 0.0f ? fabsf(zr - z) : 1e9f, zl > 0.0f ? fabsf(zl - z) : 1e9f);
  const float gy = fminf(zd > 0.0f ? fabsf(zd - z) : 1e9f, zu > 0.0f ? fabsf(zu - z) : 1e9f);
  const float zg = fminf(fmaxf(gx, gy), z);
  const float h[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
  const float dcls[5] = {1.0f, 1.41421356237f, 2.0f, 2.2360679775f, 2.82842712475f};
  float izd[5];
#pragma unroll
  for (int c = 0; c < 5; c++) izd[c] = 1.0f / (f.sigma_z * zg * (dcls[c] * (float)STEP) + 1e-3f);
  const float ilum = 1.0f / denomL;
  float sw = h[2] * h[2];
  float scx = center.x * sw, scy = center.y * sw, scz = center.z * sw;
  float sv = center.w * sw * sw;
#pragma unroll
  for (int dy = -2; dy <= 2; dy++) {
#pragma unroll
    for (int dx = -2; dx <= 2; dx++) {
      if (dx == 0 && dy == 0) continue;
      const int qx = x + dx * STEP, qy = y + dy * STEP;
      if (qx < 0 || qy < 0 || qx >= f.W || qy >= f.H) continue;
      const int t = tc + dy * STEP * T + dx * STEP;
      const float4 ndq = sN[t];
      if (ndq.w < 0.0f) continue;
      const float4 cq = sC[t];
      const int d2 = dx * dx + dy * dy;
      const int cls = d2 == 1 ? 0 : (d2 == 2 ? 1 : (d2 == 4 ? 2 : (d2 == 5 ? 3 : 4)));
      const float wz = fabsf(ndq.w - nd.w) * izd[cls];
      const float wn = svgf_wn(fmaxf(0.0f, dot3(ndq, nd)), f.sigma_n);
      const float wl = fabsf(sL[t] - lp) * ilum;
      const float w = h[dx + 2] * h[dy + 2] * wn * __expf(-wz - wl);
      sw += w;
      scx += w * cq.x; scy += w * cq.y; scz += w * cq.z;
      sv += w * w * cq.w;
    }
  }
  const float4 r = make_float4(scx / sw, scy / sw, scz / sw, sv / (sw * sw));
  sth(out, o, r);
  if (iter == 0) sth(f.hist, o, make_float4(r.x, r.y, r.z, 0.f));
}

// RESOLVE (svgf.js:241-270). The reference samples the history through a hardware bilinear sampler
// (clamp-to-edge); here the same texel footprint is weighted exactly in f32.
HD_INL float3 svgf_remod(const SvgfFrame &f, const uint2 *il, int qx, int qy) {
  const int cx = clampi(qx, 0, f.W - 1), cy = clampi(qy, 0, f.H - 1);
  const float4 a = ldh(il, cy * f.W + cx), m = ldh(f.mat, cy * f.p_mat + cx), e = ldh(f.emi, cy * f.p_emi + cx);
  return make_float3(a.x * m.x + e.x, a.y * m.y + e.y, a.z * m.z + e.z);
}

__global__ void k_svgf_resolve(const SvgfFrame f, const uint2 *il) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= f.W || y >= f.H) return;
  const int o = y * f.W + x;
  const float3 cur = tmap(svgf_remod(f, il, x, y));
  if (!f.use_taa) {
    const float3 r = itmap(cur);
    sth(f.taa, o, make_float4(r.x, r.y, r.z, 1.0f));
    return;
  }
  // E[c^2] - E[c]^2 cancels catastrophically when the neighbourhood is flat: its products are rounded separately
  // (no FMA contraction), as an unfused f32 shader computes them
  float3 m1 = make_float3(0.f, 0.f, 0.f), m2 = m1;
  for (int dy = -1; dy <= 1; dy++)
    for (int dx = -1; dx <= 1; dx++) {
      const float3 c = to_ycocg(tmap(svgf_remod(f, il, x + dx, y + dy)));
      m1.x += c.x; m1.y += c.y; m1.z += c.z;
      m2.x = __fadd_rn(m2.x, __fmul_rn(c.x, c.x));
      m2.y = __fadd_rn(m2.y, __fmul_rn(c.y, c.y));
      m2.z = __fadd_rn(m2.z, __fmul_rn(c.z, c.z));
    }
  m1.x /= 9.0f; m1.y /= 9.0f; m1.z /= 9.0f;
  m2.x /= 9.0f; m2.y /= 9.0f; m2.z /= 9.0f;
  const float sdx = sqrtf(fmaxf(__fsub_rn(m2.x, __fmul_rn(m1.x, m1.x)), 0.0f)),
              sdy = sqrtf(fmaxf(__fsub_rn(m2.y, __fmul_rn(m1.y, m1.y)), 0.0f)),
              sdz = sqrtf(fmaxf(__fsub_rn(m2.z, __fmul_rn(m1.z, m1.z)), 0.0f));
  const float4 mv = ldh(f.mv, y * f.p_mv + x);
  const float uvx = ((float)x + 0.5f + mv.x) / (float)f.W, uvy = ((float)y + 0.5f + mv.y) / (float)f.H;
  const float a = f.taa_alpha;
  float3 res = cur;
  if (uvx >= 0.0f && uvy >= 0.0f && uvx <= 1.0f && uvy <= 1.0f && !f.reset) {
    const float ppx = uvx * (float)f.W - 0.5f, ppy = uvy * (float)f.H - 0.5f;
    const float bxf = floorf(ppx), byf = floorf(ppy);
    const float fx = ppx - bxf, fy = ppy - byf;
    float3 hist = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int ox = j & 1, oy = j >> 1;
      const float wb = (ox == 1 ? fx : 1.0f - fx) * (oy == 1 ? fy : 1.0f - fy);
      const float4 t = ldh(f.taa_prev, clampi((int)byf + oy, 0, f.H - 1) * f.W + clampi((int)bxf + ox, 0, f.W - 1));
      hist.x += wb * t.x; hist.y += wb * t.y; hist.z += wb * t.z;
    }
    float3 hh = to_ycocg(tmap(hist));
    hh.x = fminf(fmaxf(hh.x, m1.x - 1.25f * sdx), m1.x + 1.25f * sdx);
    hh.y = fminf(fmaxf(hh.y, m1.y - 1.25f * sdy), m1.y + 1.25f * sdy);
    hh.z = fminf(fmaxf(hh.z, m1.z - 1.25f * sdz), m1.z + 1.25f * sdz);
    const float3 h = from_ycocg(hh);
    res = make_float3(h.x * (1.0f - a) + cur.x * a, h.y * (1.0f - a) + cur.y * a, h.z * (1.0f - a) + cur.z * a);
  }
  const float3 r = itmap(res);
  sth(f.taa, o, make_float4(r.x, r.y, r.z, 1.0f));
}

thread_local std::string g_svgf_err;

}  // namespace

struct svgf_s {
  int dev = 0, W = 0, H = 0, frame = 0;
  bool reset = true;
  svgf_options o;
  char *pool = nullptr;
  uint2 *hist[2] = {}, *mom[2] = {}, *tmp = nullptr, *atrous[2] = {}, *taa[2] = {};
  const void *last_out = nullptr;
  std::string last_error;
};

static int svgf_fail(svgf_t *s, int code, const std::string &m) {
  if (s) s->last_error = m;
  g_svgf_err = m;
  return code;
}

extern "C" svgf_options svgf_options_default(void) {
  svgf_options o;
  o.iterations = 5;
  o.sigma_l = 4.0f; o.sigma_n = 128.0f; o.sigma_z = 1.0f;
  o.alpha_color = 0.2f; o.alpha_moments = 0.2f; o.taa_alpha = 0.1f;
  o.taa = 1;
  return o;
}

static int svgf_alloc(svgf_t *s, int W, int H) {
  const size_t img = ((size_t)W * H * 8 + 255) & ~(size_t)255;
  char *p = nullptr;
  cudaError_t e = cudaMalloc(&p, img * 9);
  if (e != cudaSuccess) return svgf_fail(s, HUSH_ERR_CUDA, std::string("SVGF: cudaMalloc: ") + cudaGetErrorString(e));
  cudaMemset(p, 0, img * 9);
  if (s->pool) cudaFree(s->pool);
  s->pool = p;
  uint2 **slots[9] = {&s->hist[0], &s->hist[1], &s->mom[0], &s->mom[1], &s->tmp,
                      &s->atrous[0], &s->atrous[1], &s->taa[0], &s->taa[1]};
  for (int i = 0; i < 9; i++) *slots[i] = (uint2 *)(p + img * i);
  s->W = W; s->H = H; s->frame = 0; s->reset = true; s->last_out = nullptr;
  return HUSH_OK;
}

extern "C" int svgf_create(int width, int height, const svgf_options *opts, int device, svgf_t **out) {
  if (!out) return svgf_fail(nullptr, HUSH_ERR_ARG, "svgf_create: out is NULL");
  *out = nullptr;
  if (!(width > 0 && height > 0))
    return svgf_fail(nullptr, HUSH_ERR_ARG, "SVGF: bad size " + std::to_string(width) + "x" + std::to_string(height));
  svgf_options o = opts ? *opts : svgf_options_default();
  if (o.iterations < 1 || o.iterations > 5)
    return svgf_fail(nullptr, HUSH_ERR_ARG, "SVGF: iterations must be 1..5 (got " + std::to_string(o.iterations) + ")");
  int dev = device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return svgf_fail(nullptr, HUSH_ERR_CUDA, "SVGF: cudaGetDevice");
  if (cudaSetDevice(dev) != cudaSuccess) return svgf_fail(nullptr, HUSH_ERR_CUDA, "SVGF: cudaSetDevice");
  svgf_t *s = new svgf_t();
  s->dev = dev;
  s->o = o;
  int rc = svgf_alloc(s, width, height);
  if (rc != HUSH_OK) { delete s; return rc; }
  *out = s;
  return HUSH_OK;
}

extern "C" void svgf_destroy(svgf_t *s) {
  if (!s) return;
  cudaSetDevice(s->dev);
  if (s->pool) cudaFree(s->pool);
  delete s;
}

extern "C" int svgf_resize(svgf_t *s, int w, int h) {
  if (!s) return svgf_fail(nullptr, HUSH_ERR_ARG, "svgf_resize: NULL instance");
  if (!(w > 0 && h > 0)) return svgf_fail(s, HUSH_ERR_ARG, "SVGF: bad size " + std::to_string(w) + "x" + std::to_string(h));
  if (w == s->W && h == s->H) return HUSH_OK;
  cudaSetDevice(s->dev);
  return svgf_alloc(s, w, h);
}

extern "C" int svgf_reset(svgf_t *s) {
  if (!s) return svgf_fail(nullptr, HUSH_ERR_ARG, "svgf_reset: NULL instance");
  s->reset = true;
  return HUSH_OK;
}

static const char *SVGF_NAMES[7] = {"radiance", "normalDepth", "motion", "material", "emission", "prevNormalDepth",
                                    "prevMotion"};

extern "C" int svgf_encode(svgf_t *s, const svgf_inputs *in, void *stream, const void **out) {
  if (!s) return svgf_fail(nullptr, HUSH_ERR_ARG, "svgf_encode: NULL instance");
  if (!in) return svgf_fail(s, HUSH_ERR_ARG, "SVGF.encode: missing inputs");
  const void *p[7] = {in->radiance, in->normal_depth, in->motion, in->material, in->emission,
                      in->prev_normal_depth, in->prev_motion};
  int pt[7];
  for (int k = 0; k < 7; k++) {
    if (!p[k]) return svgf_fail(s, HUSH_ERR_ARG, std::string("SVGF.encode: missing input '") + SVGF_NAMES[k] + "'");
    if (in->pitch[k] && (in->pitch[k] % 8 || in->pitch[k] < (size_t)s->W * 8))
      return svgf_fail(s, HUSH_ERR_ARG, std::string("SVGF.encode: bad pitch for '") + SVGF_NAMES[k] + "'");
    pt[k] = in->pitch[k] ? (int)(in->pitch[k] / 8) : s->W;
  }
  cudaSetDevice(s->dev);
  cudaStream_t st = (cudaStream_t)stream;
  const int cur = s->frame & 1, prev = cur ^ 1;
  SvgfFrame f;
  std::memset(&f, 0, sizeof(f));
  f.W = s->W; f.H = s->H;
  f.reset = s->reset ? 1 : 0;
  f.use_taa = s->o.taa ? 1 : 0;
  f.sigma_l = s->o.sigma_l; f.sigma_n = s->o.sigma_n; f.sigma_z = s->o.sigma_z;
  f.alpha_color = s->o.alpha_color; f.alpha_moments = s->o.alpha_moments; f.taa_alpha = s->o.taa_alpha;
  f.rad = (const uint2 *)p[0]; f.nd = (const uint2 *)p[1]; f.mv = (const uint2 *)p[2]; f.mat = (const uint2 *)p[3];
  f.emi = (const uint2 *)p[4]; f.pnd = (const uint2 *)p[5]; f.pmv = (const uint2 *)p[6];
  f.p_rad = pt[0]; f.p_nd = pt[1]; f.p_mv = pt[2]; f.p_mat = pt[3]; f.p_emi = pt[4]; f.p_pnd = pt[5]; f.p_pmv = pt[6];
  f.hist_prev = s->hist[prev]; f.mom_prev = s->mom[prev]; f.taa_prev = s->taa[prev];
  f.tmp = s->tmp; f.mom = s->mom[cur]; f.hist = s->hist[cur]; f.taa = s->taa[cur];
  const dim3 blk(8, 8), grd((s->W + 7) / 8, (s->H + 7) / 8);  // workgroup 8 x 8 (svgf.js:41)
  k_svgf_temporal<<<grd, blk, 0, st>>>(f);
  k_svgf_variance<<<grd, blk, 0, st>>>(f, s->atrous[0]);
  int src = 0;
  const dim3 tblk(16, 16), tgrd((s->W + 15) / 16, (s->H + 15) / 16);
  for (int i = 0; i < s->o.iterations; i++) {
    const uint2 *a = s->atrous[src];
    uint2 *b = s->atrous[src ^ 1];
    if (i == 0) k_svgf_atrous_tile<1><<<tgrd, tblk, 0, st>>>(f, a, b, i);
    else if (i == 1) k_svgf_atrous_tile<2><<<tgrd, tblk, 0, st>>>(f, a, b, i);
    else if (i == 2) k_svgf_atrous_tile<4><<<tgrd, tblk, 0, st>>>(f, a, b, i);
    else k_svgf_atrous<<<grd, blk, 0, st>>>(f, a, b, i, 1 << i);
    src ^= 1;
  }
  k_svgf_resolve<<<grd, blk, 0, st>>>(f, s->atrous[src]);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return svgf_fail(s, HUSH_ERR_CUDA, std::string("SVGF: kernel launch: ") + cudaGetErrorString(e));
  s->reset = false;
  s->frame++;
  s->last_out = s->taa[cur];
  if (out) *out = s->last_out;
  return HUSH_OK;
}

// The reference's getter returns taa[frame & 1] after frame++, i.e. the previous frame's image (svgf.js:327, 376);
// this returns the image encode() produced last.
extern "C" const void *svgf_output(const svgf_t *s) { return s ? s->last_out : nullptr; }
extern "C" const char *svgf_last_error(const svgf_t *s) { return s ? s->last_error.c_str() : g_svgf_err.c_str(); }
