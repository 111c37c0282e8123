// The fused B200 frame. Same arithmetic as the per-pass kernels (hush_passes.cu); different kernel boundaries:
//
//   stage 0  temporal   TEMPORAL + block features + the MLP heads (hush.js:79-308, 312-365) in one kernel: the 2x2
//                       blocks align with the tile, so the 20 features never leave the SM (the reference writes
//                       F0/F1 and reads them back in INFER). Writes A0, mom, key, par0..2 and the half-res block
//                       means Ah (= F2.zw) and guide Gh (= F3.xy).
//   stage 1  mid1|c1    mid1 (INFER's a-trous, hush.js:366) and COARSE1 (hush.js:404-421) in one launch
//   stage 2  mid2|c2    mid2 (hush.js:753) and coarse2 (hush.js:752) in one launch
//   stage 3  mid3       hush.js:754
//   stage 4  fine+final hush.js:560-621
//   stage 5  taa        hush.js:639-677
//
// Levels with a neighbourhood (the a-trous levels, TAA) stay separate launches: fusing them needs recomputed halos,
// and on B200 these passes are bound by instruction issue rather than HBM, so recomputation costs more than the
// L2-resident round trip of a half-res image.
#include <cuda.h>  // CUtensorMap and its enums (types only: the encoder is fetched from the driver)
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cstring>
#include <type_traits>

#include "hush_device.cuh"
#include "hush_pair.cuh"
#include "hush_internal.h"
#include "umma.cuh"

namespace hush {

// ------------------------------------------------------------------------------------------------ loaders
HD_INL float4 gh_decode(float4 g) {  // (oct normal, depth, count) -> (normal, depth)
  float4 n = oct_dec(g.x, g.y);
  n.w = g.z;
  return n;
}

// ------------------------------------------------------------------------------------------------ stage 0
// TEMPORAL pixel() (hush.js:111-223), block() (hush.js:226-282) and INFER's MLP with its heads (hush.js:312-365) in
// one kernel, one thread per 2x2 block (k_temporal_block below).
constexpr uint32_t MBAR_POLLS = 1u << 22;
// L of a tile entry outside the image or on sky (a valid luminance is finite and far above it)
constexpr float L_INVALID = -1e30f;
HD_INL bool l_valid(float L) { return L > -1e29f; }

// Eight values as one 16-byte operand row segment (hi), and the rounding residuals v - hi rounded again (lo): a
// split-precision operand, hi + lo carrying 16 (bf16) or 22 (f16) significant bits of v. Two values per conversion
// (cvt.rn.bf16x2.f32 / cvt.rn.f16x2.f32) and per residual subtraction (FP32x2).
HD_INL uint32_t cvt2(float a, float b, std::true_type) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}
HD_INL uint32_t cvt2(float a, float b, std::false_type) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}
HD_INL float2 back2(uint32_t u, std::true_type) {
  return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
}
HD_INL float2 back2(uint32_t u, std::false_type) {
  return __half22float2(*reinterpret_cast<const __half2 *>(&u));
}
template <bool BF16>
HD_INL void pack8_split(const float *v, uint4 &hi, uint4 &lo) {
  using T = std::integral_constant<bool, BF16>;
  uint32_t h[4], l[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    h[k] = cvt2(v[2 * k], v[2 * k + 1], T{});
    const float2 r = __fadd2_rn(make_float2(v[2 * k], v[2 * k + 1]), [&] {
      const float2 b = back2(h[k], T{});
      return make_float2(-b.x, -b.y);
    }());
    l[k] = cvt2(r.x, r.y, T{});
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// pixel()'s inputs to block(): P0..P4 as block() reads them and the decoded normal (Ns.w = 1 with a surface).
struct PixOut {
  float4 P0, P1, P2, P3, P4, Ns;
};
HD_INL PixOut pix_none() {
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  return PixOut{z4, z4, make_float4(0.f, 0.f, -1.0f, 0.f), z4, z4, z4};
}

// The loads of one pixel's pixel(): its G-buffer texels and the reprojection gathers of the previous frame's key,
// colour and moments (bilinear footprint) and par0, as temporal_pixel_fast() reads them.
struct PixLoads {
  uint2 nd, mv, mat, k4[4], c4[4], m4[4], pq;
};

// A pixel's loads are issued as cp.async copies into a shared-memory slot (no registers held while they fly): slot
// entry k of this thread at g[k * stride]: 0 normalDepth, 1 material, 2 previous par0, 3-6 key, 7-10 colour history,
// 11-14 moments of the bilinear footprint. The caller commits the group.
HD_INL void cp_async8(const uint2 *dst_smem, const uint2 *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(umma::smem_u32(dst_smem)), "l"(src) : "memory");
}
HD_INL void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
HD_INL void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
template <int STRIDE>
HD_INL void pixel_issue_async(const HushFrame &f, int px, int py, uint2 mvr, uint2 *g) {
  const int W = f.W, H = f.H;
  cp_async8(g, f.nd + py * f.p_nd + px);
  cp_async8(g + STRIDE, f.mat + py * f.p_mat + px);
  if (f.reset) return;
  const float4 mv = h4_to_f4(mvr);
  const float ppx = (float)px + mv.x, ppy = (float)py + mv.y;
  const int bix = __float2int_rz(floorf(ppx)), biy = __float2int_rz(floorf(ppy));
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int q = clampi(biy + (i >> 1), 0, H - 1) * W + clampi(bix + (i & 1), 0, W - 1);
    cp_async8(g + (3 + i) * STRIDE, f.key_prev + q);
    cp_async8(g + (7 + i) * STRIDE, f.hist_prev + q);
    cp_async8(g + (11 + i) * STRIDE, f.mom_prev + q);
  }
  const int cx = __float2int_rz(floorf(ppx + 0.5f)), cy = __float2int_rz(floorf(ppy + 0.5f));
  cp_async8(g + 2 * STRIDE, f.par0_prev + (clampi(cy, 0, H - 1) >> 1) * f.W2 + (clampi(cx, 0, W - 1) >> 1));
}
template <int STRIDE>
HD_INL PixLoads pixel_fetch(const uint2 *g, uint2 mvr, bool reset) {
  PixLoads L;
  L.nd = g[0];
  L.mat = g[STRIDE];
  L.mv = mvr;
  if (!reset) {
    L.pq = g[2 * STRIDE];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      L.k4[i] = g[(3 + i) * STRIDE];
      L.c4[i] = g[(7 + i) * STRIDE];
      L.m4[i] = g[(11 + i) * STRIDE];
    }
  }
  return L;
}

// pixel() of hush.js:111-223 over the (r, g, b, L) tile from the preloaded texels; same arithmetic as
// temporal_pixel(). Writes A0, mom, key and returns the pixel's inputs to block().
template <class Tile>
HD_INL PixOut temporal_pixel_fast(const HushFrame &f, int px, int py, const Tile &T, const PixLoads &PL) {
  const int W = f.W, H = f.H;
  const float4 nd = h4_to_f4(PL.nd), mv = h4_to_f4(PL.mv);
  const int oi = py * W + px;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  if (nd.w < 0.0f) {
    f.A0[oi] = make_uint2(0, 0);
    f.mom[oi] = make_uint2(0, 0);
    sth(f.key, oi, make_float4(0.f, 0.f, -1.0f, mv.z));
    return pix_none();
  }
  float fx = 0.f, fy = 0.f;
  int bix = 0, biy = 0, cx = 0, cy = 0;
  if (!f.reset) {
    const float ppx = (float)px + mv.x, ppy = (float)py + mv.y;
    const float bx = floorf(ppx), by = floorf(ppy);
    fx = ppx - bx;
    fy = ppy - by;
    bix = __float2int_rz(bx);
    biy = __float2int_rz(by);
    cx = __float2int_rz(floorf(ppx + 0.5f));
    cy = __float2int_rz(floorf(ppy + 0.5f));
  }
  const uint2 *k4 = PL.k4, *c4 = PL.c4, *m4 = PL.m4;
  const uint2 pqr = PL.pq, mrr = PL.mat;
  // 3x3 statistics of the illumination (valid neighbours), two passes
  const float4 illum = T(0, 0);
  const float l = illum.w;
  // (r, g) as one packed FP32x2 lane pair, b and (in the second pass) L as the other: the same arithmetic per lane
  float2 s1xy = f2(0.f, 0.f);
  float s1z = 0.f, cnt = 0.f;
#pragma unroll
  for (int j = 0; j < 9; j++) {
    const float4 c = T(j % 3 - 1, j / 3 - 1);
    s1xy = add2(s1xy, lo2(c));  // invalid entries hold rgb = 0
    s1z += c.z;
    cnt += l_valid(c.w) ? 1.0f : 0.0f;
  }
  cnt = fmaxf(cnt, 1.0f);
  const float mux = s1xy.x / cnt, muy = s1xy.y / cnt, muz = s1z / cnt;
  const float slm = lum3(mux, muy, muz);
  const float2 nmu_xy = f2(-mux, -muy), nmu_zl = f2(-muz, -slm);
  float2 svxy = f2(0.f, 0.f), svzl = f2(0.f, 0.f);
#pragma unroll
  for (int j = 0; j < 9; j++) {
    const float4 c = T(j % 3 - 1, j / 3 - 1);
    if (l_valid(c.w)) {
      const float2 dxy = add2(lo2(c), nmu_xy), dzl = add2(hi2(c), nmu_zl);
      svxy = fma2(dxy, dxy, svxy);
      svzl = fma2(dzl, dzl, svzl);
    }
  }
  const float sdx = sqrtf(fmaxf(svxy.x / cnt, 1e-12f)), sdy = sqrtf(fmaxf(svxy.y / cnt, 1e-12f)),
              sdz = sqrtf(fmaxf(svzl.x / cnt, 1e-12f));
  float svar = svzl.y / cnt;
  bool has = false;
  float hcx = 0.f, hcy = 0.f, hcz = 0.f;
  float4 hm = z4;
  float v = 0.f, alpha = 1.0f, gamma = 1.0f;
  if (!f.reset) {
    float sumW = 0.f;
    const float wts[4] = {(1.0f - fx) * (1.0f - fy), fx * (1.0f - fy), (1.0f - fx) * fy, fx * fy};
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int qx = bix + (i & 1), qy = biy + (i >> 1);
      if (wts[i] > 0.0f && qx >= 0 && qy >= 0 && qx < W && qy < H && check_key(h4_to_f4(k4[i]), nd, mv.w, mv.z)) {
        const float4 c = h4_to_f4(c4[i]), m = h4_to_f4(m4[i]);
        const float2 w2 = bc2(wts[i]);
        sumW += wts[i];
        const float2 hxy = fma2(w2, lo2(c), f2(hcx, hcy));
        hcx = hxy.x; hcy = hxy.y;
        hcz += wts[i] * c.z;
        const float2 mxy = fma2(w2, lo2(m), f2(hm.x, hm.y)), mzw = fma2(w2, hi2(m), f2(hm.z, hm.w));
        hm = make_float4(mxy.x, mxy.y, mzw.x, mzw.y);
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
      hm = z4;
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
    const float4 pq = h4_to_f4(pqr);
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
  const float ox = qf16(oc.x), oy = qf16(oc.y);
  PixOut o;
  o.P0 = make_float4(E * lum(Aq), E * qf16(l), fmaxf(m2 - m1 * m1, 0.0f), len1);
  o.P1 = make_float4(qf16(v), qf16(lag), E * qf16(nfast), m1);
  o.P2 = make_float4(ox, oy, qf16(nd.w), qf16(sqrtf(mv.x * mv.x + mv.y * mv.y)));
  o.P3 = h4_to_f4(mrr);
  o.P4 = Aq;
  o.Ns = oct_dec(ox, oy);  // block() decodes the stored oct normal (hush.js:238)
  o.Ns.w = 1.0f;
  return o;
}

HD_INL float4 scale4(float4 v, float k) { return make_float4(v.x * k, v.y * k, v.z * k, v.w * k); }

HD_INL float4 ffma4(float s, float4 w, float4 a) {  // a + s * w as two packed FP32x2 FMAs
  const float2 lo = __ffma2_rn(make_float2(s, s), make_float2(w.x, w.y), make_float2(a.x, a.y));
  const float2 hi = __ffma2_rn(make_float2(s, s), make_float2(w.z, w.w), make_float2(a.z, a.w));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}

// ------------------------------------------------------------------------------------------------ k_temporal_block
// One thread per 2x2 block: tile 64 x 16 pixels = 32 x 8 blocks, 256 threads. Each thread runs pixel() for its four
// pixels in block order, accumulates block()'s sums in registers in the WGSL's order (hush.js:226-282), forms the 20
// features once and runs the whole FP32 MLP (weights in the constant bank, a kernel parameter: each FMA takes its
// weight as a broadcast operand), so after the tile barrier no thread waits for another. The tile is stored
// column-parity-split (even and odd columns in separate rows of 33 entries): neighbouring threads, two pixel columns
// apart, then read consecutive 16-byte entries. The per-pixel loads (G-buffer texels and the dependent reprojection
// gathers) go by cp.async into two shared-memory slots per thread, one pixel ahead: pixel q + 2's gathers are in
// flight while pixel q + 1 computes, without holding registers. The tensor-core
// forms instead write each block's features as one operand row and run each layer as two tcgen05 MMAs (M = 128,
// N = 16) over the CTA's 256 rows, FP32 accumulators in TMEM; bias, ReLU and the heads stay FP32.
constexpr int KB_TW = 64, KB_TH = 16, KB_NT = (KB_TW / 2) * (KB_TH / 2);
constexpr int KB_SWL = KB_TW + 2, KB_SH = KB_TH + 2, KB_HW = KB_SWL / 2;
HD_INL int kb_tix(int r, int c) { return (2 * r + (c & 1)) * KB_HW + (c >> 1); }

constexpr int KB_NTEX = 15;  // texels of one pixel's loads (pixel_issue_async)
struct KbSmem {
  float4 I[2 * KB_HW * KB_SH];   // illumination (r, g, b) and L (luminance or L_INVALID), apron 1
  float2 Lq[2 * KB_HW * KB_SH];  // (E * qf16(L), 1) for valid entries, (0, 0) otherwise
  uint2 G[2][KB_NTEX][KB_NT];    // two pixels' loads in flight per thread, thread-minor (conflict-free)
};
// Tensor-core forms: the same tile plus the MMA operands of the CTA's 256 rows (one per block) in the K-major
// no-swizzle layout, each as a split-precision pair (hi, lo): A1 256 x 32 (features, zero padded), A2 256 x 16
// (hidden layers), then the weights B1 / B2 / B3 (hi, and for bf16 lo).
// The per-pixel load slots (pixel phase) and the MMA operands (MLP phase, after a CTA barrier) share their space.
struct KbTcSmem {
  float4 I[2 * KB_HW * KB_SH];
  float2 Lq[2 * KB_HW * KB_SH];
  union {
    uint2 G[2][KB_NTEX][KB_NT];
    struct {
      alignas(128) uint8_t a1[KB_NT * 32 * 2];
      alignas(128) uint8_t a1lo[KB_NT * 32 * 2];
      alignas(128) uint8_t a2[KB_NT * 16 * 2];
      alignas(128) uint8_t a2lo[KB_NT * 16 * 2];
    };
  };
  alignas(128) uint8_t b[2 * MLP_TC_BLOB_BYTES];
  alignas(8) uint64_t mbar[2];  // one per 128-row group
  uint32_t tmem;
};

// One MMA layer over the CTA's 256 rows, as two independent 128-row groups: warps 0-3 (rows 0-127, TMEM columns
// [0, 16)) and warps 4-7 (rows 128-255, columns [16, 32)). A group waits only for its own four warps (a named barrier
// of 128 threads), then its first thread issues the group's MMAs and commits them to the group's mbarrier, so one
// group's MMAs run while the other group's warps are still forming their rows. Per K block the products A_hi B_hi,
// A_lo B_hi and (with lo weights, bf16) A_hi B_lo accumulate into the same FP32 accumulator; the dropped A_lo B_lo
// term is 2^-16 (bf16) / 2^-22 (f16) of the product. Every thread waits on its group's mbarrier (bounded) and loads
// its own row: warp w reads lanes 32 (w % 4) of column block w / 4. Returns false if the wait gave up.
HD_INL bool tc_layer_256(KbTcSmem &S, int li, const uint8_t *a, const uint8_t *alo, uint32_t kcore_a, int kblocks,
                         uint32_t b_off, bool b_lo, uint32_t kcore_b, uint32_t idesc, uint32_t phase, float *d) {
  const int g = li >> 7;
  umma::fence_proxy_async();
  umma::fence_before_sync();
  if (g == 0) asm volatile("bar.sync 1, 128;" ::: "memory");  // named barriers 1 / 2 (0 is __syncthreads)
  else asm volatile("bar.sync 2, 128;" ::: "memory");
  const uint32_t mbar = umma::smem_u32(&S.mbar[g]);
  if ((li & 127) == 0) {
    umma::fence_after_sync();
    const uint32_t b = umma::smem_u32(S.b) + b_off;
    const uint32_t ah = umma::smem_u32(a) + (uint32_t)g * 16u * 128u * kcore_a;
    const uint32_t al = umma::smem_u32(alo) + (uint32_t)g * 16u * 128u * kcore_a;
    for (int kb = 0; kb < kblocks; kb++) {
      const uint64_t bh = umma::sdesc(b + 256u * kb, 128, 128 * kcore_b);
      umma::mma_f16(S.tmem + 16u * g, umma::sdesc(ah + 256u * kb, 128, 128 * kcore_a), bh, idesc, kb > 0 ? 1u : 0u);
      umma::mma_f16(S.tmem + 16u * g, umma::sdesc(al + 256u * kb, 128, 128 * kcore_a), bh, idesc, 1u);
      if (b_lo)
        umma::mma_f16(S.tmem + 16u * g, umma::sdesc(ah + 256u * kb, 128, 128 * kcore_a),
                      umma::sdesc(b + MLP_TC_BLOB_BYTES + 256u * kb, 128, 128 * kcore_b), idesc, 1u);
    }
    umma::commit(mbar);
  }
  const bool ok = umma::mbar_wait_bounded(mbar, phase, MBAR_POLLS);
  umma::fence_after_sync();
  const int w = li >> 5;
  umma::ld16(S.tmem + ((uint32_t)(32 * (w & 3)) << 16) + 16u * (uint32_t)(w >> 2), d);
  return ok;
}

struct ParityTile {
  const float4 *I;
  int r, c;  // tile row / column of the pixel
  HD_INL float4 operator()(int dx, int dy) const { return I[kb_tix(r + dy, c + dx)]; }
};

// MODE 0: FP32 MLP per thread; 1 / 2: tensor-core MLP on split bf16 / f16 operands (dynamic shared memory);
// 3: the reference's f16-arithmetic MLP per thread (the `f16` option).
template <int MODE>
__global__ void __launch_bounds__(KB_NT, 2)
    k_temporal_block(const __grid_constant__ HushFrame f, const __grid_constant__ MlpConst wp,
                     const uint4 *__restrict__ blob) {
  constexpr bool TC = MODE == 1 || MODE == 2;
  using Smem = std::conditional_t<TC, KbTcSmem, KbSmem>;
  extern __shared__ __align__(128) unsigned char kb_smem[];
  Smem &S = *reinterpret_cast<Smem *>(kb_smem);
  const int li = threadIdx.x;
  const float E = f.exposure;
  if constexpr (TC) {
    if (li < 32) {
      umma::tmem_alloc(umma::smem_u32(&S.tmem), 32);
      umma::tmem_relinquish();
    }
    if (li == 0) {
      umma::mbar_init(umma::smem_u32(&S.mbar[0]), 1);
      umma::mbar_init(umma::smem_u32(&S.mbar[1]), 1);
    }
    constexpr int NB = (MODE == 1 ? 2 : 1) * MLP_TC_BLOB_BYTES / 16;  // bf16: hi and lo weights
    for (int i = li; i < NB; i += KB_NT) reinterpret_cast<uint4 *>(S.b)[i] = __ldg(blob + i);
    umma::fence_proxy_async();
    umma::fence_before_sync();
  }
  const int lbx = li % (KB_TW / 2), lby = li / (KB_TW / 2);
  const int px0 = blockIdx.x * KB_TW + 2 * lbx, py0 = blockIdx.y * KB_TH + 2 * lby;
  // phase 1: the four pixels' motion first (each pixel's reprojection gathers then wait for one load round trip, not
  // two), then the first pixels' loads and gathers in flight with the tile loads
  uint2 mvq[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int px = px0 + (q & 1), py = py0 + (q >> 1);
    mvq[q] = (px < f.W && py < f.H) ? __ldg(f.mv + py * f.p_mv + px) : make_uint2(0, 0);
  }
  PixLoads PL;
  const int ox = blockIdx.x * KB_TW - 1, oy = blockIdx.y * KB_TH - 1;
  constexpr int N = KB_SWL * KB_SH;
#pragma unroll 1
  for (int i0 = 0; i0 < N; i0 += 2 * KB_NT) {
    uint2 tn[2], tr[2], tm[2];
    bool tin[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int i = i0 + u * KB_NT + li;
      const int qx = ox + i % KB_SWL, qy = oy + i / KB_SWL;
      tin[u] = i < N && qx >= 0 && qy >= 0 && qx < f.W && qy < f.H;
      const int cx = clampi(qx, 0, f.W - 1), cy = clampi(qy, 0, f.H - 1);
      tn[u] = __ldg(f.nd + cy * f.p_nd + cx);
      tr[u] = __ldg(f.rad + cy * f.p_rad + cx);
      tm[u] = __ldg(f.mat + cy * f.p_mat + cx);
    }
    if (i0 == 0) {  // the first two pixels' loads (cp.async into their slots), behind the first tile loads
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int px = px0 + (q & 1), py = py0 + (q >> 1);
        if (px < f.W && py < f.H) pixel_issue_async<KB_NT>(f, px, py, mvq[q], &S.G[q][0][li]);
        cp_async_commit();
      }
    }
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int i = i0 + u * KB_NT + li;
      if (i >= N) continue;
      float4 e = make_float4(0.f, 0.f, 0.f, L_INVALID);
      float2 lq = make_float2(0.f, 0.f);
      if (tin[u] && h4_to_f4(tn[u]).w >= 0.0f) {
        const float4 r = h4_to_f4(tr[u]), m = h4_to_f4(tm[u]);
        e.x = r.x / fmaxf(m.x, 1e-3f);
        e.y = r.y / fmaxf(m.y, 1e-3f);
        e.z = r.z / fmaxf(m.z, 1e-3f);
        e.w = lum3(e.x, e.y, e.z);
        lq = make_float2(E * qf16(e.w), 1.0f);
      }
      const int t = kb_tix(i / KB_SWL, i % KB_SWL);
      S.I[t] = e;
      S.Lq[t] = lq;
    }
  }
  __syncthreads();
  if constexpr (TC) umma::fence_after_sync();
  // phase 2: pixel() of the four pixels (block order: top-left, top-right, bottom-left, bottom-right), block() sums
  float nv = 0.f, Nx = 0.f, Ny = 0.f, Nz = 0.f, MV = 0.f, Z = 0.f;
  float4 S0 = make_float4(0.f, 0.f, 0.f, 0.f), S1 = S0, S3 = S0, AC = S0;
  float la[4], zs[4], nx4[4], ny4[4], nz4[4];
  bool okp[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int px = px0 + (q & 1), py = py0 + (q >> 1);
    const bool pin = px < f.W && py < f.H;
    if (q < 3) cp_async_wait<1>();  // this pixel's group has landed (the next pixel's may still fly)
    else cp_async_wait<0>();
    if (pin) PL = pixel_fetch<KB_NT>(&S.G[q & 1][0][li], mvq[q], f.reset);
    const PixOut p = pin ? temporal_pixel_fast(f, px, py, ParityTile{S.I, 2 * lby + (q >> 1) + 1, 2 * lbx + (q & 1) + 1}, PL)
                         : pix_none();
    if (q < 2) {  // pixel q + 2 into the slot pixel q has finished reading
      const int qx = px0 + (q & 1), qy = py0 + 1;
      if (qx < f.W && qy < f.H) pixel_issue_async<KB_NT>(f, qx, qy, mvq[q + 2], &S.G[q & 1][0][li]);
      cp_async_commit();
    }
    okp[q] = p.Ns.w != 0.0f;
    la[q] = p.P0.x;
    zs[q] = p.P2.z;
    nx4[q] = p.Ns.x; ny4[q] = p.Ns.y; nz4[q] = p.Ns.z;
    if (okp[q]) {
      nv += 1.0f;
      S0.x += p.P0.x; S0.y += p.P0.y; S0.z += p.P0.z; S0.w += p.P0.w;
      S1.x += p.P1.x; S1.y += p.P1.y; S1.z += p.P1.z; S1.w += p.P1.w;
      Nx += p.Ns.x; Ny += p.Ns.y; Nz += p.Ns.z;
      S3.x += p.P3.x; S3.y += p.P3.y; S3.z += p.P3.z; S3.w += p.P3.w;
      AC.x += p.P4.x; AC.y += p.P4.y; AC.z += p.P4.z; AC.w += p.P4.w;
      MV += p.P2.w;
      Z += p.P2.z;
    }
  }
  // phase 3: block() (hush.js:226-282)
  const int X = blockIdx.x * (KB_TW / 2) + lbx, Y = blockIdx.y * (KB_TH / 2) + lby;
  const bool valid = X < f.W2 && Y < f.H2;
  const bool ok = nv != 0.0f;
  float fe[N_FEAT];
  float4 G = make_float4(0.f, 0.f, -1.0f, 0.f);
  {
    const float k = ok ? 1.0f / nv : 0.0f;
    S0 = scale4(S0, k); S1 = scale4(S1, k); S3 = scale4(S3, k); AC = scale4(AC, k);
    Nx *= k; Ny *= k; Nz *= k;
    MV *= k;
    Z *= k;
    const float Lacc = S0.x;
    float VA = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (okp[q]) VA += (la[q] - Lacc) * (la[q] - Lacc);
    VA *= k;
    // 4x4 neighbourhood (block +-1) of the quantised luminance, row-major
    float s1 = 0.f, n4 = 0.f;
    float2 w16[16];
#pragma unroll
    for (int e = 0; e < 16; e++) {
      w16[e] = S.Lq[kb_tix(2 * lby + (e >> 2), 2 * lbx + (e & 3))];
      s1 += w16[e].y * w16[e].x;
      n4 += w16[e].y;
    }
    const float mu4 = s1 / fmaxf(n4, 1.0f);
    float var4 = 0.f;
#pragma unroll
    for (int e = 0; e < 16; e++) {
      const float d = w16[e].x - mu4;
      var4 += w16[e].y * d * d;
    }
    var4 /= fmaxf(n4, 1.0f);
    const float nl = fmaxf(sqrtf(Nx * Nx + Ny * Ny + Nz * Nz), 1e-6f);
    const float nnx = Nx / nl, nny = Ny / nl, nnz = Nz / nl;
    float zmax = -1e30f, zmin = 1e30f, mind = 1e30f;
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (okp[q]) {
        zmax = fmaxf(zmax, zs[q]);
        zmin = fminf(zmin, zs[q]);
        mind = fminf(mind, nx4[q] * nnx + ny4[q] * nny + nz4[q] * nnz);
      }
    const float dz = fminf(fmaxf((zmax - zmin) / fmaxf(zmin, 1e-6f), 0.0f), 1.0f);
    const float dn = fminf(fmaxf(1.0f - mind, 0.0f), 2.0f);
    const float2 oc = oct_enc(nnx, nny, nnz);
    fe[0] = log1p_w(Lacc); fe[1] = log1p_w(S0.y); fe[2] = log1p_w(S0.z); fe[3] = log1p_w(var4);
    fe[4] = S0.w / HMAX; fe[5] = S1.x; fe[6] = log1p_w(S1.y);
    fe[7] = log1p_w(fabsf(S1.z - S1.w) / (S1.w + 1e-3f));
    fe[8] = oc.x; fe[9] = oc.y; fe[10] = dz; fe[11] = dn;
    fe[12] = S3.x; fe[13] = S3.y; fe[14] = S3.z; fe[15] = S3.w;
    fe[16] = 1.0f - nv / 4.0f; fe[17] = log1p_w(MV); fe[18] = log1p_w(mu4); fe[19] = log1p_w(VA);
    if (ok) G = make_float4(oc.x, oc.y, Z, nv);
  }
  const int o = Y * f.W2 + X;
  if (valid) {
    // block means and guide: F2.zw and F3.xy of hush.js:280-281 (hush.js:241-244 without valid pixels)
    f.Ah[o] = ok ? make_uint2(pk(AC.x, AC.y), pk(AC.z, AC.w)) : make_uint2(0, 0);
    f.Gh[o] = ok ? make_uint2(pk(G.x, G.y), pk(G.z, G.w)) : make_uint2(pk(0.f, 0.f), pk(-1.0f, 0.f));
    // the decoded guide every half-res consumer forms from F3 (octDec of the stored oct normal, stored depth)
    float4 gd = oct_dec(ok ? quant1(qf16(G.x)) : 0.f, ok ? quant1(qf16(G.y)) : 0.f);
    gd.w = ok ? quant1(qf16(G.z)) : -1.0f;
    f.Gd[o] = gd;
  }
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  if constexpr (TC) {
    __syncthreads();  // every thread is done with its load slots, which the operand rows overwrite
    // phase 4 (tensor cores): every thread writes its block's operand row (zeros for blocks outside the image or
    // without valid pixels) and takes part in all three layers
    constexpr bool BF16 = MODE == 1;
    constexpr int B1 = 16 * N_FEAT, B2 = B1 + 16 + 16 * 16, B3 = B2 + 16 + N_OUT * 16;
    const float *wb = reinterpret_cast<const float *>(wp.w);  // the decoded weights (their biases)
    constexpr uint32_t ID = umma::idesc_f16(BF16 ? 1 : 0, 128, 16);
    auto put_row = [&](uint8_t *hi, uint8_t *lo, int k0, int kcore, const float *v) {
      uint4 h, l;
      pack8_split<BF16>(v, h, l);
      *reinterpret_cast<uint4 *>(hi + umma::kmajor_off(li, k0, kcore)) = h;
      *reinterpret_cast<uint4 *>(lo + umma::kmajor_off(li, k0, kcore)) = l;
    };
#pragma unroll
    for (int c = 0; c < 4; c++) {
      float v8[8];
#pragma unroll
      for (int e = 0; e < 8; e++)
        v8[e] = (8 * c + e < N_FEAT && valid && ok) ? __half2float(__ushort_as_half(f2h(qf16(fe[8 * c + e])))) : 0.f;
      put_row(S.a1, S.a1lo, 8 * c, 4, v8);
    }
    float row[16], d[16];
    bool good = tc_layer_256(S, li, S.a1, S.a1lo, 4, 2, 0, BF16, 4, ID, 0, d);
#pragma unroll
    for (int j = 0; j < 16; j++) row[j] = fmaxf(d[j] + wb[B1 + j], 0.0f);
    put_row(S.a2, S.a2lo, 0, 2, row);
    put_row(S.a2, S.a2lo, 8, 2, row + 8);
    good &= tc_layer_256(S, li, S.a2, S.a2lo, 2, 1, 1024, BF16, 2, ID, 1, d);
#pragma unroll
    for (int j = 0; j < 16; j++) row[j] = fmaxf(d[j] + wb[B2 + j], 0.0f);
    put_row(S.a2, S.a2lo, 0, 2, row);
    put_row(S.a2, S.a2lo, 8, 2, row + 8);
    good &= tc_layer_256(S, li, S.a2, S.a2lo, 2, 1, 1536, BF16, 2, ID, 0, d);
    float out[N_OUT];
#pragma unroll
    for (int j = 0; j < N_OUT; j++) out[j] = d[j] + wb[B3 + j];
    umma::fence_before_sync();
    __syncthreads();
    if (li < 32) {
      umma::fence_after_sync();
      umma::tmem_dealloc(S.tmem, 32);
    }
    if (!good) {
      atomicOr(f.err, 1u);
      return;
    }
    if (!valid) return;
    if (!ok) {
      sth(f.par0, o, z4); sth(f.par1, o, z4); sth(f.par2, o, z4);
      return;
    }
    float4 p0, p1, p2;
    mlp_heads(out, p0, p1, p2);
    sth(f.par0, o, p0);
    sth(f.par1, o, p1);
    sth(f.par2, o, p2);
    return;
  }
  if (!valid) return;
  if (!ok) {  // INFER on a block without valid pixels writes zeros (hush.js:343-346)
    sth(f.par0, o, z4); sth(f.par1, o, z4); sth(f.par2, o, z4);
    return;
  }
  if constexpr (MODE == 3) {
    // phase 4 (the `f16` option, hush.js:683-703): f16 products and running sums per unit in the WGSL's order (bias,
    // then the inputs in increasing index), two units per f16x2 instruction, weights as f16x2 unit pairs in the
    // constant bank; the features enter as stored (packed f16, hush.js:278-280)
    const uint32_t *Wh = reinterpret_cast<const uint32_t *>(wp.w);
    uint32_t a[8], b[8];
#pragma unroll
    for (int p = 0; p < 8; p++) a[p] = Wh[MLP_HALF_B1 + p];
#pragma unroll
    for (int i = 0; i < N_FEAT; i++) {
      const uint32_t x = hdup(f2h(qf16(fe[i])));
#pragma unroll
      for (int p = 0; p < 8; p++) a[p] = hadd2_rn(a[p], hmul2_rn(x, Wh[MLP_HALF_W1 + i * 8 + p]));
    }
#pragma unroll
    for (int p = 0; p < 8; p++) { a[p] = hrelu2(a[p]); b[p] = Wh[MLP_HALF_B2 + p]; }
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const uint32_t x = hdup((i & 1) ? a[i >> 1] >> 16 : a[i >> 1]);
#pragma unroll
      for (int p = 0; p < 8; p++) b[p] = hadd2_rn(b[p], hmul2_rn(x, Wh[MLP_HALF_W2 + i * 8 + p]));
    }
#pragma unroll
    for (int p = 0; p < 8; p++) b[p] = hrelu2(b[p]);
#pragma unroll
    for (int p = 0; p < 6; p++) a[p] = Wh[MLP_HALF_B3 + p];
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const uint32_t x = hdup((i & 1) ? b[i >> 1] >> 16 : b[i >> 1]);
#pragma unroll
      for (int p = 0; p < 6; p++) a[p] = hadd2_rn(a[p], hmul2_rn(x, Wh[MLP_HALF_W3 + i * 6 + p]));
    }
    float out[N_OUT];
#pragma unroll
    for (int p = 0; p < 6; p++) { out[2 * p] = hlo(a[p]); out[2 * p + 1] = hhi(a[p]); }
    float4 p0, p1, p2;
    mlp_heads(out, p0, p1, p2);
    sth(f.par0, o, p0);
    sth(f.par1, o, p1);
    sth(f.par2, o, p2);
    return;
  }
  // phase 4: the MLP (hush.js:681-704) on the features as stored (packed f16, hush.js:278-280, 348-353); each unit
  // is its bias plus the inputs in increasing index, FP32 with packed FP32x2 FMAs
#pragma unroll
  for (int i = 0; i < N_FEAT; i++) fe[i] = __half2float(__ushort_as_half(f2h(qf16(fe[i]))));
  const float4 *Wt;
  if constexpr (!TC) Wt = wp.w;
  float4 a[4];
#pragma unroll
  for (int q = 0; q < 4; q++) a[q] = Wt[MLP_FP32_B1 + q];
#pragma unroll
  for (int i = 0; i < N_FEAT; i++)
#pragma unroll
    for (int q = 0; q < 4; q++) a[q] = ffma4(fe[i], Wt[MLP_FP32_W1 + i * 4 + q], a[q]);
  float h[16];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    h[4 * q] = fmaxf(a[q].x, 0.f); h[4 * q + 1] = fmaxf(a[q].y, 0.f);
    h[4 * q + 2] = fmaxf(a[q].z, 0.f); h[4 * q + 3] = fmaxf(a[q].w, 0.f);
  }
#pragma unroll
  for (int q = 0; q < 4; q++) a[q] = Wt[MLP_FP32_B2 + q];
#pragma unroll
  for (int i = 0; i < 16; i++)
#pragma unroll
    for (int q = 0; q < 4; q++) a[q] = ffma4(h[i], Wt[MLP_FP32_W2 + i * 4 + q], a[q]);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    h[4 * q] = fmaxf(a[q].x, 0.f); h[4 * q + 1] = fmaxf(a[q].y, 0.f);
    h[4 * q + 2] = fmaxf(a[q].z, 0.f); h[4 * q + 3] = fmaxf(a[q].w, 0.f);
  }
#pragma unroll
  for (int q = 0; q < 4; q++) a[q] = Wt[MLP_FP32_B3 + q];  // (output q, 4 + q, 8 + q, 0)
#pragma unroll
  for (int i = 0; i < 16; i++)
#pragma unroll
    for (int q = 0; q < 4; q++) a[q] = ffma4(h[i], Wt[MLP_FP32_W3 + i * 4 + q], a[q]);
  float out[N_OUT];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    out[q] = a[q].x;
    out[4 + q] = a[q].y;
    out[8 + q] = a[q].z;
  }
  float4 p0, p1, p2;
  mlp_heads(out, p0, p1, p2);
  sth(f.par0, o, p0);
  sth(f.par1, o, p1);
  sth(f.par2, o, p2);
}

// ------------------------------------------------------------------------------------------------ half / quarter
// 16 x 8 tiles like the reference. One launch runs two kinds of tiles: blockIdx.x < nA runs kind A, the rest kind B.
constexpr int HT_W = 16, HT_H = 8;

// mid1 (hush.js:326, 366): 3x3 step 1 with prefilter on the block means, learned s_1 / c_1 (stored par1.y / par2.y
// are the qf16 values INFER passes).
// TMA staging of a mid level's halo tile (interior tiles): the guide Gd (float4 per texel, a 3-d FLOAT32 map
// {4, W2, H2}) lands in sG as is, the level (8-byte texels, a 2-d UINT64 map {W2, H2}) in a staging array that is
// widened to float4 afterwards. Both copies start at x = bx - STEP, even for STEP = 2 / 4, so the 8-byte map's
// innermost coordinate is 16-byte aligned; the boxes are (16 + 2 STEP) x (8 + 2 STEP) texels.
struct HalfMaps {
  CUtensorMap gd2, gd4, bh0, bh1;  // Gd with the step-2 / step-4 box; Bh0 (mid2's source) and Bh1 (mid3's)
  CUtensorMap gd1, ah;             // mid1: Gd with an 18 x 10 box at x = bx - 1; Ah with a 20 x 10 box at x = bx - 2
  CUtensorMap cgd, c1;             // coarse2 (quarter resolution): CGd and C1 with 24 x 16 boxes at x = bx - 4
  int ok;                          // 0: every tile loads with plain loads (odd W2, or no encoder)
  int qok;                         // the same for the quarter-resolution maps (odd W4)
};
constexpr uint32_t TMA_POLLS = 1u << 22;
// Waits (bounded) for a halo tile's TMA copies. On giving up it sets bit 3 of the error word and returns false: the
// caller then fills its tile with the plain clamped loads, so the output stays defined. Interior tiles need no
// clamping, so a copy that still lands later writes the very values those loads wrote.
HD_INL bool tma_wait_or_flag(const HushFrame &f, uint32_t mb) {
  if (umma::mbar_wait_bounded(mb, 0, TMA_POLLS)) return true;
  atomicOr(f.err, 8u);
  return false;
}
// FINE_FINAL's A0 / key tiles (8-byte texels, 2-d UINT64 maps {W, H}) on interior tiles: the copies start at
// x = bx - 2 (even, so 16-byte aligned) with a 36 x 10 box; the tile's column c is the box's column c + 1.
struct FineMaps {
  CUtensorMap a0, key;
  int ok;
};

HD_INL void tma_expect(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
HD_INL void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}
HD_INL void tma_load_3d(uint32_t dst, const CUtensorMap *map, int c, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

// mid1 (hush.js:326, 366): the block means Ah and the guide, apron 1. On interior tiles the guide lands in sG by TMA
// (3-d map, no alignment rule on x) and Ah in a staging array from x = bx - 2 (the 8-byte map's x must be even), the
// tile's column c being the staged column c + 1.
HD_INL void tile_mid1(const HushFrame &f, int tileX, int tileY, float4 *sA, float4 *sG, const HalfMaps *M) {
  constexpr int AP = 1, SW = HT_W + 2, SH = HT_H + 2, BW = HT_W + 4;
  __shared__ alignas(128) uint2 stage[BW * SH];
  __shared__ alignas(8) uint64_t mbar;
  const int li = threadIdx.x;
  const int bx = tileX * HT_W, by = tileY * HT_H;
  const bool interior = bx - 2 >= 0 && by - 1 >= 0 && bx + HT_W + 2 <= f.W2 && by + HT_H + 1 <= f.H2;
  const bool inner = M && interior;
  const int X = bx + li % HT_W, Y = by + li / HT_W;
  const bool in_img = X < f.W2 && Y < f.H2;
  const int o = Y * f.W2 + X;
  // this pixel's parameters, in flight while the tile arrives
  uint2 p1 = make_uint2(0, 0), p2 = make_uint2(0, 0);
  if (in_img) { p1 = __ldg(f.par1 + o); p2 = __ldg(f.par2 + o); }
  bool staged = false;
  if (inner) {
    const uint32_t mb = umma::smem_u32(&mbar);
    if (li == 0) umma::mbar_init(mb, 1);
    __syncthreads();
    if (li == 0) {
      tma_expect(mb, BW * SH * 8 + SW * SH * 16);
      tma_load_2d(umma::smem_u32(stage), &M->ah, bx - 2, by - 1, mb);
      tma_load_3d(umma::smem_u32(sG), &M->gd1, 0, bx - 1, by - 1, mb);
    }
    staged = tma_wait_or_flag(f, mb);
    if (staged)
      for (int i = li; i < SW * SH; i += HT_W * HT_H) sA[i] = h4_to_f4(stage[(i / SW) * BW + i % SW + 1]);
  }
  if (!staged) {
    for (int i = li; i < SW * SH; i += HT_W * HT_H) {
      const int q = clampi(by - AP + i / SW, 0, f.H2 - 1) * f.W2 + clampi(bx - AP + i % SW, 0, f.W2 - 1);
      sA[i] = ldh(f.Ah, q);
      sG[i] = __ldg(f.Gd + q);
    }
  }
  __syncthreads();
  if (!in_img) return;
  const int lx = li % HT_W + AP, ly = li / HT_W + AP;
  if (sG[ly * SW + lx].w < 0.0f) { sth(f.Bh0, o, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  const float s = h4_to_f4(p1).y, c = h4_to_f4(p2).y;
  sth(f.Bh0, o, interior ? filt_x<1, 1, true, SW, false>(sA, sG, lx, ly, X, Y, f.W2, f.H2, s, c)
                         : filt_x<1, 1, true, SW, true>(sA, sG, lx, ly, X, Y, f.W2, f.H2, s, c));
}

template <int STEP, int COMP>
HD_INL void tile_mid(const HushFrame &f, int tileX, int tileY, const uint2 *src, uint2 *dst, float4 *sA, float4 *sG,
                     const CUtensorMap *mg, const CUtensorMap *ms) {
  constexpr int AP = STEP, SW = HT_W + 2 * AP, SH = HT_H + 2 * AP;
  __shared__ alignas(128) uint2 stage[SW * SH];
  __shared__ alignas(8) uint64_t mbar;
  const int li = threadIdx.x;
  const int bx = tileX * HT_W, by = tileY * HT_H;
  const bool interior = bx - AP >= 0 && by - AP >= 0 && bx + HT_W + AP <= f.W2 && by + HT_H + AP <= f.H2;
  const bool inner = mg && interior;
  const int X = bx + li % HT_W, Y = by + li / HT_W;
  const bool in_img = X < f.W2 && Y < f.H2;
  const int o = Y * f.W2 + X;
  uint2 p1 = make_uint2(0, 0), p2 = make_uint2(0, 0);  // this pixel's parameters, in flight with the tile
  if (in_img) { p1 = __ldg(f.par1 + o); p2 = __ldg(f.par2 + o); }
  bool staged = false;
  if (inner) {
    const uint32_t mb = umma::smem_u32(&mbar);
    if (li == 0) umma::mbar_init(mb, 1);
    __syncthreads();
    if (li == 0) {
      tma_expect(mb, SW * SH * (8 + 16));
      tma_load_2d(umma::smem_u32(stage), ms, bx - AP, by - AP, mb);
      tma_load_3d(umma::smem_u32(sG), mg, 0, bx - AP, by - AP, mb);
    }
    staged = tma_wait_or_flag(f, mb);
    if (staged)
      for (int i = li; i < SW * SH; i += HT_W * HT_H) sA[i] = h4_to_f4(stage[i]);
  }
  if (!staged) {
    for (int i = li; i < SW * SH; i += HT_W * HT_H) {
      const int q = clampi(by - AP + i / SW, 0, f.H2 - 1) * f.W2 + clampi(bx - AP + i % SW, 0, f.W2 - 1);
      sA[i] = ldh(src, q);
      sG[i] = __ldg(f.Gd + q);
    }
  }
  __syncthreads();
  if (!in_img) return;
  const int lx = li % HT_W + AP, ly = li / HT_W + AP;
  if (sG[ly * SW + lx].w < 0.0f) { sth(dst, o, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  const float4 a = h4_to_f4(p1), b = h4_to_f4(p2);
  const float s = COMP == 2 ? a.z : a.w, c = COMP == 2 ? b.z : b.w;
  sth(dst, o, interior ? filt_x<1, STEP, false, SW, false>(sA, sG, lx, ly, X, Y, f.W2, f.H2, s, c)
                       : filt_x<1, STEP, false, SW, true>(sA, sG, lx, ly, X, Y, f.W2, f.H2, s, c));
}

// down() (hush.js:385-402) from the half-res planes.
HD_INL void down_h(const HushFrame &f, int Qx, int Qy, float4 &c, float4 &g) {
  float N = 0.f, vr = 0.f, z = 0.f, cx = 0.f, cy = 0.f, cz = 0.f, nx = 0.f, ny = 0.f, nz = 0.f;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int hx = Qx * 2 + (j & 1), hy = Qy * 2 + (j >> 1);
    if (hx >= f.W2 || hy >= f.H2) continue;
    const float w = ldh(f.Gh, hy * f.W2 + hx).w;  // pixel count of the block
    if (w <= 0.0f) continue;
    const float4 a = ldh(f.Ah, hy * f.W2 + hx);
    const float4 n = __ldg(f.Gd + hy * f.W2 + hx);
    N += w;
    cx += w * a.x; cy += w * a.y; cz += w * a.z;
    vr += w * a.w;
    nx += w * n.x; ny += w * n.y; nz += w * n.z;
    z += w * n.w;
  }
  if (N == 0.0f) {
    c = make_float4(0.f, 0.f, 0.f, 0.f);
    g = make_float4(0.f, 0.f, -1.0f, 0.f);
    return;
  }
  const float nl = fmaxf(sqrtf(nx * nx + ny * ny + nz * nz), 1e-6f);
  const float2 o = oct_enc(nx / nl, ny / nl, nz / nl);
  c = make_float4(qf16(cx / N), qf16(cy / N), qf16(cz / N), qf16(vr / N / N));
  g = make_float4(qf16(o.x), qf16(o.y), qf16(z / N), 0.0f);
}

HD_INL void tile_coarse1(const HushFrame &f, int tileX, int tileY, float4 *sA, float4 *sG) {
  constexpr int AP = 2, SW = HT_W + 2 * AP, SH = HT_H + 2 * AP;
  const int li = threadIdx.x;
  const int bx = tileX * HT_W, by = tileY * HT_H;
  for (int i = li; i < SW * SH; i += HT_W * HT_H) {
    const int lqx = bx - AP + i % SW, lqy = by - AP + i / SW;
    const int qx = clampi(lqx, 0, f.W4 - 1), qy = clampi(lqy, 0, f.H4 - 1);
    float4 c, g;
    down_h(f, qx, qy, c, g);
    sA[i] = c;
    sG[i] = gh_decode(g);
    if (lqx == qx && lqy == qy && lqx >= bx && lqy >= by && lqx < bx + HT_W && lqy < by + HT_H) {
      sth(f.CG, qy * f.W4 + qx, g);
      // coarse2 and FINE_FINAL read the guide back from its rgba16float texture
      f.CGd[qy * f.W4 + qx] = gh_decode(quant4(g));
    }
  }
  __syncthreads();
  const int X = bx + li % HT_W, Y = by + li / HT_W;
  if (X >= f.W4 || Y >= f.H4) return;
  const int lx = li % HT_W + AP, ly = li / HT_W + AP;
  if (sG[ly * SW + lx].w < 0.0f) { sth(f.C1, Y * f.W4 + X, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  const bool interior = bx - AP >= 0 && by - AP >= 0 && bx + HT_W + AP <= f.W4 && by + HT_H + AP <= f.H4;
  sth(f.C1, Y * f.W4 + X, interior ? filt_x<2, 1, true, SW, false>(sA, sG, lx, ly, X, Y, f.W4, f.H4, COARSE_S, 1.0f)
                                   : filt_x<2, 1, true, SW, true>(sA, sG, lx, ly, X, Y, f.W4, f.H4, COARSE_S, 1.0f));
}

// coarse2 (hush.js:482-525, kind coarse): C1 and the decoded quarter-res guide, apron 4; interior tiles by TMA as
// the mid levels (x = bx - 4 is even).
HD_INL void tile_coarse2(const HushFrame &f, int tileX, int tileY, float4 *sA, float4 *sG, const HalfMaps *M) {
  constexpr int AP = 4, SW = HT_W + 2 * AP, SH = HT_H + 2 * AP;
  __shared__ alignas(128) uint2 stage[SW * SH];
  __shared__ alignas(8) uint64_t mbar;
  const int li = threadIdx.x;
  const int bx = tileX * HT_W, by = tileY * HT_H;
  const bool inner = M && bx - AP >= 0 && by - AP >= 0 && bx + HT_W + AP <= f.W4 && by + HT_H + AP <= f.H4;
  bool staged = false;
  if (inner) {
    const uint32_t mb = umma::smem_u32(&mbar);
    if (li == 0) umma::mbar_init(mb, 1);
    __syncthreads();
    if (li == 0) {
      tma_expect(mb, SW * SH * (8 + 16));
      tma_load_2d(umma::smem_u32(stage), &M->c1, bx - AP, by - AP, mb);
      tma_load_3d(umma::smem_u32(sG), &M->cgd, 0, bx - AP, by - AP, mb);
    }
    staged = tma_wait_or_flag(f, mb);
    if (staged)
      for (int i = li; i < SW * SH; i += HT_W * HT_H) sA[i] = h4_to_f4(stage[i]);
  }
  if (!staged) {
    for (int i = li; i < SW * SH; i += HT_W * HT_H) {
      const int q = clampi(by - AP + i / SW, 0, f.H4 - 1) * f.W4 + clampi(bx - AP + i % SW, 0, f.W4 - 1);
      sA[i] = ldh(f.C1, q);
      sG[i] = __ldg(f.CGd + q);
    }
  }
  __syncthreads();
  const int X = bx + li % HT_W, Y = by + li / HT_W;
  if (X >= f.W4 || Y >= f.H4) return;
  const int lx = li % HT_W + AP, ly = li / HT_W + AP;
  if (sG[ly * SW + lx].w < 0.0f) { sth(f.C0, Y * f.W4 + X, make_float4(0.f, 0.f, 0.f, 0.f)); return; }
  const bool interior = bx - AP >= 0 && by - AP >= 0 && bx + HT_W + AP <= f.W4 && by + HT_H + AP <= f.H4;
  sth(f.C0, Y * f.W4 + X, interior ? filt_x<2, 2, true, SW, false>(sA, sG, lx, ly, X, Y, f.W4, f.H4, COARSE_S, 1.0f)
                                   : filt_x<2, 2, true, SW, true>(sA, sG, lx, ly, X, Y, f.W4, f.H4, COARSE_S, 1.0f));
}

// mid2 / mid3 (hush.js:482-525, 753-754) on 32 x 8 tiles in two-pixel lanes (filt_pair): the level and the decoded
// guide of the (32 + 2 STEP) x (8 + 2 STEP) window are loaded as texel pairs (one 16-byte load for the two 8-byte
// level texels of an even column pair when the row pitch allows it, clamped single loads at the image border), every
// load of the thread issued before the first is unpacked, and stored in the even-column pair layout.
constexpr int MP_W = 32;  // tile width of the two-pixel mid tiles (16 lanes x 8 rows)
template <int STEP>
constexpr int mid_pair_smem() {
  return 4 * ((MP_W + 2 * STEP) / 2) * (HT_H + 2 * STEP) * 16;
}
template <int STEP, int COMP>
HD_INL void tile_mid_pair(const HushFrame &f, int tileX, int tileY, const uint2 *src, uint2 *dst, float4 *smem) {
  constexpr int AP = STEP, SW = MP_W + 2 * AP, SH = HT_H + 2 * AP, EW = SW / 2, NE = EW * SH;
  constexpr int NT = HT_W * HT_H, NIT = (NE + NT - 1) / NT;
  const PairTile T{smem, smem + NE, smem + 2 * NE, smem + 3 * NE};
  const int li = threadIdx.x;
  const int bx = tileX * MP_W, by = tileY * HT_H;
  const bool interior = bx - AP >= 0 && by - AP >= 0 && bx + MP_W + AP <= f.W2 && by + HT_H + AP <= f.H2;
  const int tx = li % (MP_W / 2), ty = li / (MP_W / 2);
  const int X = bx + 2 * tx, Y = by + ty;
  const bool in0 = X < f.W2 && Y < f.H2, in1 = in0 && X + 1 < f.W2;
  const int o = Y * f.W2 + X;
  // this pair's parameters, in flight with the tile
  uint2 pa1 = make_uint2(0, 0), pa2 = pa1, pb1 = pa1, pb2 = pa1;
  if (in0) { pa1 = __ldg(f.par1 + o); pa2 = __ldg(f.par2 + o); }
  if (in1) { pb1 = __ldg(f.par1 + o + 1); pb2 = __ldg(f.par2 + o + 1); }
  const bool even_w = !(f.W2 & 1);
  uint4 lv[NIT];
  float4 qa[NIT], qb[NIT];
#pragma unroll
  for (int i = 0; i < NIT; i++) {
    const int e = li + i * NT;
    const int r = e / EW, k = e % EW;
    const int gy = clampi(by - AP + r, 0, f.H2 - 1), gx = bx - AP + 2 * k;
    const int x0 = clampi(gx, 0, f.W2 - 1), x1 = clampi(gx + 1, 0, f.W2 - 1);
    if (e < NE) {
      if (even_w && gx >= 0 && gx + 1 < f.W2) {
        lv[i] = __ldg(reinterpret_cast<const uint4 *>(src + gy * f.W2 + gx));
      } else {
        const uint2 a = __ldg(src + gy * f.W2 + x0), b = __ldg(src + gy * f.W2 + x1);
        lv[i] = make_uint4(a.x, a.y, b.x, b.y);
      }
      qa[i] = __ldg(f.Gd + gy * f.W2 + x0);
      qb[i] = __ldg(f.Gd + gy * f.W2 + x1);
    }
  }
#pragma unroll
  for (int i = 0; i < NIT; i++) {
    const int e = li + i * NT;
    if (e < NE)
      pair_put(T, e, h4_to_f4(make_uint2(lv[i].x, lv[i].y)), h4_to_f4(make_uint2(lv[i].z, lv[i].w)), qa[i], qb[i]);
  }
  __syncthreads();
  if (!in0) return;
  const float4 a0 = h4_to_f4(pa1), b0 = h4_to_f4(pa2), a1 = h4_to_f4(pb1), b1 = h4_to_f4(pb2);
  const float2 s = COMP == 2 ? f2(a0.z, a1.z) : f2(a0.w, a1.w), c = COMP == 2 ? f2(b0.z, b1.z) : f2(b0.w, b1.w);
  const int row = ty + AP, col = 2 * tx + AP;
  float4 r0, r1;
  if (interior) filt_pair<1, STEP, false, false, false, EW>(T, row, col, X, Y, f.W2, f.H2, s, c, r0, r1);
  else filt_pair<1, STEP, false, false, true, EW>(T, row, col, X, Y, f.W2, f.H2, s, c, r0, r1);
  const float4 zc = T.g1[pe<false, EW>(row, col)];  // centre depths (z, z') in .z / .w
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  if (zc.z < 0.0f) r0 = z4;  // sky centres write zeros (hush.js:505)
  if (zc.w < 0.0f) r1 = z4;
  if (in1 && even_w) {
    const uint2 u0 = f4_to_h4(r0), u1 = f4_to_h4(r1);
    *reinterpret_cast<uint4 *>(dst + o) = make_uint4(u0.x, u0.y, u1.x, u1.y);
  } else {
    sth(dst, o, r0);
    if (in1) sth(dst, o + 1, r1);
  }
}

// The half-res levels, one kind of tile per launch (PART, a HalfPart): stage 1 mid1 (HP_MID) or COARSE1 (HP_COARSE)
// tiles, stage 2 mid2 or coarse2 tiles, stage 3 mid3 tiles; block b is mid tile b (nA of them, nAx per row) or
// coarse tile b (nBx per row).
template <int STAGE, int PART>
__global__ void __launch_bounds__(HT_W *HT_H) k_half_stage(const __grid_constant__ HushFrame f, int nAx, int nA,
                                                           int nBx, const __grid_constant__ HalfMaps M) {
  constexpr int SMAX = (HT_W + 8) * (HT_H + 8);
  __shared__ alignas(128) float4 sA[SMAX];
  __shared__ alignas(128) float4 sG[SMAX];
  const int b = (int)blockIdx.x;
  if (PART == HP_MID) {
    if (b >= nA) return;
    const int tX = b % nAx, tY = b / nAx;
    if (STAGE == 1) tile_mid1(f, tX, tY, sA, sG, M.ok ? &M : nullptr);
    else if (STAGE == 2) tile_mid<2, 2>(f, tX, tY, f.Bh0, f.Bh1, sA, sG, M.ok ? &M.gd2 : nullptr, &M.bh0);
    else tile_mid<4, 3>(f, tX, tY, f.Bh1, f.Bh0, sA, sG, M.ok ? &M.gd4 : nullptr, &M.bh1);
  } else {
    const int tX = b % nBx, tY = b / nBx;
    if (STAGE == 1) tile_coarse1(f, tX, tY, sA, sG);
    else if (STAGE == 2) tile_coarse2(f, tX, tY, sA, sG, M.qok ? &M : nullptr);
  }
}

// stages 2 and 3 with the two-pixel mid tiles: 32 x 8 mid2 / mid3 tiles (HP_MID), or stage 2's coarse2 tiles (16 x 8,
// quarter resolution; HP_COARSE). Dynamic shared memory: the pair tile, or coarse2's two float4 tiles.
template <int STAGE, int PART>
__global__ void __launch_bounds__(HT_W *HT_H) k_half_pair(const __grid_constant__ HushFrame f, int nAx, int nA,
                                                          int nBx, const __grid_constant__ HalfMaps M) {
  extern __shared__ __align__(128) float4 hp_smem[];  // 128-byte aligned: coarse2 stages its guide by TMA
  const int b = (int)blockIdx.x;
  if (PART == HP_MID) {
    if (b >= nA) return;
    if (STAGE == 2) tile_mid_pair<2, 2>(f, b % nAx, b / nAx, f.Bh0, f.Bh1, hp_smem);
    else tile_mid_pair<4, 3>(f, b % nAx, b / nAx, f.Bh1, f.Bh0, hp_smem);
  } else if (STAGE == 2) {
    constexpr int SMAX = (HT_W + 8) * (HT_H + 8);
    tile_coarse2(f, b % nBx, b / nBx, hp_smem, hp_smem + SMAX, M.qok ? &M : nullptr);
  }
}

// ------------------------------------------------------------------------------------------------ stage 4 / 5
constexpr int FT_W = 32, FT_H = 8;

// FINE_FINAL with a 32 x 8 tile. Before the barrier the CTA stages, besides the A0 / guide tile of the fine filter,
// everything its pixels' recombination reads: the half-res footprint (guide Gd, block means Ah, mid level Bh0; 18 x 6
// texels, decoded once), the quarter-res footprint (guide CGd, coarse level C0; 10 x 4) and the per-block filter
// parameters (s0, c0, beta, kappa; 16 x 4). Each texel is then read from shared memory by the 16 or so taps that use
// it instead of being fetched and decoded per tap.
constexpr int FH_W = FT_W / 2 + 2, FH_H = FT_H / 2 + 2, FQ_W = FT_W / 4 + 2, FQ_H = FT_H / 4 + 2;
constexpr int FB_W = FT_W + 4, FB_H = FT_H + 2;  // the TMA box of the A0 / key tiles
__global__ void __launch_bounds__(FT_W *FT_H, 4) k_fine_final_fused(const __grid_constant__ HushFrame f,
                                                                     const __grid_constant__ FineMaps M) {
  constexpr int AP = 1, SW = FT_W + 2, SH = FT_H + 2;
  constexpr int NH = FH_W * FH_H, NQ = FQ_W * FQ_H, NP = (FT_W / 2) * (FT_H / 2);
  __shared__ float4 sA[SW * SH], sG[SW * SH];
  __shared__ float4 sHG[NH], sHA[NH], sHB[NH], sQG[NQ], sQC[NQ], sPar[NP];
  __shared__ alignas(128) uint2 stA[FB_W * FB_H];
  __shared__ alignas(128) uint2 stK[FB_W * FB_H];
  __shared__ alignas(8) uint64_t mbar;
  const int li = threadIdx.x;
  const int bx = blockIdx.x * FT_W, by = blockIdx.y * FT_H;
  const bool interior = bx - 2 >= 0 && by - 1 >= 0 && bx + FT_W + 2 <= f.W && by + FT_H + 1 <= f.H;
  const bool inner = M.ok && interior;
  const uint32_t mb = umma::smem_u32(&mbar);
  // this pixel's material and emission, in flight while the tiles arrive
  const int px = bx + li % FT_W, py = by + li / FT_W;
  const bool in_img = px < f.W && py < f.H;
  uint2 mat_r = make_uint2(0, 0), emi_r = make_uint2(0, 0);
  if (in_img) {
    mat_r = __ldg(f.mat + py * f.p_mat + px);
    emi_r = __ldg(f.emi + py * f.p_emi + px);
  }
  if (inner) {
    if (li == 0) {
      umma::mbar_init(mb, 1);
      tma_expect(mb, FB_W * FB_H * 16);
      tma_load_2d(umma::smem_u32(stA), &M.a0, bx - 2, by - 1, mb);
      tma_load_2d(umma::smem_u32(stK), &M.key, bx - 2, by - 1, mb);
    }
  }
  const int hx0 = bx / 2 - 1, hy0 = by / 2 - 1, qx0 = bx / 4 - 1, qy0 = by / 4 - 1;
  if (li < NH) {
    const int q = clampi(hy0 + li / FH_W, 0, f.H2 - 1) * f.W2 + clampi(hx0 + li % FH_W, 0, f.W2 - 1);
    sHG[li] = __ldg(f.Gd + q);
    sHA[li] = ldh(f.Ah, q);
    sHB[li] = ldh(f.Bh0, q);
  } else if (li < NH + NQ) {
    const int i = li - NH;
    const int r = clampi(qy0 + i / FQ_W, 0, f.H4 - 1) * f.W4 + clampi(qx0 + i % FQ_W, 0, f.W4 - 1);
    sQG[i] = __ldg(f.CGd + r);
    sQC[i] = ldh(f.C0, r);
  } else if (li < NH + NQ + NP) {
    const int i = li - NH - NQ;
    const int hq = clampi(by / 2 + i / (FT_W / 2), 0, f.H2 - 1) * f.W2 + clampi(bx / 2 + i % (FT_W / 2), 0, f.W2 - 1);
    const float4 p0 = ldh(f.par0, hq);
    sPar[i] = make_float4(ldh(f.par1, hq).x, ldh(f.par2, hq).x, p0.z, p0.w);  // s0, c0, beta, kappa
  }
  bool staged = false;
  if (inner) {
    __syncthreads();  // the mbarrier's initialisation, before anyone waits on it
    staged = tma_wait_or_flag(f, mb);
    if (staged)
      for (int i = li; i < SW * SH; i += FT_W * FT_H) {
        const int t = (i / SW) * FB_W + i % SW + 1;
        sA[i] = h4_to_f4(stA[t]);
        const float4 k = h4_to_f4(stK[t]);
        float4 g = oct_dec(k.x, k.y);
        g.w = k.z;
        sG[i] = g;
      }
  }
  if (!staged) {
    for (int i = li; i < SW * SH; i += FT_W * FT_H) {
      const int q = clampi(by - AP + i / SW, 0, f.H - 1) * f.W + clampi(bx - AP + i % SW, 0, f.W - 1);
      sA[i] = ldh(f.A0, q);
      const float4 k = ldh(f.key, q);
      float4 g = oct_dec(k.x, k.y);
      g.w = k.z;
      sG[i] = g;
    }
  }
  __syncthreads();
  if (!in_img) return;
  const int lx = li % FT_W + AP, ly = li / FT_W + AP;
  const float4 alb = h4_to_f4(mat_r), emi = h4_to_f4(emi_r);
  const float4 gp = sG[ly * SW + lx];
  const int o = py * f.W + px;
  if (gp.w < 0.0f) {
    sth(f.hist, o, make_float4(0.f, 0.f, 0.f, 0.f));
    sth(f.X, o, make_float4(emi.x, emi.y, emi.z, 0.f));
    return;
  }
  const float4 pr = sPar[((py - by) >> 1) * (FT_W / 2) + ((px - bx) >> 1)];
  const float4 A1 = interior ? filt_x<1, 1, true, SW, false>(sA, sG, lx, ly, px, py, f.W, f.H, pr.x, pr.y)
                             : filt_x<1, 1, true, SW, true>(sA, sG, lx, ly, px, py, f.W, f.H, pr.x, pr.y);
  sth(f.hist, o, A1);
  // recombination (hush.js:580-620) with the half-res block means (Ah) and decoded guides (Gd, CGd)
  const float fx = qf16(A1.x), fy = qf16(A1.y), fz = qf16(A1.z);
  const float z = gp.w;
  const float rzl = LOG2E / (0.05f * z + 1e-3f);
  const int hsx = (f.W + 1) / 2, hsy = (f.H + 1) / 2;
  const float hposx = ((float)px + 0.5f) / 2.0f - 0.5f, hposy = ((float)py + 0.5f) / 2.0f - 0.5f;
  const float hbx = floorf(hposx), hby = floorf(hposy);
  const int qsx = (f.W + 3) / 4, qsy = (f.H + 3) / 4;
  const float cposx = ((float)px + 0.5f) / 4.0f - 0.5f, cposy = ((float)py + 0.5f) / 4.0f - 0.5f;
  const float cbx = floorf(cposx), cby = floorf(cposy);
  // jbw() of two taps at a time: the (n.n)^8 and weight products as packed FP32x2, the accumulation in tap order
  auto jbw2 = [&](float2 wb, float4 n0, float4 n1) {
    const float2 d = make_float2(fmaxf(dot3(n0, gp), 0.0f), fmaxf(dot3(n1, gp), 0.0f));
    const float2 d2 = __fmul2_rn(d, d), d4 = __fmul2_rn(d2, d2);
    const float2 e = make_float2(ex2_approx(-fabsf(n0.w - z) * rzl), ex2_approx(-fabsf(n1.w - z) * rzl));
    return __fmul2_rn(__fmul2_rn(__fmul2_rn(wb, e), d4), d4);
  };
  auto wbx = [](float fx_, float fy_, int j) {
    return ((j & 1) == 1 ? fx_ : 1.0f - fx_) * ((j >> 1) == 1 ? fy_ : 1.0f - fy_);
  };
  float uBx = 0.f, uBy = 0.f, uBz = 0.f, uAx = 0.f, uAy = 0.f, uAz = 0.f, swh = 0.f;
  const float hfx = hposx - hbx, hfy = hposy - hby;
#pragma unroll
  for (int j = 0; j < 4; j += 2) {
    const int qy = (int)hby + (j >> 1);
    const int qx0 = (int)hbx, qx1 = qx0 + 1;
    const int t0 = (qy - hy0) * FH_W + (qx0 - hx0), t1 = t0 + 1;
    const float4 g0 = sHG[t0], g1 = sHG[t1];
    const bool iy = qy >= 0 && qy < hsy;
    const bool ok0 = iy && qx0 >= 0 && qx0 < hsx && g0.w >= 0.0f, ok1 = iy && qx1 >= 0 && qx1 < hsx && g1.w >= 0.0f;
    const float2 w = jbw2(make_float2(wbx(hfx, hfy, j), wbx(hfx, hfy, j + 1)), g0, g1);
    if (ok0) {
      const float4 a = sHA[t0], m = sHB[t0];
      swh += w.x;
      uBx += w.x * m.x; uBy += w.x * m.y; uBz += w.x * m.z;
      uAx += w.x * a.x; uAy += w.x * a.y; uAz += w.x * a.z;
    }
    if (ok1) {
      const float4 a = sHA[t1], m = sHB[t1];
      swh += w.y;
      uBx += w.y * m.x; uBy += w.y * m.y; uBz += w.y * m.z;
      uAx += w.y * a.x; uAy += w.y * a.y; uAz += w.y * a.z;
    }
  }
  float ix = fx, iy = fy, iz = fz;
  if (swh > 1e-4f) {
    ix = uBx / swh + pr.w * (fx - uAx / swh);
    iy = uBy / swh + pr.w * (fy - uAy / swh);
    iz = uBz / swh + pr.w * (fz - uAz / swh);
  }
  float uCx = 0.f, uCy = 0.f, uCz = 0.f, swq = 0.f;
  const float cfx = cposx - cbx, cfy = cposy - cby;
#pragma unroll
  for (int j = 0; j < 4; j += 2) {
    const int ry = (int)cby + (j >> 1);
    const int rx0 = (int)cbx, rx1 = rx0 + 1;
    const int t0 = (ry - qy0) * FQ_W + (rx0 - qx0), t1 = t0 + 1;
    const float4 g0 = sQG[t0], g1 = sQG[t1];
    const bool iy = ry >= 0 && ry < qsy;
    const bool ok0 = iy && rx0 >= 0 && rx0 < qsx && g0.w >= 0.0f, ok1 = iy && rx1 >= 0 && rx1 < qsx && g1.w >= 0.0f;
    const float2 w = jbw2(make_float2(wbx(cfx, cfy, j), wbx(cfx, cfy, j + 1)), g0, g1);
    if (ok0) {
      const float4 c = sQC[t0];
      swq += w.x;
      uCx += w.x * c.x; uCy += w.x * c.y; uCz += w.x * c.z;
    }
    if (ok1) {
      const float4 c = sQC[t1];
      swq += w.y;
      uCx += w.y * c.x; uCy += w.y * c.y; uCz += w.y * c.z;
    }
  }
  float upx = ix, upy = iy, upz = iz;
  if (swq > 1e-4f) { upx = uCx / swq; upy = uCy / swq; upz = uCz / swq; }
  ix = ix + (upx - ix) * pr.z;
  iy = iy + (upy - iy) * pr.z;
  iz = iz + (upz - iz) * pr.z;
  sth(f.X, o, make_float4(ix * alb.x + emi.x, iy * alb.y + emi.y, iz * alb.z + emi.z, 0.0f));
}

// TAA (hush.js:639-677) with a 32 x 8 tile. The pixel's motion, colour and the four history texels of its bilinear
// footprint are loaded before the tile barrier, so the motion -> history dependency overlaps the tile loads. The
// YCoCg tile is held as (Y, Co) pairs beside a Cg plane, so the 3x3 statistics, the history sum, the clip bounds and
// the blend run (Y, Co) as one packed FP32x2 operation and Cg as a scalar one, lane by lane the same arithmetic
// (40 registers: six CTAs per SM).
__global__ void __launch_bounds__(FT_W *FT_H) k_taa_fused(const __grid_constant__ HushFrame f) {
  constexpr int SW = FT_W + 2, SH = FT_H + 2, NT = FT_W * FT_H, NIT = (SW * SH + NT - 1) / NT;
  __shared__ float2 sXY[SW * SH];
  __shared__ float sXZ[SW * SH];
  const int li = threadIdx.x;
  const int tx = li % FT_W, ty = li / FT_W;
  const int px = blockIdx.x * FT_W + tx, py = blockIdx.y * FT_H + ty;
  const int cpx = min(px, f.W - 1), cpy = min(py, f.H - 1);
  const uint2 mvr = __ldg(f.mv + cpy * f.p_mv + cpx);
  const int ox = blockIdx.x * FT_W - 1, oy = blockIdx.y * FT_H - 1;
  uint2 tl[NIT];
#pragma unroll
  for (int it = 0; it < NIT; it++) {
    const int i = min(li + it * NT, SW * SH - 1);
    tl[it] = __ldg(f.X + clampi(oy + i / SW, 0, f.H - 1) * f.W + clampi(ox + i % SW, 0, f.W - 1));
  }
  const uint2 xr = __ldg(f.X + cpy * f.W + cpx);
  // the history footprint (clamped loads; used only when the reprojected position lies inside the image)
  const float4 mv = h4_to_f4(mvr);
  const float szx = (float)f.W, szy = (float)f.H;
  const float uvx = ((float)px + 0.5f + mv.x) / szx, uvy = ((float)py + 0.5f + mv.y) / szy;
  const float ppx = uvx * szx - 0.5f, ppy = uvy * szy - 0.5f;
  const float bxf = floorf(ppx), byf = floorf(ppy);
  const int ibx = (int)bxf, iby = (int)byf;
  uint2 hq[4];
#pragma unroll
  for (int j = 0; j < 4; j++)
    hq[j] = __ldg(f.taa_prev + clampi(iby + (j >> 1), 0, f.H - 1) * f.W + clampi(ibx + (j & 1), 0, f.W - 1));
#pragma unroll
  for (int it = 0; it < NIT; it++) {
    const int i = li + it * NT;
    if (i >= SW * SH) continue;
    const float4 x = h4_to_f4(tl[it]);
    const float3 y = to_ycocg(tmap(make_float3(x.x, x.y, x.z)));
    sXY[i] = make_float2(y.x, y.y);
    sXZ[i] = y.z;
  }
  __syncthreads();
  if (px >= f.W || py >= f.H) return;
  const int o = py * f.W + px;
  const float4 x = h4_to_f4(xr);
  const float3 cur = tmap(make_float3(x.x, x.y, x.z));
  float3 r;
  if (f.reset) {
    r = itmap(cur);
  } else {
    const int ti = (ty + 1) * SW + tx + 1;
    auto c9 = [&](int j) {
      const int t = ti + (j / 3 - 1) * SW + (j % 3 - 1);
      const float2 a = sXY[t];
      return make_float4(a.x, a.y, sXZ[t], 0.0f);
    };
    float2 s2 = f2(0.f, 0.f);
    float s1 = 0.f;
#pragma unroll
    for (int j = 0; j < 9; j++) {
      const float4 c = c9(j);
      s2 = add2(s2, lo2(c));
      s1 += c.z;
    }
    const float m1x = s2.x / 9.0f, m1y = s2.y / 9.0f, m1z = s1 / 9.0f;
    const float2 nm = f2(-m1x, -m1y);
    float2 v2 = f2(0.f, 0.f);
    float v1 = 0.f;
#pragma unroll
    for (int j = 0; j < 9; j++) {
      const float4 c = c9(j);
      const float2 d = add2(lo2(c), nm);
      const float dz = c.z - m1z;
      v2 = fma2(d, d, v2);
      v1 += dz * dz;
    }
    const float sdx = sqrtf(fmaxf(v2.x / 9.0f, 1e-12f)), sdy = sqrtf(fmaxf(v2.y / 9.0f, 1e-12f)),
                sdz = sqrtf(fmaxf(v1 / 9.0f, 1e-12f));
    float3 res = cur;
    if (uvx >= 0.0f && uvy >= 0.0f && uvx <= 1.0f && uvy <= 1.0f) {
      const float fx = ppx - bxf, fy = ppy - byf;
      float2 h2 = f2(0.f, 0.f);
      float h1 = 0.f;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int oxj = j & 1, oyj = j >> 1;
        const float wb = (oxj == 1 ? fx : 1.0f - fx) * (oyj == 1 ? fy : 1.0f - fy);
        const float4 t = h4_to_f4(hq[j]);
        h2 = fma2(bc2(wb), lo2(t), h2);
        h1 += wb * t.z;
      }
      float3 hh = to_ycocg(tmap(make_float3(h2.x, h2.y, h1)));
      const float2 sd2 = f2(sdx, sdy), m12 = f2(m1x, m1y);
      const float2 lo = fma2(bc2(-1.25f), sd2, m12), hi = fma2(bc2(1.25f), sd2, m12);
      hh.x = fminf(fmaxf(hh.x, lo.x), hi.x);
      hh.y = fminf(fmaxf(hh.y, lo.y), hi.y);
      hh.z = fminf(fmaxf(hh.z, m1z - 1.25f * sdz), m1z + 1.25f * sdz);
      const float3 hr = from_ycocg(hh);
      const float2 hr2 = f2(hr.x, hr.y);
      const float2 b2 = fma2(add2(f2(cur.x, cur.y), f2(-hr.x, -hr.y)), bc2(0.1f), hr2);
      res = make_float3(b2.x, b2.y, hr.z + (cur.z - hr.z) * 0.1f);
    }
    r = itmap(res);
  }
  sth(f.taa, o, make_float4(r.x, r.y, r.z, 1.0f));
}

// ------------------------------------------------------------------------------------------------ launchers
static const char *STAGE_LABELS[6] = {"temporal+mlp", "mid1+coarse1", "mid2+coarse2", "mid3", "fine+final", "taa"};
int fused_stage_count() { return 6; }
const char *fused_stage_label(int s) { return (s >= 0 && s < 6) ? STAGE_LABELS[s] : "?"; }

// The half stages' tensor maps for the frame's buffers, encoded when the buffers or sizes change (per host thread).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

static const HalfMaps &half_maps(const HushFrame &f) {
  struct Cache {
    const void *gd = nullptr, *b0 = nullptr, *b1 = nullptr, *ah = nullptr, *cgd = nullptr, *c1 = nullptr;
    int w = -1, h = -1;
    HalfMaps m{};
  };
  static thread_local Cache c;
  if (c.gd == f.Gd && c.b0 == f.Bh0 && c.b1 == f.Bh1 && c.ah == f.Ah && c.cgd == f.CGd && c.c1 == f.C1 &&
      c.w == f.W2 && c.h == f.H2)
    return c.m;
  c.gd = f.Gd; c.b0 = f.Bh0; c.b1 = f.Bh1; c.ah = f.Ah; c.cgd = f.CGd; c.c1 = f.C1; c.w = f.W2; c.h = f.H2;
  std::memset(&c.m, 0, sizeof(c.m));
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (enc && !(f.W4 & 1) && f.W4 >= HT_W + 8 && f.H4 >= HT_H + 8) {  // coarse2's quarter-resolution maps
    const cuuint32_t one3[3] = {1, 1, 1};
    const cuuint64_t gdim[3] = {4, (cuuint64_t)f.W4, (cuuint64_t)f.H4};
    const cuuint64_t gstr[2] = {16, (cuuint64_t)f.W4 * 16};
    const cuuint32_t gbox[3] = {4, (cuuint32_t)(HT_W + 8), (cuuint32_t)(HT_H + 8)};
    const cuuint64_t ldim[2] = {(cuuint64_t)f.W4, (cuuint64_t)f.H4};
    const cuuint64_t lstr[1] = {(cuuint64_t)f.W4 * 8};
    const cuuint32_t lbox[2] = {(cuuint32_t)(HT_W + 8), (cuuint32_t)(HT_H + 8)};
    c.m.qok = enc(&c.m.cgd, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)f.CGd, gdim, gstr, gbox, one3,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
              enc(&c.m.c1, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, (void *)f.C1, ldim, lstr, lbox, one3,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS
                  ? 1
                  : 0;
  }
  // the 8-byte level map needs a row pitch that is a multiple of 16 bytes
  if (!enc || (f.W2 & 1) || f.W2 < HT_W + 8 || f.H2 < HT_H + 8) return c.m;
  const cuuint32_t one[3] = {1, 1, 1};
  auto gd = [&](CUtensorMap *m, int ap) {
    const cuuint64_t dim[3] = {4, (cuuint64_t)f.W2, (cuuint64_t)f.H2};
    const cuuint64_t str[2] = {16, (cuuint64_t)f.W2 * 16};
    const cuuint32_t box[3] = {4, (cuuint32_t)(HT_W + 2 * ap), (cuuint32_t)(HT_H + 2 * ap)};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)f.Gd, dim, str, box, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  };
  auto lv = [&](CUtensorMap *m, const uint2 *p, int ap) {
    const cuuint64_t dim[2] = {(cuuint64_t)f.W2, (cuuint64_t)f.H2};
    const cuuint64_t str[1] = {(cuuint64_t)f.W2 * 8};
    const cuuint32_t box[2] = {(cuuint32_t)(HT_W + 2 * ap), (cuuint32_t)(HT_H + 2 * ap)};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, (void *)p, dim, str, box, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  };
  bool ok = gd(&c.m.gd2, 2) == CUDA_SUCCESS && gd(&c.m.gd4, 4) == CUDA_SUCCESS && gd(&c.m.gd1, 1) == CUDA_SUCCESS &&
            lv(&c.m.bh0, f.Bh0, 2) == CUDA_SUCCESS && lv(&c.m.bh1, f.Bh1, 4) == CUDA_SUCCESS;
  {  // Ah: box (16 + 4) x (8 + 2) from an even x
    const cuuint64_t dim[2] = {(cuuint64_t)f.W2, (cuuint64_t)f.H2};
    const cuuint64_t str[1] = {(cuuint64_t)f.W2 * 8};
    const cuuint32_t box[2] = {(cuuint32_t)(HT_W + 4), (cuuint32_t)(HT_H + 2)};
    ok = ok && enc(&c.m.ah, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, (void *)f.Ah, dim, str, box, one,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  }
  c.m.ok = ok ? 1 : 0;
  return c.m;
}

// FINE_FINAL's maps for the frame's A0 and key (which alternates with the frame parity: two cached entries).
static const FineMaps &fine_maps(const HushFrame &f) {
  struct Entry {
    const void *a0 = nullptr, *key = nullptr;
    int w = -1, h = -1;
    FineMaps m{};
  };
  static thread_local Entry c[2];
  static thread_local int next = 0;
  for (Entry &e : c)
    if (e.a0 == f.A0 && e.key == f.key && e.w == f.W && e.h == f.H) return e.m;
  Entry &e = c[next];
  next ^= 1;
  e.a0 = f.A0; e.key = f.key; e.w = f.W; e.h = f.H;
  std::memset(&e.m, 0, sizeof(e.m));
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || (f.W & 1) || f.W < FB_W || f.H < FB_H) return e.m;
  const cuuint32_t one[2] = {1, 1};
  const cuuint64_t dim[2] = {(cuuint64_t)f.W, (cuuint64_t)f.H};
  const cuuint64_t str[1] = {(cuuint64_t)f.W * 8};
  const cuuint32_t box[2] = {(cuuint32_t)FB_W, (cuuint32_t)FB_H};
  auto lv = [&](CUtensorMap *m, const void *p) {
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void *>(p), dim, str, box, one,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  };
  e.m.ok = (lv(&e.m.a0, f.A0) == CUDA_SUCCESS && lv(&e.m.key, f.key) == CUDA_SUCCESS) ? 1 : 0;
  return e.m;
}

cudaError_t launch_fused_stage(int stage, int part, const HushFrame &f, const MlpConst &mc, int mlp_mode,
                               const void *mlp_tc, cudaStream_t st) {
  const int hx = (f.W2 + HT_W - 1) / HT_W, hy = (f.H2 + HT_H - 1) / HT_H;
  const int qx = (f.W4 + HT_W - 1) / HT_W, qy = (f.H4 + HT_H - 1) / HT_H;
  const int hpx = (f.W2 + MP_W - 1) / MP_W;  // two-pixel mid tiles per row
  switch (stage) {
    case 0: {
      // blob: the tensor-core forms' bf16 hi / lo operands and f16 operands; mc: the weights as a kernel parameter
      const uint4 *blob = (const uint4 *)mlp_tc;
      int dev = 0;
      cudaGetDevice(&dev);
      if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
      const dim3 g((f.W + KB_TW - 1) / KB_TW, (f.H + KB_TH - 1) / KB_TH);
      // every form needs more than 48 KB of dynamic shared memory: opt in once per device and form
      static bool opted[4][64] = {};
      const int m = mlp_mode & 3;
      void (*const kern[4])(HushFrame, MlpConst, const uint4 *) = {k_temporal_block<0>, k_temporal_block<1>,
                                                                   k_temporal_block<2>, k_temporal_block<3>};
      const int smem = (m == 1 || m == 2) ? (int)sizeof(KbTcSmem) : (int)sizeof(KbSmem);
      if (!opted[m][dev]) {
        const cudaError_t e = cudaFuncSetAttribute(kern[m], cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        opted[m][dev] = true;
      }
      const uint4 *b = m == 1 ? blob + MLP_BLOB_BF16 / 16 : m == 2 ? blob + MLP_BLOB_F16 / 16 : blob;
      kern[m]<<<g, KB_NT, smem, st>>>(f, mc, b);
      break;
    }
    // stages 1 and 2: the mid tiles and the coarse tiles are separate kernels (each with its own register count);
    // both parts run them one after the other on `st`
    case 1:
      if (part != HP_COARSE)
        k_half_stage<1, HP_MID><<<hx * hy, HT_W * HT_H, 0, st>>>(f, hx, hx * hy, qx, half_maps(f));
      if (part != HP_MID)
        k_half_stage<1, HP_COARSE><<<qx * qy, HT_W * HT_H, 0, st>>>(f, hx, hx * hy, qx, half_maps(f));
      break;
    case 2: {
      constexpr int smc = 2 * (HT_W + 8) * (HT_H + 8) * 16;  // coarse2's two float4 tiles
      if (part != HP_COARSE)
        k_half_pair<2, HP_MID><<<hpx * hy, HT_W * HT_H, mid_pair_smem<2>(), st>>>(f, hpx, hpx * hy, qx, half_maps(f));
      if (part != HP_MID)
        k_half_pair<2, HP_COARSE><<<qx * qy, HT_W * HT_H, smc, st>>>(f, hpx, hpx * hy, qx, half_maps(f));
      break;
    }
    case 3:
      if (part == HP_COARSE) break;  // no coarse level in stage 3
      k_half_pair<3, HP_MID><<<hpx * hy, HT_W * HT_H, mid_pair_smem<4>(), st>>>(f, hpx, hpx * hy, qx, half_maps(f));
      break;
    case 4:
      k_fine_final_fused<<<dim3((f.W + FT_W - 1) / FT_W, (f.H + FT_H - 1) / FT_H), FT_W * FT_H, 0, st>>>(f, fine_maps(f));
      break;
    case 5: k_taa_fused<<<dim3((f.W + FT_W - 1) / FT_W, (f.H + FT_H - 1) / FT_H), FT_W * FT_H, 0, st>>>(f); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

size_t fused_scratch_bytes(int, int) { return 0; }

int fused_kernel_param_count(const void *func) {
  const void *three[4] = {(const void *)k_temporal_block<0>, (const void *)k_temporal_block<1>,
                          (const void *)k_temporal_block<2>, (const void *)k_temporal_block<3>};
  for (const void *k : three)
    if (func == k) return 3;  // (f, wp, blob)
  const void *half[5] = {(const void *)k_half_stage<1, HP_MID>, (const void *)k_half_stage<1, HP_COARSE>,
                         (const void *)k_half_pair<2, HP_MID>, (const void *)k_half_pair<2, HP_COARSE>,
                         (const void *)k_half_pair<3, HP_MID>};
  for (const void *k : half)
    if (func == k) return 5;  // (f, nAx, nA, nBx, M)
  if (func == (const void *)k_fine_final_fused) return 2;  // (f, M)
  if (func == (const void *)k_taa_fused) return 1;          // (f)
  return 0;
}

}  // namespace hush
