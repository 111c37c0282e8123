// Device helpers shared by the Hush kernels: f16 texel I/O and the reference's COMMON / TILE_FNS functions
// (src/denoise/hush.js:28-49, 67-74, 98-108).
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

#define HD_INL __device__ __forceinline__

namespace hush {

// ------------------------------------------------------------------------------------------------ texels
// A texel of an rgba16float image is 8 bytes (uint2); a packed-feature texel (rgba32uint) is 16 bytes (uint4).
HD_INL float4 h4_to_f4(uint2 t) {
  __half2 a = *reinterpret_cast<__half2 *>(&t.x), b = *reinterpret_cast<__half2 *>(&t.y);
  float2 fa = __half22float2(a), fb = __half22float2(b);
  return make_float4(fa.x, fa.y, fb.x, fb.y);
}
// f32 -> f16 rounded toward zero: the storage-write rounding the reference models (hush.js:98).
HD_INL uint16_t f2h(float x) { return __half_as_ushort(__float2half_rz(x)); }
// Two values in one conversion (cvt.rz.f16x2.f32 puts its first source in the upper half): a in bits 0-15.
HD_INL uint32_t pack2(float a, float b) {
  uint32_t r;
  asm("cvt.rz.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
  return r;
}
HD_INL uint2 f4_to_h4(float4 v) { return make_uint2(pack2(v.x, v.y), pack2(v.z, v.w)); }
HD_INL float2 unpack2(uint32_t u) {
  __half2 h = *reinterpret_cast<__half2 *>(&u);
  return __half22float2(h);
}
HD_INL float4 ldh(const uint2 *__restrict__ p, int idx) { return h4_to_f4(__ldg(p + idx)); }
HD_INL void sth(uint2 *__restrict__ p, int idx, float4 v) { p[idx] = f4_to_h4(v); }
HD_INL float4 quant4(float4 v) {  // value after an rgba16float round trip
  return h4_to_f4(f4_to_h4(v));
}
HD_INL float quant1(float v) { return __half2float(__float2half_rz(v)); }

// qf16 (hush.js:68, 99): clamp to the f16 range, drop the low 13 mantissa bits.
HD_INL float qf16(float x) {
  return __uint_as_float(__float_as_uint(fminf(fmaxf(x, -65504.0f), 65504.0f)) & 0xffffe000u);
}
// pk (hush.js:101): pack2x16float of qf16 values.
HD_INL uint32_t pk(float a, float b) { return pack2(qf16(a), qf16(b)); }

// ------------------------------------------------------------------------------------------------ COMMON
HD_INL float lum3(float r, float g, float b) { return r * 0.2126f + g * 0.7152f + b * 0.0722f; }
HD_INL float lum(float4 c) { return lum3(c.x, c.y, c.z); }
HD_INL float dot3(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

HD_INL float2 oct_enc(float nx, float ny, float nz) {
  float den = fmaxf(fabsf(nx) + fabsf(ny) + fabsf(nz), 1e-20f);
  float vx = nx / den, vy = ny / den, vz = nz / den;
  float sx = vx >= 0.0f ? 1.0f : -1.0f, sy = vy >= 0.0f ? 1.0f : -1.0f;
  if (vz < 0.0f) return make_float2((1.0f - fabsf(vy)) * sx, (1.0f - fabsf(vx)) * sy);
  return make_float2(vx, vy);
}
// Decoded normal in xyz; w is left for the caller (depth).
HD_INL float4 oct_dec(float ex, float ey) {
  float vx = ex, vy = ey, vz = 1.0f - fabsf(ex) - fabsf(ey);
  float t = fmaxf(-vz, 0.0f);
  vx += vx >= 0.0f ? -t : t;
  vy += vy >= 0.0f ? -t : t;
  float l = fmaxf(sqrtf(vx * vx + vy * vy + vz * vz), 1e-20f);
  return make_float4(vx / l, vy / l, vz / l, 0.0f);
}
HD_INL float log1p_w(float x) { return logf(1.0f + x); }  // hush.js:47: log(1 + x)
HD_INL float pow128(float x) {
  float x2 = x * x, x4 = x2 * x2, x8 = x4 * x4, x16 = x8 * x8, x32 = x16 * x16, x64 = x32 * x32;
  return x64 * x64;
}
HD_INL float sigmoidf_(float x) { return 1.0f / (1.0f + expf(-x)); }
HD_INL int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

constexpr float HMAX = 32.0f;
constexpr float COARSE_S = 0.25f;  // hush.js:26
constexpr int N_FEAT = 20;
constexpr int N_OUT = 12;

}  // namespace hush
