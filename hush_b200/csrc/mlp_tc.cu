// Host side of the tensor-core MLP: the three weight matrices of the h = 16 network as UMMA B operands.
#include <cstring>

#include "hush_internal.h"
#include "umma.cuh"

namespace hush {

static uint16_t f32_to_bf16_rn(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0;
  return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}

// f32 -> f16 round to nearest even (the weights are f16 values already, so this is exact for them).
static uint16_t f32_to_f16_rn(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  const uint32_t s = (u >> 16) & 0x8000u, a = u & 0x7fffffffu;
  if (a > 0x7f800000u) return (uint16_t)(s | 0x7e00u);
  if (a >= 0x477ff000u) return (uint16_t)(s | 0x7c00u);  // rounds to infinity
  if (a >= 0x38800000u) {                               // normal
    uint32_t m = a - 0x38000000u;                       // rebias exponent
    uint32_t r = (m + 0xfffu + ((m >> 13) & 1u)) >> 13;
    return (uint16_t)(s | r);
  }
  if (a < 0x33000000u) return (uint16_t)s;  // below half the smallest subnormal
  const uint32_t e = a >> 23, mant = (a & 0x7fffffu) | 0x800000u, shift = 126u - e;  // subnormal: mant >> shift
  uint32_t q = mant >> shift, rem = mant & ((1u << shift) - 1u), half = 1u << (shift - 1u);
  if (rem > half || (rem == half && (q & 1u))) q++;
  return (uint16_t)(s | q);
}

static float bf16_to_f32(uint16_t h) {
  const uint32_t u = (uint32_t)h << 16;
  float x;
  std::memcpy(&x, &u, 4);
  return x;
}

void mlp_tc_build_blob(const float *w, int bf16, int lo, uint8_t *blob) {
  std::memset(blob, 0, MLP_TC_BLOB_BYTES);
  auto put = [&](uint8_t *base, int n, int k, int kcore, float v) {
    // lo (bf16 only): the rounding residual v - bf16(v), itself rounded to bf16; hi + lo holds any f16 value exactly
    uint16_t h = bf16 ? f32_to_bf16_rn(v) : f32_to_f16_rn(v);
    if (bf16 && lo) h = f32_to_bf16_rn(v - bf16_to_f32(h));
    std::memcpy(base + umma::kmajor_off(n, k, kcore), &h, 2);
  };
  const int W1 = 0, B1 = 16 * 20, W2 = B1 + 16, B2 = W2 + 256, W3 = B2 + 16;
  for (int n = 0; n < 16; n++)
    for (int k = 0; k < 20; k++) put(blob, n, k, 4, w[W1 + n * 20 + k]);
  for (int n = 0; n < 16; n++)
    for (int k = 0; k < 16; k++) put(blob + 1024, n, k, 2, w[W2 + n * 16 + k]);
  for (int n = 0; n < 12; n++)
    for (int k = 0; k < 16; k++) put(blob + 1536, n, k, 2, w[W3 + n * 16 + k]);
}

void mlp_half_build_blob(const float *w, uint32_t *blob) {
  std::memset(blob, 0, MLP_HALF_BLOB_BYTES);
  const int W1 = 0, B1 = 16 * 20, W2 = B1 + 16, B2 = W2 + 256, W3 = B2 + 16, B3 = W3 + 12 * 16;
  auto pair = [](float a, float b) { return (uint32_t)f32_to_f16_rn(a) | ((uint32_t)f32_to_f16_rn(b) << 16); };
  for (int i = 0; i < 20; i++)
    for (int p = 0; p < 8; p++) blob[MLP_HALF_W1 + i * 8 + p] = pair(w[W1 + 2 * p * 20 + i], w[W1 + (2 * p + 1) * 20 + i]);
  for (int i = 0; i < 16; i++)
    for (int p = 0; p < 8; p++) blob[MLP_HALF_W2 + i * 8 + p] = pair(w[W2 + 2 * p * 16 + i], w[W2 + (2 * p + 1) * 16 + i]);
  for (int i = 0; i < 16; i++)
    for (int p = 0; p < 6; p++) blob[MLP_HALF_W3 + i * 6 + p] = pair(w[W3 + 2 * p * 16 + i], w[W3 + (2 * p + 1) * 16 + i]);
  for (int p = 0; p < 8; p++) {
    blob[MLP_HALF_B1 + p] = pair(w[B1 + 2 * p], w[B1 + 2 * p + 1]);
    blob[MLP_HALF_B2 + p] = pair(w[B2 + 2 * p], w[B2 + 2 * p + 1]);
    if (p < 6) blob[MLP_HALF_B3 + p] = pair(w[B3 + 2 * p], w[B3 + 2 * p + 1]);
  }
}

void mlp_fp32_build_blob(const float *w, float *blob) {
  std::memset(blob, 0, MLP_FP32_BLOB_BYTES);
  const int W1 = 0, B1 = 16 * 20, W2 = B1 + 16, B2 = W2 + 256, W3 = B2 + 16, B3 = W3 + 12 * 16;
  for (int i = 0; i < 20; i++)
    for (int k = 0; k < 4; k++)
      for (int c = 0; c < 4; c++) blob[(MLP_FP32_W1 + i * 4 + k) * 4 + c] = w[W1 + (4 * k + c) * 20 + i];
  for (int i = 0; i < 16; i++)
    for (int k = 0; k < 4; k++)
      for (int c = 0; c < 4; c++) blob[(MLP_FP32_W2 + i * 4 + k) * 4 + c] = w[W2 + (4 * k + c) * 16 + i];
  for (int i = 0; i < 16; i++)
    for (int k = 0; k < 4; k++)
      for (int c = 0; c < 3; c++) blob[(MLP_FP32_W3 + i * 4 + k) * 4 + c] = w[W3 + (4 * c + k) * 16 + i];
  for (int k = 0; k < 4; k++)
    for (int c = 0; c < 4; c++) {
      blob[(MLP_FP32_B1 + k) * 4 + c] = w[B1 + 4 * k + c];
      blob[(MLP_FP32_B2 + k) * 4 + c] = w[B2 + 4 * k + c];
      if (c < 3) blob[(MLP_FP32_B3 + k) * 4 + c] = w[B3 + 4 * c + k];
    }
}

void mlp_const_build(const float *w, int mlp_mode, MlpConst &c) {
  std::memset(&c, 0, sizeof(c));
  if (mlp_mode == 0) mlp_fp32_build_blob(w, reinterpret_cast<float *>(c.w));
  else if (mlp_mode == 3) mlp_half_build_blob(w, reinterpret_cast<uint32_t *>(c.w));
  else std::memcpy(c.w, w, sizeof(MlpW16));
}

}  // namespace hush
