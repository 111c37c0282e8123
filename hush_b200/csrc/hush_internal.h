// Host-side declarations shared by the kernel files and the C ABI implementation.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "hush_device.cuh"

namespace hush {

enum {
  PASS_TEMPORAL = 0, PASS_INFER, PASS_MID2, PASS_MID3, PASS_COARSE1, PASS_COARSE2, PASS_FINE_FINAL, PASS_TAA,
  PASS_COUNT
};

// One reference pass (hush_passes.cu).
cudaError_t launch_pass(int pass, const HushFrame &f, const MlpW16 &w16, cudaStream_t st);

// Fused frame kernels (hush_fused.cu). mlp_mode: 0 FP32, 1 BF16 tensor cores, 2 F16 tensor cores, 3 f16 arithmetic.
struct FusedPlan {
  int n_kernels;
  const char *labels[8];
};
struct MlpConst;
// Which tiles of a half-res stage a launch runs. The mid tiles and the coarse tiles are separate kernels, so that the
// coarse chain (COARSE1 -> coarse2) can run beside the mid chain (mid1 -> mid2 -> mid3) on another stream and each
// kernel keeps its own register count; HP_BOTH runs the stage's two kernels one after the other.
enum HalfPart { HP_BOTH = 0, HP_MID = 1, HP_COARSE = 2 };
// One stage of the fused frame on `st`; part (a HalfPart) selects the tiles of stages 1 and 2, the half-res levels
// with a coarse level beside them (stage 3 has no coarse tiles, the other stages ignore it).
cudaError_t launch_fused_stage(int stage, int part, const HushFrame &f, const MlpConst &mc, int mlp_mode,
                               const void *mlp_tc, cudaStream_t st);
int fused_stage_count();
const char *fused_stage_label(int stage);
size_t fused_scratch_bytes(int W, int H);
// Number of parameters of a fused-schedule kernel (its first parameter is the HushFrame), 0 for any other function.
int fused_kernel_param_count(const void *func);

// Tensor-core MLP weight operands for h = 16 in the UMMA K-major no-swizzle shared-memory layout: B1 (16 x 32, W1
// zero-padded along K), B2 (16 x 16), B3 (16 x 16, W3 zero-padded along N), in bf16 or f16 (mlp_tc.cu). lo = 1
// (bf16): the bf16 residuals w - bf16(w) instead, the low half of a split-precision operand.
constexpr int MLP_TC_BLOB_BYTES = 2048;
void mlp_tc_build_blob(const float *w812, int bf16, int lo, uint8_t *blob);
// f16 weights of the h = 16 network for the f16-arithmetic MLP, as f16x2 unit pairs (low half = the even unit): per
// layer, for input i and pair p the word (w[2p][i], w[2p+1][i]) at i * (units / 2) + p, then the bias pairs.
constexpr int MLP_HALF_W1 = 0, MLP_HALF_B1 = 160, MLP_HALF_W2 = 168, MLP_HALF_B2 = 296, MLP_HALF_W3 = 304,
              MLP_HALF_B3 = 400;  // offsets in 32-bit words
constexpr int MLP_HALF_BLOB_BYTES = 416 * 4;  // 406 words, padded to a multiple of 16 bytes
void mlp_half_build_blob(const float *w812, uint32_t *blob);
// The instance's tensor-core weight operands on the device: bf16 hi | bf16 lo | f16.
constexpr int MLP_BLOB_BF16 = 0, MLP_BLOB_F16 = 2 * MLP_TC_BLOB_BYTES, MLP_BLOB_BYTES = 3 * MLP_TC_BLOB_BYTES;
// FP32 weights of the h = 16 network for the 4-lane MLP: per input i and lane k the float4 of the units lane k owns
// (layer 1 / 2: units 4k..4k+3; layer 3: outputs k, 4+k, 8+k), then the biases in the same grouping.
constexpr int MLP_FP32_W1 = 0, MLP_FP32_W2 = 80, MLP_FP32_W3 = 144, MLP_FP32_B1 = 208, MLP_FP32_B2 = 212,
              MLP_FP32_B3 = 216;  // offsets in float4
constexpr int MLP_FP32_BLOB_BYTES = 220 * 16;
void mlp_fp32_build_blob(const float *w812, float *blob);

// Stage 0's MLP weights as one kernel parameter, so that they sit in the constant bank: every lane of a warp reads
// the same weight, which reaches the FMA as a broadcast operand, and no CTA copies them into shared memory. Mode 0
// holds the FP32 blob, mode 3 the f16x2 blob, the tensor-core modes the decoded weights (they add the biases).
struct MlpConst {
  float4 w[MLP_FP32_BLOB_BYTES / 16];
};
static_assert(MLP_HALF_BLOB_BYTES <= sizeof(MlpConst) && sizeof(MlpW16) <= sizeof(MlpConst), "MlpConst size");
// The parameter for one mode from the 812 decoded weights of the h = 16 network (mlp_tc.cu).
void mlp_const_build(const float *w812, int mlp_mode, MlpConst &c);

}  // namespace hush
