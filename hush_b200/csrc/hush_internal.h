// Host-side declarations shared by the kernel files and the C ABI implementation.
#pragma once
#include <cuda_runtime.h>

#include "hush_device.cuh"

namespace hush {

enum {
  PASS_TEMPORAL = 0, PASS_INFER, PASS_MID2, PASS_MID3, PASS_COARSE1, PASS_COARSE2, PASS_FINE_FINAL, PASS_TAA,
  PASS_COUNT
};

// One reference pass (hush_passes.cu).
cudaError_t launch_pass(int pass, const HushFrame &f, const MlpW16 &w16, cudaStream_t st);

// Fused frame kernels (hush_fused.cu). mlp_mode: 0 FP32, 1 BF16 tensor cores, 2 F16 tensor cores.
struct FusedPlan {
  int n_kernels;
  const char *labels[8];
};
cudaError_t launch_fused_stage(int stage, const HushFrame &f, const MlpW16 &w16, int mlp_mode, const void *mlp_tc,
                               cudaStream_t st);
int fused_stage_count();
const char *fused_stage_label(int stage);
size_t fused_scratch_bytes(int W, int H);

// Tensor-core MLP operand blob (weights in the UMMA shared-memory layout), built on the host (mlp_tc.cu).
size_t mlp_tc_blob_bytes();
void mlp_tc_build_blob(const float *w812, int bf16, void *host_blob);

}  // namespace hush
