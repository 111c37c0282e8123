// The Hush instance (the reference's `Hush` object, hush.js:725-875), shared by the C ABI and the trainer.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "hush.h"
#include "hush_internal.h"

struct hush_s {
  int dev = 0;
  int W = 0, H = 0, W2 = 0, H2 = 0, W4 = 0, H4 = 0;
  int frame = 0;
  bool reset = true;
  float exposure = 1.0f;
  int hidden = 16;
  int mlp_mode = HUSH_MLP_FP32;
  int schedule = HUSH_SCHED_FUSED;
  std::vector<float> wf;
  hush::MlpW16 w16;
  hush::MlpConst mconst[4];  // stage 0's weights per MLP form (kernel parameter)
  float *w_dev = nullptr;
  void *tc_blob_dev = nullptr;
  // state images (hush.js:783-793) plus the fused path's half-res planes
  char *pool = nullptr;
  size_t pool_bytes = 0;
  uint2 *A0 = nullptr, *X = nullptr, *Bh[2] = {}, *mom[2] = {}, *key[2] = {}, *hist[2] = {}, *taa[2] = {},
        *par0[2] = {}, *par1 = nullptr, *par2 = nullptr, *C[2] = {}, *CG = nullptr, *Ah = nullptr, *Gh = nullptr;
  float4 *Gd = nullptr, *CGd = nullptr;
  uint4 *F[4] = {};
  unsigned int *err = nullptr;
  const void *last_out = nullptr;
  std::string last_error;
  // timer
  int timer_mode = 0;
  int n_events = 0;
  cudaEvent_t ev[17] = {};
  const char *ev_label[16] = {};
  // graph replay
  bool use_graph = false;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  const void *gkey[2][5] = {};
  int gkey_reset[2] = {-1, -1};
  float gkey_exposure[2] = {0, 0};
  // the captured graph each executable graph came from, and its kernel nodes in launch order: a frame whose input
  // buffers differ only updates the nodes' HushFrame parameter instead of capturing the frame again
  cudaGraph_t gtmpl[2] = {nullptr, nullptr};
  std::vector<cudaGraphNode_t> gnodes[2];
  // host-buffer frames (hush_denoise_host): two device staging sets for the five inputs, a copy-in and a copy-out
  // stream, and the events that order them against the frames
  void *hin_pool = nullptr;
  uint2 *hin[2][5] = {};
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_in[2] = {}, ev_used[2] = {}, ev_out[2] = {};
  // the fused frame's coarse branch (COARSE1 -> coarse2 beside mid1 -> mid3): its stream and the fork / join events
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

// helpers of hush_api.cu
hush::HushFrame hush_make_frame(hush_t *h, const hush_inputs *in);
int hush_check_inputs(hush_t *h, const hush_inputs *in);
int hush_fail(hush_t *h, int code, const std::string &msg);
int hush_cuda_fail(hush_t *h, cudaError_t e, const char *what);
