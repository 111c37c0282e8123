// C ABI of the Hush denoiser: the host side of the reference's `Hush` class (src/denoise/hush.js:719-875) over
// CUDA device buffers and streams.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hush.h"
#include "hush_instance.h"
#include "hush_internal.h"
#include "umma.cuh"
#include "weights_builtin.inc"  // generated at build time from hush_b200/data/hush-weights.bin

using namespace hush;

static thread_local std::string g_err;

static float half_to_float(uint16_t h) {  // halfToFloat (hush.js:706-711)
  const int s = (h & 0x8000) ? -1 : 1, e = (h >> 10) & 0x1f, m = h & 0x3ff;
  if (e == 0) return (float)(s * m * std::ldexp(1.0, -24));
  if (e == 31) return m ? NAN : s * INFINITY;
  return (float)(s * (1.0 + m / 1024.0) * std::ldexp(1.0, e - 15));
}


int hush_fail(hush_t *h, int code, const std::string &msg) {
  if (h) h->last_error = msg;
  g_err = msg;
  return code;
}
int hush_cuda_fail(hush_t *h, cudaError_t e, const char *what) {
  return hush_fail(h, HUSH_ERR_CUDA, std::string("Hush: ") + what + ": " + cudaGetErrorString(e));
}

extern "C" int hush_hidden_of(long n) {
  for (long h = 1; h <= 256; h++)
    if (h * h + (N_FEAT + N_OUT + 2) * h + N_OUT == n) return (int)h;
  return 0;
}

extern "C" hush_desc hush_desc_default(int width, int height) {
  hush_desc d;
  std::memset(&d, 0, sizeof(d));
  d.width = width;
  d.height = height;
  d.exposure = 1.0f;
  d.weights = nullptr;
  d.n_weights = 0;
  d.f16 = 0;
  d.mlp_mode = HUSH_MLP_FP32;
  d.schedule = HUSH_SCHED_FUSED;
  d.device = -1;
  return d;
}

extern "C" void hush_required_limits(int *cc_major, int *cc_minor, size_t *shared_bytes) {
  if (cc_major) *cc_major = 10;
  if (cc_minor) *cc_minor = 0;
  if (shared_bytes) *shared_bytes = 100 * 1024;
}

static void drop_graphs(hush_t *h) {
  for (int i = 0; i < 2; i++) {
    if (h->gexec[i]) cudaGraphExecDestroy(h->gexec[i]);
    if (h->gtmpl[i]) cudaGraphDestroy(h->gtmpl[i]);
    h->gexec[i] = nullptr;
    h->gtmpl[i] = nullptr;
    h->gnodes[i].clear();
    h->gkey_reset[i] = -1;
  }
}

// The kernel nodes of a captured fused frame in launch order, or none if the graph holds anything the parameter
// update below cannot rewrite (another node type, a kernel outside the fused schedule).
static std::vector<cudaGraphNode_t> frame_kernel_nodes(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0 || n > 16) return {};
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return {};
  for (cudaGraphNode_t nd : nodes) {
    cudaGraphNodeType t;
    cudaKernelNodeParams p;
    if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeKernel ||
        cudaGraphKernelNodeGetParams(nd, &p) != cudaSuccess || hush::fused_kernel_param_count(p.func) == 0)
      return {};
  }
  return nodes;
}

// A frame of the same parity, reset flag and exposure as the executable graph's, with other input buffers: every
// fused kernel takes the frame as its first parameter, so the graph is brought up to date by setting that parameter
// of each kernel node (the other parameters, which depend only on the instance's own buffers, are kept).
static cudaError_t update_frame_params(hush_t *h, int cur, const hush::HushFrame &f) {
  for (cudaGraphNode_t nd : h->gnodes[cur]) {
    cudaKernelNodeParams p;
    cudaError_t e = cudaGraphKernelNodeGetParams(nd, &p);
    if (e != cudaSuccess) return e;
    const int n = hush::fused_kernel_param_count(p.func);
    if (n <= 0 || n > 8 || !p.kernelParams) return cudaErrorInvalidValue;
    void *args[8];
    args[0] = const_cast<hush::HushFrame *>(&f);
    for (int i = 1; i < n; i++) args[i] = p.kernelParams[i];
    p.kernelParams = args;
    p.extra = nullptr;
    e = cudaGraphExecKernelNodeSetParams(h->gexec[cur], nd, &p);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static void free_host_staging(hush_t *h) {
  if (h->hin_pool) {
    cudaDeviceSynchronize();  // copies into the staging sets may still be in flight
    cudaFree(h->hin_pool);
  }
  h->hin_pool = nullptr;
  for (auto &set : h->hin)
    for (auto &p : set) p = nullptr;
}

static void free_state(hush_t *h) {
  if (h->pool) cudaFree(h->pool);
  h->pool = nullptr;
  h->pool_bytes = 0;
  drop_graphs(h);
  free_host_staging(h);
}

// resize (hush.js:764-794): one pool for every state image, 256-byte aligned sub-allocations, zero-initialised like
// fresh WebGPU textures.
static int alloc_state(hush_t *h, int width, int height) {
  const int W = width, H = height, W2 = (W + 1) / 2, H2 = (H + 1) / 2, W4 = (W2 + 1) / 2, H4 = (H2 + 1) / 2;
  const size_t full = (size_t)W * H * 8, half = (size_t)W2 * H2 * 8, quarter = (size_t)W4 * H4 * 8,
               half16 = (size_t)W2 * H2 * 16;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  size_t total = al(full) * 10 + al(half) * 8 + al(half16) * 5 + al(quarter) * 3 + al(quarter * 2) + 256;
  char *pool = nullptr;
  cudaError_t e = cudaMalloc(&pool, total);
  if (e != cudaSuccess) return hush_cuda_fail(h, e, "cudaMalloc of the state images");
  e = cudaMemset(pool, 0, total);
  if (e != cudaSuccess) { cudaFree(pool); return hush_cuda_fail(h, e, "cudaMemset"); }
  free_state(h);
  h->pool = pool;
  h->pool_bytes = total;
  size_t off = 0;
  auto take = [&](size_t b) { char *p = pool + off; off += al(b); return p; };
  h->A0 = (uint2 *)take(full); h->X = (uint2 *)take(full);
  for (int i = 0; i < 2; i++) {
    h->mom[i] = (uint2 *)take(full); h->key[i] = (uint2 *)take(full); h->hist[i] = (uint2 *)take(full);
    h->taa[i] = (uint2 *)take(full);
  }
  for (int i = 0; i < 2; i++) { h->Bh[i] = (uint2 *)take(half); h->par0[i] = (uint2 *)take(half); }
  h->par1 = (uint2 *)take(half); h->par2 = (uint2 *)take(half); h->Ah = (uint2 *)take(half); h->Gh = (uint2 *)take(half);
  for (int i = 0; i < 4; i++) h->F[i] = (uint4 *)take(half16);
  h->Gd = (float4 *)take(half16);
  h->C[0] = (uint2 *)take(quarter); h->C[1] = (uint2 *)take(quarter); h->CG = (uint2 *)take(quarter);
  h->CGd = (float4 *)take(quarter * 2);
  h->err = (unsigned int *)take(256);
  h->W = W; h->H = H; h->W2 = W2; h->H2 = H2; h->W4 = W4; h->H4 = H4;
  h->frame = 0;
  h->reset = true;
  h->last_out = nullptr;
  return HUSH_OK;
}

static int set_weights(hush_t *h, const uint16_t *weights, size_t n) {
  const int hd = hush_hidden_of((long)n);
  if (!hd) return hush_fail(h, HUSH_ERR_ARG, "hush weights: " + std::to_string(n) + " f16 values fit no MLP size");
  std::vector<float> wf(n);
  for (size_t i = 0; i < n; i++) wf[i] = half_to_float(weights[i]);
  float *wd = nullptr;
  cudaError_t e = cudaMalloc(&wd, n * sizeof(float));
  if (e != cudaSuccess) return hush_cuda_fail(h, e, "cudaMalloc of the weights");
  e = cudaMemcpy(wd, wf.data(), n * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cudaFree(wd); return hush_cuda_fail(h, e, "cudaMemcpy of the weights"); }
  if (h->w_dev) cudaFree(h->w_dev);
  h->w_dev = wd;
  h->wf = wf;
  h->hidden = hd;
  std::memset(&h->w16, 0, sizeof(h->w16));
  if (hd == 16) {
    std::memcpy(h->w16.w, wf.data(), sizeof(h->w16.w));
    // stage 0's constant-bank weights per MLP form, and the tensor-core operands (bf16 hi, bf16 lo, f16)
    for (int m = 0; m < 4; m++) mlp_const_build(wf.data(), m, h->mconst[m]);
    alignas(16) uint8_t blob[MLP_BLOB_BYTES];
    mlp_tc_build_blob(wf.data(), 1, 0, blob + MLP_BLOB_BF16);
    mlp_tc_build_blob(wf.data(), 1, 1, blob + MLP_BLOB_BF16 + MLP_TC_BLOB_BYTES);
    mlp_tc_build_blob(wf.data(), 0, 0, blob + MLP_BLOB_F16);
    if (!h->tc_blob_dev) {
      e = cudaMalloc(&h->tc_blob_dev, sizeof(blob));
      if (e != cudaSuccess) return hush_cuda_fail(h, e, "cudaMalloc of the tensor-core weights");
    }
    e = cudaMemcpy(h->tc_blob_dev, blob, sizeof(blob), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return hush_cuda_fail(h, e, "cudaMemcpy of the tensor-core weights");
  }
  drop_graphs(h);  // graphs bake the weights in as kernel parameters
  return HUSH_OK;
}

extern "C" int hush_create(const hush_desc *desc, hush_t **out) {
  if (!out) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_create: out is NULL");
  *out = nullptr;
  if (!desc) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_create: desc is NULL");
  int dev = desc->device;
  cudaError_t e;
  if (dev < 0) {
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return hush_cuda_fail(nullptr, e, "cudaGetDevice");
  }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) return hush_cuda_fail(nullptr, e, "cudaGetDeviceProperties");
  int need_major, need_minor;
  size_t need_smem;
  hush_required_limits(&need_major, &need_minor, &need_smem);
  if (prop.major != need_major || prop.sharedMemPerBlockOptin < need_smem) {
    return hush_fail(nullptr, HUSH_ERR_DEVICE,
                "Hush needs the device limit computeCapability == " + std::to_string(need_major) + "." +
                    std::to_string(need_minor) + " (sm_100a) and sharedMemPerBlockOptin >= " +
                    std::to_string(need_smem) + " (this device: " + std::to_string(prop.major) + "." +
                    std::to_string(prop.minor) + ", " + std::to_string(prop.sharedMemPerBlockOptin) + ")");
  }
  if (!(desc->width > 0 && desc->height > 0))
    return hush_fail(nullptr, HUSH_ERR_ARG,
                "Hush: bad size " + std::to_string(desc->width) + "x" + std::to_string(desc->height));
  if (desc->mlp_mode < HUSH_MLP_FP32 || desc->mlp_mode > HUSH_MLP_HALF)
    return hush_fail(nullptr, HUSH_ERR_ARG, "Hush: unknown mlp_mode " + std::to_string(desc->mlp_mode));
  if (desc->schedule != HUSH_SCHED_FUSED && desc->schedule != HUSH_SCHED_PASSES)
    return hush_fail(nullptr, HUSH_ERR_ARG, "Hush: unknown schedule " + std::to_string(desc->schedule));
  e = cudaSetDevice(dev);
  if (e != cudaSuccess) return hush_cuda_fail(nullptr, e, "cudaSetDevice");
  hush_t *h = new hush_t();
  h->dev = dev;
  h->exposure = desc->exposure;
  h->mlp_mode = desc->mlp_mode;
  if (desc->f16 && h->mlp_mode == HUSH_MLP_FP32) h->mlp_mode = HUSH_MLP_HALF;  // the reference's f16 arithmetic
  h->schedule = desc->schedule;
  const uint16_t *w = desc->weights ? desc->weights : HUSH_BUILTIN_WEIGHTS;
  const size_t n = desc->weights ? desc->n_weights : HUSH_BUILTIN_WEIGHT_COUNT;
  int rc = set_weights(h, w, n);
  if (rc == HUSH_OK) rc = alloc_state(h, desc->width, desc->height);
  if (rc == HUSH_OK) {
    for (int i = 0; i < 17 && rc == HUSH_OK; i++) {
      e = cudaEventCreate(&h->ev[i]);
      if (e != cudaSuccess) rc = hush_cuda_fail(h, e, "cudaEventCreate");
    }
  }
  if (rc == HUSH_OK) {  // the fused frame's coarse branch
    e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) rc = hush_cuda_fail(h, e, "creating the coarse-level stream");
  }
  if (rc != HUSH_OK) {
    g_err = h->last_error;
    hush_destroy(h);
    return rc;
  }
  *out = h;
  return HUSH_OK;
}

extern "C" void hush_destroy(hush_t *h) {
  if (!h) return;
  cudaSetDevice(h->dev);
  free_state(h);
  if (h->w_dev) cudaFree(h->w_dev);
  if (h->tc_blob_dev) cudaFree(h->tc_blob_dev);
  for (int i = 0; i < 17; i++)
    if (h->ev[i]) cudaEventDestroy(h->ev[i]);
  for (int i = 0; i < 2; i++)
    for (cudaEvent_t e : {h->ev_in[i], h->ev_used[i], h->ev_out[i]})
      if (e) cudaEventDestroy(e);
  if (h->h2d) cudaStreamDestroy(h->h2d);
  if (h->d2h) cudaStreamDestroy(h->d2h);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  if (h->side) cudaStreamDestroy(h->side);
  delete h;
}

extern "C" int hush_resize(hush_t *h, int width, int height) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_resize: NULL instance");
  if (!(width > 0 && height > 0))
    return hush_fail(h, HUSH_ERR_ARG, "Hush: bad size " + std::to_string(width) + "x" + std::to_string(height));
  if (width == h->W && height == h->H) return HUSH_OK;
  cudaSetDevice(h->dev);
  return alloc_state(h, width, height);
}

extern "C" int hush_reset(hush_t *h) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_reset: NULL instance");
  h->reset = true;
  return HUSH_OK;
}
extern "C" int hush_set_exposure(hush_t *h, float e) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_set_exposure: NULL instance");
  h->exposure = e;
  return HUSH_OK;
}
extern "C" float hush_get_exposure(const hush_t *h) { return h ? h->exposure : 0.0f; }
extern "C" int hush_set_weights(hush_t *h, const uint16_t *w, size_t n) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_set_weights: NULL instance");
  if (!w) return hush_fail(h, HUSH_ERR_ARG, "hush weights: NULL blob");
  cudaSetDevice(h->dev);
  return set_weights(h, w, n);
}
extern "C" int hush_set_mlp_mode(hush_t *h, int mode) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_set_mlp_mode: NULL instance");
  if (mode < HUSH_MLP_FP32 || mode > HUSH_MLP_HALF) return hush_fail(h, HUSH_ERR_ARG, "Hush: unknown mlp_mode");
  h->mlp_mode = mode;
  drop_graphs(h);
  return HUSH_OK;
}
extern "C" int hush_set_schedule(hush_t *h, int s) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_set_schedule: NULL instance");
  if (s != HUSH_SCHED_FUSED && s != HUSH_SCHED_PASSES) return hush_fail(h, HUSH_ERR_ARG, "Hush: unknown schedule");
  h->schedule = s;
  drop_graphs(h);
  return HUSH_OK;
}
extern "C" int hush_get_size(const hush_t *h, int *w, int *hh) {
  if (!h) return HUSH_ERR_ARG;
  if (w) *w = h->W;
  if (hh) *hh = h->H;
  return HUSH_OK;
}
extern "C" int hush_get_hidden(const hush_t *h) { return h ? h->hidden : 0; }
extern "C" int hush_get_frame(const hush_t *h) { return h ? h->frame : 0; }
extern "C" const char *hush_last_error(const hush_t *h) { return h ? h->last_error.c_str() : g_err.c_str(); }
extern "C" const char *hush_global_error(void) { return g_err.c_str(); }

static const char *INPUT_NAMES[5] = {"radiance", "normalDepth", "motion", "material", "emission"};

// Input checks of denoise() (hush.js:814-820).
int hush_check_inputs(hush_t *h, const hush_inputs *in) {
  if (!in) return hush_fail(h, HUSH_ERR_ARG, "Hush.denoise: missing inputs");
  const void *p[5] = {in->radiance, in->normal_depth, in->motion, in->material, in->emission};
  for (int k = 0; k < 5; k++) {
    if (!p[k]) return hush_fail(h, HUSH_ERR_ARG, std::string("Hush.denoise: missing input '") + INPUT_NAMES[k] + "'");
    const int w = in->width[k], hh = in->height[k];
    if ((w || hh) && (w != h->W || hh != h->H)) {
      return hush_fail(h, HUSH_ERR_ARG,
                  std::string("Hush.denoise: '") + INPUT_NAMES[k] + "' is " + std::to_string(w) + "x" +
                      std::to_string(hh) + ", the denoiser " + std::to_string(h->W) + "x" + std::to_string(h->H) +
                      " (call resize)");
    }
    const size_t pitch = in->pitch[k];
    if (pitch && (pitch % 8 || pitch < (size_t)h->W * 8))
      return hush_fail(h, HUSH_ERR_ARG, std::string("Hush.denoise: bad pitch for '") + INPUT_NAMES[k] + "'");
    if ((uintptr_t)p[k] % 8)
      return hush_fail(h, HUSH_ERR_ARG, std::string("Hush.denoise: '") + INPUT_NAMES[k] + "' is not 8-byte aligned");
  }
  return HUSH_OK;
}

HushFrame hush_make_frame(hush_t *h, const hush_inputs *in) {
  const int cur = h->frame & 1, prev = cur ^ 1;
  HushFrame f;
  std::memset(&f, 0, sizeof(f));
  f.W = h->W; f.H = h->H; f.W2 = h->W2; f.H2 = h->H2; f.W4 = h->W4; f.H4 = h->H4;
  f.reset = h->reset ? 1 : 0;
  f.exposure = h->exposure;
  if (in) {
    const void *p[5] = {in->radiance, in->normal_depth, in->motion, in->material, in->emission};
    int pt[5];
    for (int k = 0; k < 5; k++) pt[k] = in->pitch[k] ? (int)(in->pitch[k] / 8) : h->W;
    f.rad = (const uint2 *)p[0]; f.nd = (const uint2 *)p[1]; f.mv = (const uint2 *)p[2];
    f.mat = (const uint2 *)p[3]; f.emi = (const uint2 *)p[4];
    f.p_rad = pt[0]; f.p_nd = pt[1]; f.p_mv = pt[2]; f.p_mat = pt[3]; f.p_emi = pt[4];
  }
  f.key_prev = h->key[prev]; f.hist_prev = h->hist[prev]; f.mom_prev = h->mom[prev];
  f.par0_prev = h->par0[prev]; f.taa_prev = h->taa[prev];
  f.A0 = h->A0; f.X = h->X; f.mom = h->mom[cur]; f.key = h->key[cur]; f.hist = h->hist[cur]; f.taa = h->taa[cur];
  f.par0 = h->par0[cur]; f.par1 = h->par1; f.par2 = h->par2; f.Bh0 = h->Bh[0]; f.Bh1 = h->Bh[1];
  f.C0 = h->C[0]; f.C1 = h->C[1]; f.CG = h->CG;
  f.F0 = h->F[0]; f.F1 = h->F[1]; f.F2 = h->F[2]; f.F3 = h->F[3];
  f.Ah = h->Ah; f.Gh = h->Gh; f.Gd = h->Gd; f.CGd = h->CGd;
  f.w_glob = h->w_dev;
  f.hidden = h->hidden;
  f.mlp_half = h->mlp_mode == HUSH_MLP_HALF ? 1 : 0;
  f.err = h->err;
  return f;
}

static const char *PASS_LABELS[PASS_COUNT] = {"temporal", "infer+mid", "infer+mid", "infer+mid",
                                              "coarse",   "coarse",    "fine+final", "taa"};

// encode (hush.js:835-874): the frame's kernels on `st`, with optional timing events around each.
static int encode_frame(hush_t *h, const HushFrame &f, cudaStream_t st, bool timed) {
  cudaError_t e = cudaSuccess;
  int n = 0;
  auto mark = [&](const char *label) {
    if (!timed) return;
    if (h->timer_mode == 1 || n == 0) {
      cudaEventRecord(h->ev[n], st);
      h->ev_label[n] = label;
      n++;
    }
  };
  // the tensor-core MLP exists in the fused temporal kernel for h = 16; other widths run the reference passes
  if (h->schedule == HUSH_SCHED_PASSES || h->hidden != 16) {
    for (int p = 0; p < PASS_COUNT && e == cudaSuccess; p++) {
      mark(PASS_LABELS[p]);
      e = launch_pass(p, f, h->w16, st);
    }
  } else {
    // The coarse chain (the coarse tiles of stages 1 and 2: COARSE1, then coarse2) needs only stage 0's outputs and
    // feeds only FINE_FINAL (stage 4). Untimed, it runs on the instance's side stream beside the mid chain (mid1 ->
    // mid2 -> mid3), forked after stage 0 and joined before stage 4 (a captured frame holds them as two parallel
    // branches), so its tiles fill the issue slots the latency-bound mid kernels leave and each kernel keeps its own
    // register count. Timed frames keep one stream and run each stage's mid and coarse kernels one after the other,
    // so that the stage times add up to the frame.
    const bool fork = !timed && h->side;
    const MlpConst &mc = h->mconst[h->mlp_mode];
    const int ns = fused_stage_count();
    for (int s = 0; s < ns && e == cudaSuccess; s++) {
      mark(fused_stage_label(s));
      if (fork && s == 1) {
        e = cudaEventRecord(h->ev_fork, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(h->side, h->ev_fork, 0);
        for (int c = 1; c <= 2 && e == cudaSuccess; c++)
          e = launch_fused_stage(c, HP_COARSE, f, mc, h->mlp_mode, h->tc_blob_dev, h->side);
        if (e == cudaSuccess) e = cudaEventRecord(h->ev_join, h->side);
      }
      if (fork && s == 4 && e == cudaSuccess) e = cudaStreamWaitEvent(st, h->ev_join, 0);
      if (e != cudaSuccess) break;
      const int part = (s == 1 || s == 2) && fork ? HP_MID : HP_BOTH;
      e = launch_fused_stage(s, part, f, mc, h->mlp_mode, h->tc_blob_dev, st);
    }
  }
  if (timed) {
    cudaEventRecord(h->ev[n], st);
    h->n_events = n + 1;
  }
  if (e != cudaSuccess) return hush_cuda_fail(h, e, "kernel launch");
  return HUSH_OK;
}

extern "C" int hush_denoise(hush_t *h, const hush_inputs *in, void *stream, const void **out) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_denoise: NULL instance");
  int rc = hush_check_inputs(h, in);
  if (rc != HUSH_OK) return rc;
  cudaSetDevice(h->dev);
  cudaStream_t st = (cudaStream_t)stream;
  const int cur = h->frame & 1;
  const HushFrame f = hush_make_frame(h, in);
  const bool timed = h->timer_mode != 0;
  if (h->use_graph && !timed) {
    // one graph per ping-pong parity, keyed by the input pointers, the reset flag and the exposure
    const void *key[5] = {in->radiance, in->normal_depth, in->motion, in->material, in->emission};
    bool hit = h->gexec[cur] && h->gkey_reset[cur] == f.reset && h->gkey_exposure[cur] == f.exposure &&
               std::memcmp(h->gkey[cur], key, sizeof(key)) == 0;
    if (!hit && h->gexec[cur] && !h->gnodes[cur].empty() && h->gkey_reset[cur] == f.reset &&
        h->gkey_exposure[cur] == f.exposure) {
      // only the input buffers changed: rewrite the frame parameter of each kernel node
      if (update_frame_params(h, cur, f) == cudaSuccess) {
        std::memcpy(h->gkey[cur], key, sizeof(key));
        hit = true;
      } else {
        cudaGetLastError();  // clear the failure; capture instead
      }
    }
    if (!hit) {
      // capture the frame again; an existing executable graph of the same parity is updated in place (same
      // kernels, new parameters), which is much cheaper than instantiating a new one
      cudaStream_t cs;
      cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
      if (e != cudaSuccess) return hush_cuda_fail(h, e, "cudaStreamCreate");
      e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) { cudaStreamDestroy(cs); return hush_cuda_fail(h, e, "cudaStreamBeginCapture"); }
      rc = encode_frame(h, f, cs, false);
      cudaGraph_t g = nullptr;
      e = cudaStreamEndCapture(cs, &g);
      cudaStreamDestroy(cs);
      if (rc != HUSH_OK) { if (g) cudaGraphDestroy(g); return rc; }
      if (e != cudaSuccess) return hush_cuda_fail(h, e, "cudaStreamEndCapture");
      bool updated = false;
      if (h->gexec[cur]) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(h->gexec[cur], g, &info) == cudaSuccess;
        if (!updated) {
          cudaGetLastError();  // clear the update failure; instantiate instead
          cudaGraphExecDestroy(h->gexec[cur]);
          h->gexec[cur] = nullptr;
        }
      }
      if (updated) {
        // the executable graph keeps the node identities of the graph it was instantiated from (gtmpl)
        cudaGraphDestroy(g);
      } else {
        e = cudaGraphInstantiate(&h->gexec[cur], g, 0);
        if (h->gtmpl[cur]) cudaGraphDestroy(h->gtmpl[cur]);
        h->gtmpl[cur] = nullptr;
        h->gnodes[cur].clear();
        if (e != cudaSuccess) {
          cudaGraphDestroy(g);
          h->gexec[cur] = nullptr;
          return hush_cuda_fail(h, e, "cudaGraphInstantiate");
        }
        // keep the captured graph: its kernel nodes name the executable graph's nodes for parameter updates (their
        // parameters other than the frame depend only on the instance's buffers, sizes, weights and MLP form, and
        // any change of those drops the graphs)
        h->gtmpl[cur] = g;
        if (h->schedule == HUSH_SCHED_FUSED) h->gnodes[cur] = frame_kernel_nodes(g);
      }
      std::memcpy(h->gkey[cur], key, sizeof(key));
      h->gkey_reset[cur] = f.reset;
      h->gkey_exposure[cur] = f.exposure;
    }
    cudaError_t e = cudaGraphLaunch(h->gexec[cur], st);
    if (e != cudaSuccess) return hush_cuda_fail(h, e, "cudaGraphLaunch");
  } else {
    rc = encode_frame(h, f, st, timed);
    if (rc != HUSH_OK) return rc;
  }
  h->reset = false;
  h->frame++;
  h->last_out = h->taa[cur];
  if (out) *out = h->last_out;
  return HUSH_OK;
}

// Host-buffer frames. Frame t uses staging set t & 1: its five input copies run on the copy-in stream after frame
// t - 2 has finished reading that set, the frame runs on `stream` after its copies, and the output copy runs on the
// copy-out stream after the frame; frame t + 2, which rewrites the same output image, waits for that copy. So the
// input copy of frame t + 1 and the output copy of frame t - 1 overlap frame t's kernels.
extern "C" int hush_denoise_host(hush_t *h, const hush_inputs *in, void *out_host, size_t out_pitch, void *stream) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_denoise_host: NULL instance");
  int rc = hush_check_inputs(h, in);
  if (rc != HUSH_OK) return rc;
  if (!out_host) return hush_fail(h, HUSH_ERR_ARG, "hush_denoise_host: missing output buffer");
  const size_t row = (size_t)h->W * 8, opitch = out_pitch ? out_pitch : row;
  if (opitch < row) return hush_fail(h, HUSH_ERR_ARG, "hush_denoise_host: output pitch is smaller than a row");
  cudaSetDevice(h->dev);
  cudaError_t e = cudaSuccess;
  if (!h->h2d) {
    e = cudaStreamCreateWithFlags(&h->h2d, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->d2h, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; i++)
      for (cudaEvent_t *ev : {&h->ev_in[i], &h->ev_used[i], &h->ev_out[i]})
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return hush_cuda_fail(h, e, "hush_denoise_host: stream / event creation");
    for (int i = 0; i < 2 && e == cudaSuccess; i++) {  // nothing to wait for before the first frames
      e = cudaEventRecord(h->ev_used[i], h->h2d);
      if (e == cudaSuccess) e = cudaEventRecord(h->ev_out[i], h->d2h);
    }
    if (e != cudaSuccess) return hush_cuda_fail(h, e, "hush_denoise_host: cudaEventRecord");
  }
  if (!h->hin_pool) {
    const size_t img = ((size_t)h->W * h->H * 8 + 255) & ~(size_t)255;
    e = cudaMalloc(&h->hin_pool, img * 10);
    if (e != cudaSuccess) {
      h->hin_pool = nullptr;
      return hush_cuda_fail(h, e, "hush_denoise_host: staging allocation");
    }
    for (int s = 0; s < 2; s++)
      for (int k = 0; k < 5; k++) h->hin[s][k] = reinterpret_cast<uint2 *>(static_cast<char *>(h->hin_pool) + img * (5 * s + k));
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int s = h->frame & 1;
  const void *src[5] = {in->radiance, in->normal_depth, in->motion, in->material, in->emission};
  e = cudaStreamWaitEvent(h->h2d, h->ev_used[s], 0);
  for (int k = 0; k < 5 && e == cudaSuccess; k++) {
    const size_t sp = in->pitch[k] ? in->pitch[k] : row;
    e = cudaMemcpy2DAsync(h->hin[s][k], row, src[k], sp, row, (size_t)h->H, cudaMemcpyHostToDevice, h->h2d);
  }
  if (e == cudaSuccess) e = cudaEventRecord(h->ev_in[s], h->h2d);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h->ev_in[s], 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h->ev_out[s], 0);  // frame t - 2's output copy is done
  if (e != cudaSuccess) return hush_cuda_fail(h, e, "hush_denoise_host: input copies");
  hush_inputs dev{};
  const void **dst[5] = {&dev.radiance, &dev.normal_depth, &dev.motion, &dev.material, &dev.emission};
  for (int k = 0; k < 5; k++) *dst[k] = h->hin[s][k];
  const void *out = nullptr;
  rc = hush_denoise(h, &dev, stream, &out);
  if (rc != HUSH_OK) return rc;
  e = cudaEventRecord(h->ev_used[s], st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(h->d2h, h->ev_used[s], 0);
  if (e == cudaSuccess) e = cudaMemcpy2DAsync(out_host, opitch, out, row, row, (size_t)h->H, cudaMemcpyDeviceToHost, h->d2h);
  if (e == cudaSuccess) e = cudaEventRecord(h->ev_out[s], h->d2h);
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(h, e, "hush_denoise_host: output copy");
}

// `stream` waits until every output copy enqueued by hush_denoise_host so far has landed in host memory.
extern "C" int hush_host_join(hush_t *h, void *stream) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_host_join: NULL instance");
  if (!h->d2h) return HUSH_OK;
  cudaSetDevice(h->dev);
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaStreamWaitEvent((cudaStream_t)stream, h->ev_out[i], 0);
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(h, e, "hush_host_join");
}

extern "C" const void *hush_output(const hush_t *h) {
  if (!h) return nullptr;
  return h->taa[(h->frame + 1) & 1];
}

extern "C" int hush_timer_enable(hush_t *h, int mode) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_timer_enable: NULL instance");
  if (mode < 0 || mode > 2) return hush_fail(h, HUSH_ERR_ARG, "hush_timer_enable: mode must be 0, 1 or 2");
  h->timer_mode = mode;
  h->n_events = 0;
  return HUSH_OK;
}

extern "C" int hush_timer_read(hush_t *h, hush_timing *out, int max) {
  if (!h) return -1;
  if (h->n_events < 2) return 0;
  cudaError_t e = cudaEventSynchronize(h->ev[h->n_events - 1]);
  if (e != cudaSuccess) { hush_cuda_fail(h, e, "cudaEventSynchronize"); return -1; }
  int k = 0;
  if (h->timer_mode == 2) {
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev[0], h->ev[h->n_events - 1]);
    if (max > 0) { out[0].label = "total"; out[0].ms = ms; k = 1; }
    return k;
  }
  for (int i = 0; i + 1 < h->n_events && k < max; i++) {
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev[i], h->ev[i + 1]);
    out[k].label = h->ev_label[i];
    out[k].ms = ms;
    k++;
  }
  return k;
}

extern "C" int hush_set_graph(hush_t *h, int enable) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_set_graph: NULL instance");
  h->use_graph = enable != 0;
  return HUSH_OK;
}

extern "C" int hush_run_pass(hush_t *h, int pass, const hush_inputs *in, void *stream) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_run_pass: NULL instance");
  if (pass < 0 || pass >= PASS_COUNT) return hush_fail(h, HUSH_ERR_ARG, "hush_run_pass: bad pass id");
  const bool needs_inputs = pass == PASS_TEMPORAL || pass == PASS_FINE_FINAL || pass == PASS_TAA;
  if (needs_inputs) {
    int rc = hush_check_inputs(h, in);
    if (rc != HUSH_OK) return rc;
  }
  cudaSetDevice(h->dev);
  const HushFrame f = hush_make_frame(h, needs_inputs ? in : nullptr);
  cudaError_t e = launch_pass(pass, f, h->w16, (cudaStream_t)stream);
  if (e != cudaSuccess) return hush_cuda_fail(h, e, "kernel launch");
  return HUSH_OK;
}

// ------------------------------------------------------------------------------------------------ kernel status
// The kernels' error word: bits are set where a bounded wait gave up (1: the tensor-core MLP of stage 0, 2: the
// trainer's tensor-core MLP, 4: the wait self-test, 8: a TMA halo-tile copy). Reading it synchronises the device.
extern "C" int hush_kernel_status(hush_t *h, unsigned *word) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_kernel_status: NULL instance");
  cudaSetDevice(h->dev);
  unsigned w = 0;
  cudaError_t e = cudaMemcpy(&w, h->err, sizeof(w), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && w) e = cudaMemset(h->err, 0, sizeof(w));
  if (e != cudaSuccess) return hush_cuda_fail(h, e, "reading the kernel error word");
  if (word) *word = w;
  if (w) {
    char msg[96];
    std::snprintf(msg, sizeof(msg), "Hush: a kernel's bounded wait gave up (error word 0x%x)", w);
    return hush_fail(h, HUSH_ERR_KERNEL, msg);
  }
  return HUSH_OK;
}

// A wait that runs out: one thread waits on an mbarrier nothing arrives at, `polls` times, then sets bit 4 of the
// error word and returns, as every bounded wait in the kernels does.
__global__ void k_wait_selftest(unsigned *err, uint32_t polls) {
  __shared__ alignas(8) uint64_t mbar;
  const uint32_t a = umma::smem_u32(&mbar);
  umma::mbar_init(a, 1);
  if (!umma::mbar_wait_bounded(a, 0, polls)) atomicOr(err, 4u);
}

extern "C" int hush_selftest_wait(hush_t *h, uint32_t polls, void *stream) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_selftest_wait: NULL instance");
  cudaSetDevice(h->dev);
  k_wait_selftest<<<1, 1, 0, (cudaStream_t)stream>>>(h->err, polls);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HUSH_OK : hush_cuda_fail(h, e, "hush_selftest_wait");
}

extern "C" int hush_end_frame(hush_t *h) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_end_frame: NULL instance");
  h->last_out = h->taa[h->frame & 1];
  h->reset = false;
  h->frame++;
  return HUSH_OK;
}

extern "C" int hush_buffer(hush_t *h, int id, void **dptr, int *width, int *height, int *texel_bytes) {
  if (!h) return hush_fail(nullptr, HUSH_ERR_ARG, "hush_buffer: NULL instance");
  void *p = nullptr;
  int w = h->W, hh = h->H, tb = 8;
  switch (id) {
    case HUSH_BUF_A0: p = h->A0; break;
    case HUSH_BUF_X: p = h->X; break;
    case HUSH_BUF_BH0: p = h->Bh[0]; w = h->W2; hh = h->H2; break;
    case HUSH_BUF_BH1: p = h->Bh[1]; w = h->W2; hh = h->H2; break;
    case HUSH_BUF_MOM0: p = h->mom[0]; break;
    case HUSH_BUF_MOM1: p = h->mom[1]; break;
    case HUSH_BUF_KEY0: p = h->key[0]; break;
    case HUSH_BUF_KEY1: p = h->key[1]; break;
    case HUSH_BUF_HIST0: p = h->hist[0]; break;
    case HUSH_BUF_HIST1: p = h->hist[1]; break;
    case HUSH_BUF_TAA0: p = h->taa[0]; break;
    case HUSH_BUF_TAA1: p = h->taa[1]; break;
    case HUSH_BUF_PAR0_0: p = h->par0[0]; w = h->W2; hh = h->H2; break;
    case HUSH_BUF_PAR0_1: p = h->par0[1]; w = h->W2; hh = h->H2; break;
    case HUSH_BUF_PAR1: p = h->par1; w = h->W2; hh = h->H2; break;
    case HUSH_BUF_PAR2: p = h->par2; w = h->W2; hh = h->H2; break;
    case HUSH_BUF_F0: case HUSH_BUF_F1: case HUSH_BUF_F2: case HUSH_BUF_F3:
      p = h->F[id - HUSH_BUF_F0]; w = h->W2; hh = h->H2; tb = 16; break;
    case HUSH_BUF_C0: p = h->C[0]; w = h->W4; hh = h->H4; break;
    case HUSH_BUF_C1: p = h->C[1]; w = h->W4; hh = h->H4; break;
    case HUSH_BUF_CG: p = h->CG; w = h->W4; hh = h->H4; break;
    default: return hush_fail(h, HUSH_ERR_ARG, "hush_buffer: bad buffer id");
  }
  if (dptr) *dptr = p;
  if (width) *width = w;
  if (height) *height = hh;
  if (texel_bytes) *texel_bytes = tb;
  return HUSH_OK;
}
