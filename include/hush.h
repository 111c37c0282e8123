/* hush_b200: C ABI of the B200-native Hush denoiser (and its SVGF baseline).
 *
 * The drop-in boundary for the reference's `Hush` / `SVGF` JavaScript classes (src/index.d.ts:36-83). Device
 * buffers replace GPUTextures: every image is rgba16float, i.e. 4 x f16 = 8 bytes per texel, row-major, with a row
 * pitch in bytes (0 = dense, width * 8). The WebGPU command encoder is replaced by a CUDA stream (`void *` holding a
 * cudaStream_t; NULL = the default stream). Calls are stream-ordered and not thread-safe per instance.
 *
 * Every call returns HUSH_OK (0) or an error code; the message (same text as the reference's thrown Error) is
 * available from hush_last_error(instance) or, for calls without an instance, hush_global_error().
 */
#ifndef HUSH_B200_H
#define HUSH_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HUSH_OK 0
#define HUSH_ERR_ARG 1      /* bad argument: missing input, size mismatch, bad weights, bad size */
#define HUSH_ERR_DEVICE 2   /* device lacks a required capability (the reference's requiredLimits check) */
#define HUSH_ERR_CUDA 3     /* a CUDA runtime call failed */
#define HUSH_ERR_KERNEL 4   /* a kernel reported an error word (e.g. a bounded wait that gave up) */

typedef struct hush_s hush_t;
typedef struct svgf_s svgf_t;

/* MLP arithmetic. FP32 is the reference's default form (f32 chain, hush.js:683-704); BF16 / F16 run the three
 * layers as tcgen05 tensor-core MMAs with FP32 accumulation on split-precision operands (each operand as a rounded
 * hi part plus its rounded residual, so f16 inputs and weights stay exact); HALF is the reference's `f16` option
 * (hush.js:683-703, 740): f16 products and f16 running sums in the WGSL's order. */
enum { HUSH_MLP_FP32 = 0, HUSH_MLP_BF16 = 1, HUSH_MLP_F16 = 2, HUSH_MLP_HALF = 3 };

/* Kernel schedule: FUSED (default) = the B200 frame (fused temporal+features+MLP, half-res pyramid, fine+final+TAA);
 * PASSES = one kernel per reference dispatch (hush.js:858-870). Both give the same results. */
enum { HUSH_SCHED_FUSED = 0, HUSH_SCHED_PASSES = 1 };

/* Constructor options: replaces HushOptions (src/index.d.ts:19-29, hush.js:728-732). */
typedef struct {
  int width, height;
  float exposure;            /* default 1 when the descriptor comes from hush_desc_default() */
  const uint16_t *weights;   /* f16 blob W1 b1 W2 b2 W3 b3 (hush.js:20-21); NULL = built-in weights */
  size_t n_weights;          /* number of f16 values; the MLP width follows (hiddenOf) */
  int f16;                   /* reference option `f16` (hush.js:740): selects HUSH_MLP_HALF when mlp_mode is FP32 */
  int mlp_mode;              /* HUSH_MLP_* */
  int schedule;              /* HUSH_SCHED_* */
  int device;                /* CUDA device ordinal; -1 = current device */
} hush_desc;

/* Frame inputs: replaces HushInputs (src/index.d.ts:11-17). Device pointers to rgba16float images.
 * width/height are the sizes of the images (checked against the denoiser's, hush.js:814-820); 0 = trust the
 * caller. pitch is the row pitch in bytes, 0 = dense. */
typedef struct {
  const void *radiance, *normal_depth, *motion, *material, *emission;
  int width[5], height[5];
  size_t pitch[5];
} hush_inputs;

/* Per-pass GPU time of the last denoise(), like the reference's timer hook (hush.js:842-851, gpu.js:25-77). */
typedef struct {
  const char *label;
  float ms;
} hush_timing;

/* hiddenOf (hush.js:22-25): hidden width h for n f16 weights (n = h^2 + 34 h + 12), 0 if none fits. */
int hush_hidden_of(long n);

/* Defaults for hush_desc (exposure 1, built-in weights, FP32 MLP, fused schedule, current device). */
hush_desc hush_desc_default(int width, int height);

/* Hush.requiredLimits (hush.js:721, 726): compute capability and dynamic shared memory the kernels need. */
void hush_required_limits(int *cc_major, int *cc_minor, size_t *shared_bytes);

/* new Hush(device, options) (hush.js:731-761). */
int hush_create(const hush_desc *desc, hush_t **out);
/* destroy() (hush.js:803-807). */
void hush_destroy(hush_t *h);
/* resize(width, height) (hush.js:764-794): reallocates when the size changes and resets the history. */
int hush_resize(hush_t *h, int width, int height);
/* reset() (hush.js:801): the next frame starts without history. */
int hush_reset(hush_t *h);
/* exposure property (hush.js:739, read per frame at 828). */
int hush_set_exposure(hush_t *h, float exposure);
float hush_get_exposure(const hush_t *h);
/* Replaces the MLP weights (same blob format as the constructor option). */
int hush_set_weights(hush_t *h, const uint16_t *weights, size_t n);
/* HUSH_MLP_*: the tensor-core forms run in the fused schedule's stage 0; the pass-by-pass schedule's INFER always
 * computes the reference's FP32 form. */
int hush_set_mlp_mode(hush_t *h, int mode);
int hush_set_schedule(hush_t *h, int schedule);
int hush_get_size(const hush_t *h, int *width, int *height);
int hush_get_hidden(const hush_t *h);
int hush_get_frame(const hush_t *h);

/* denoise(encoder, inputs, timer) (hush.js:813-822, encode 835-874): enqueues one frame on `stream` and returns
 * (in *out) the instance-owned output image (rgba16float, dense, linear HDR, alpha 1). Two images alternate from
 * frame to frame: the pointer stays valid until the next-but-one call (hush.js:796-798). In the fused schedule part
 * of the frame (the coarse levels) runs on a stream the instance owns, forked from `stream` and joined back into it
 * within the frame by events, so the frame as a whole stays ordered on `stream` (also inside a stream capture). */
int hush_denoise(hush_t *h, const hush_inputs *in, void *stream, const void **out);
/* denoise with the G-buffer in host memory (a CPU renderer, a replayed capture): the five inputs (rgba16float,
 * `pitch` in bytes, pinned host memory for truly asynchronous copies) are copied into one of two instance-owned
 * device staging sets on a copy-in stream, the frame runs on `stream`, and the output is copied to out_host
 * (W x H rgba16float, out_pitch bytes, 0 = dense) on a copy-out stream. Consecutive calls overlap: frame t + 1's
 * input copies and frame t - 1's output copy run during frame t's kernels. The call only enqueues; out_host is
 * valid once hush_host_join's stream (or the device) has synchronised. No counterpart in the reference (its inputs
 * are GPU textures); it is the host-buffer form of Hush.denoise. */
int hush_denoise_host(hush_t *h, const hush_inputs *in, void *out_host, size_t out_pitch, void *stream);
/* `stream` waits for every output copy hush_denoise_host has enqueued. */
int hush_host_join(hush_t *h, void *stream);
/* output getter (hush.js:798): the last frame's output image. */
const void *hush_output(const hush_t *h);

/* Timer (hush.js:842-851): mode 0 off, 1 per pass, 2 whole frame as one span. hush_timer_read synchronises on
 * the recorded events and fills up to max entries; returns the number filled (or -1 on error). */
int hush_timer_enable(hush_t *h, int mode);
int hush_timer_read(hush_t *h, hush_timing *out, int max);

/* CUDA-graph replay of whole frames (config-5 style), one executable graph per ping-pong parity: new input pointers
 * rewrite the kernels' frame parameter in place; a change of the reset flag or the exposure captures the frame again. */
int hush_set_graph(hush_t *h, int enable);

/* The kernels' error word: a bounded wait that gave up (tensor-core MLP of stage 0: bit 0; the trainer's tensor-core
 * MLP: bit 1; hush_selftest_wait: bit 2; a TMA halo-tile copy of the a-trous stages: bit 3) sets a bit instead of
 * hanging. Reads the word into *word (may be NULL),
 * synchronising the device, clears it, and returns HUSH_ERR_KERNEL with a message if any bit was set. */
int hush_kernel_status(hush_t *h, unsigned *word);
/* Enqueues one thread that waits `polls` times on a barrier nothing arrives at and then sets bit 2 of the error
 * word: the failure path of every bounded wait, exercised without a fault. No counterpart in the reference. */
int hush_selftest_wait(hush_t *h, uint32_t polls, void *stream);

/* Last error message of the instance / of the calling thread (for hush_create failures). */
const char *hush_last_error(const hush_t *h);
const char *hush_global_error(void);

/* ---- pass-level interface (tests, adjoint checks) ------------------------------------------------------------
 * Pass ids follow the reference's dispatch order (hush.js:858-870). hush_run_pass runs one reference pass on the
 * instance's state for the current frame (ping-pong by frame parity, hush.js:837); hush_end_frame does the frame++
 * and history-reset bookkeeping (hush.js:871-872). */
enum {
  HUSH_PASS_TEMPORAL = 0, HUSH_PASS_INFER, HUSH_PASS_MID2, HUSH_PASS_MID3, HUSH_PASS_COARSE1, HUSH_PASS_COARSE2,
  HUSH_PASS_FINE_FINAL, HUSH_PASS_TAA, HUSH_PASS_COUNT
};
/* State images (hush.js:783-793). F0..F3 are 16-byte texels (8 x f16); the rest 8-byte texels (4 x f16). */
enum {
  HUSH_BUF_A0 = 0, HUSH_BUF_X, HUSH_BUF_BH0, HUSH_BUF_BH1, HUSH_BUF_MOM0, HUSH_BUF_MOM1, HUSH_BUF_KEY0,
  HUSH_BUF_KEY1, HUSH_BUF_HIST0, HUSH_BUF_HIST1, HUSH_BUF_TAA0, HUSH_BUF_TAA1, HUSH_BUF_PAR0_0, HUSH_BUF_PAR0_1,
  HUSH_BUF_PAR1, HUSH_BUF_PAR2, HUSH_BUF_F0, HUSH_BUF_F1, HUSH_BUF_F2, HUSH_BUF_F3, HUSH_BUF_C0, HUSH_BUF_C1,
  HUSH_BUF_CG, HUSH_BUF_COUNT
};
int hush_run_pass(hush_t *h, int pass, const hush_inputs *in, void *stream);
int hush_end_frame(hush_t *h);
/* Device pointer and geometry of a state image. */
int hush_buffer(hush_t *h, int id, void **dptr, int *width, int *height, int *texel_bytes);

/* ---- training twin: forward / adjoint of the frame for on-device training of the parameter MLP --------------------
 * No reference counterpart as an API: the reference's weights were trained offline by a PyTorch copy of the passes
 * that it does not ship (README.md:137, hush.js:6-7). The twin runs the frame after TEMPORAL in FP32 without f16
 * storage rounding; the loss is relative L1 of the TAA output against the noise-free image (clipped at 1 per value)
 * plus lambda times the same on frame differences. Gradients are exact for one frame with the temporal history held fixed; frames of a
 * window accumulate (truncated backpropagation through time). Trainers are tied to one Hush instance (h = 16). */
typedef struct hush_trainer_s hush_trainer_t;
/* theta: 812 FP32 initial weights (W1 b1 W2 b2 W3 b3), NULL = the instance's current weights. */
int hush_trainer_create(hush_t *h, const float *theta, hush_trainer_t **out);
void hush_trainer_destroy(hush_trainer_t *t);
/* One frame: TEMPORAL + coarse passes, twin forward, loss (in *loss_out, synchronising), and if backward != 0 the
 * adjoint added to the weight gradient. clean / clean_prev: dense f32 rgb device images (clean_prev may be NULL).
 * Does not advance the frame, so repeated calls see the same history. */
int hush_trainer_frame(hush_trainer_t *t, const hush_inputs *in, const float *clean, const float *clean_prev,
                       float lambda_t, int backward, void *stream, double *loss_out);
int hush_trainer_end_frame(hush_trainer_t *t);
/* Sum of the frame losses since the previous call (synchronises `stream`, then restarts the sum). */
int hush_trainer_loss_sum(hush_trainer_t *t, void *stream, double *out);
int hush_trainer_reset(hush_trainer_t *t);
int hush_trainer_zero_grad(hush_trainer_t *t, void *stream);
/* The accumulated weight gradient (812 doubles). */
int hush_trainer_grad(hush_trainer_t *t, double *out);
/* Device addresses of the gradient accumulator (812 doubles) and of the loss sum (1 double), valid until
 * hush_trainer_destroy. Data-parallel training all-reduces both in place (e.g. NCCL, on the trainer's stream) between
 * the last hush_trainer_frame of a step and hush_trainer_step. Either pointer may be NULL. */
int hush_trainer_accumulators(hush_trainer_t *t, double **grad, double **loss_sum);
/* Read (get != NULL) and / or replace (set != NULL) the FP32 master weights. */
int hush_trainer_theta(hush_trainer_t *t, float *get, const float *set);
/* The FP32 parameters and dL/dpar of the last frame: 12 floats per half-res pixel (alpha gamma beta kappa, s0..s3,
 * c0..c3). Either pointer may be NULL. */
int hush_trainer_par(hush_trainer_t *t, float *par, float *dpar);
/* The FP32 TAA output of the last frame (rgba, W x H). */
int hush_trainer_output(hush_trainer_t *t, float *out);
/* Adam on the accumulated gradient (clipped to global norm `clip` if > 0), then zero it; *grad_norm = its norm. */
int hush_trainer_step(hush_trainer_t *t, float lr, float beta1, float beta2, float eps, float clip, void *stream,
                      double *grad_norm);
/* Round the master weights to the f16 blob, install it in the denoiser and copy it to blob (if not NULL). */
int hush_trainer_export(hush_trainer_t *t, uint16_t *blob);
/* Arithmetic of the twin's MLP forward and adjoint: HUSH_MLP_FP32 (default; per-thread FP32, the form the gradient
 * checks hold to 1e-3) or HUSH_MLP_BF16 / HUSH_MLP_F16: tcgen05 GEMM tiles on bf16 / f16 operands with FP32
 * accumulation (the three layers, the delta products and the weight gradient as one 128 x 64 x 128 product per CTA),
 * FP32 master weights, bias / ReLU / heads in FP32. A bounded wait that gives up sets bit 1 of the instance's kernel
 * error word. */
int hush_trainer_set_mlp(hush_trainer_t *t, int mode);

/* One optimiser step over a batch, as a one-GPU training loop runs it: for each of n_windows windows of n_frames
 * frames (frames[] and cleans[] window-major; cleans[] holds device pointers to dense f32 rgb images) a history
 * reset, then per frame hush_trainer_frame with backward (clean_prev = the window's previous frame from its second
 * frame on) and hush_trainer_end_frame; then hush_trainer_step. *loss_mean = the mean frame loss of the batch (the
 * loss sum is restarted first). Synchronises `stream`. Data-parallel callers all-reduce between the frames and the
 * step instead (hush_trainer_accumulators). */
int hush_train_step(hush_trainer_t *t, const hush_inputs *frames, const float *const *cleans, int n_windows,
                    int n_frames, float lambda_t, float lr, float beta1, float beta2, float eps, float clip,
                    void *stream, double *loss_mean, double *grad_norm);

/* The training windows of the analytic scene generator (hush_scene_frame_device, declared below), without a
 * host round trip per frame: for each of n_windows seeds, the n_frames frames of scene *sc with that seed are
 * generated on the device into trainer-owned buffers (allocated on first use) and run as hush_train_step runs a
 * window (history reset, then per frame forward + backward with the temporal term from the second frame on, and
 * end-of-frame). Adds into the gradient and loss accumulators; no optimiser step (the caller all-reduces across ranks
 * if it trains data-parallel, then calls hush_trainer_step). sc's size must be the trainer's. Up to eight windows run
 * concurrently on lanes forked from and joined back to `stream` (helper trainers on private Hush instances, created
 * on first use, own history and accumulators, summed into this trainer's in lane order); each window's training
 * frames replay as a cached CUDA graph. The trainer's own Hush instance ends in the state of the windows it ran. */
struct hush_scene_s;
int hush_trainer_windows(hush_trainer_t *t, const struct hush_scene_s *sc, const uint32_t *seeds, int n_windows,
                         int n_frames, float lambda_t, void *stream);

/* ---- the twin's passes as forward / adjoint pairs -----------------------------------------------------------------
 * Each pass of the twin on its own, for gradient checks and for hosts that schedule the passes themselves. The
 * reference's passes (hush.js:835-874) map as: INFER = MLP + MID1, mid2 / mid3 = MID2 / MID3, FINE_FINAL = FINE,
 * TAA = TAA; TEMPORAL and the coarse levels run in hush_trainer_begin (their outputs do not depend on the weights).
 * hush_trainer_begin fixes the frame: the inputs must stay valid until its last pass call, and hush_trainer_end_frame
 * or hush_trainer_reset ends it. A forward pass overwrites its outputs. An adjoint pass ADDS into the gradients of its
 * inputs (hush_trainer_zero_adjoints clears dX, dOUT, dPAR and dB1..dB3), except the loss adjoint, which sets dOUT;
 * the MLP adjoint adds dL/dtheta into the weight-gradient accumulator (GRAD). Adjoints recompute what they need from
 * the pass's inputs (the a-trous weights included) and need the pass's forward inputs in place, not its outputs.
 * Running LOSS, TAA, FINE, MID3, MID2, MID1, MLP backward after the forward chain gives hush_trainer_frame's
 * gradient. */
typedef enum {
  HUSH_TWIN_MLP = 0, /* theta, features F0..F2, guide F3        -> PAR      | dPAR -> GRAD                     */
  HUSH_TWIN_MID1 = 1, /* block means (F2), guide, PAR            -> B1       | dB1  -> dPAR (s1, c1)            */
  HUSH_TWIN_MID2 = 2, /* B1, guide, PAR                          -> B2       | dB2  -> dB1, dPAR (s2, c2)       */
  HUSH_TWIN_MID3 = 3, /* B2, guide, PAR                          -> B3       | dB3  -> dB2, dPAR (s3, c3)       */
  HUSH_TWIN_FINE = 4, /* A0, key, PAR, B3, C0, CG, G-buffer      -> A1, X    | dX   -> dB3, dPAR (s0 c0 beta kappa) */
  HUSH_TWIN_TAA = 5,  /* X, motion, previous TAA output          -> OUT      | dOUT -> dX                       */
  HUSH_TWIN_LOSS = 6, /* OUT, clean, clean_prev, OUT_PREV        -> LOSS     | 1    -> dOUT                     */
  HUSH_TWIN_TEMPORAL = 7, /* G-buffer, previous history (colour, moments, key, par0) -> A0, moments, key, features |
                           * dA0, dMOM -> dHIST, dMOM_PREV, dAG (the previous frame's colour, moments, alpha / gamma) */
  HUSH_TWIN_COARSE1 = 8, /* AH (block means), counts (F3), coarse guide CG -> C1 | dC1 -> dAH                   */
  HUSH_TWIN_COARSE2 = 9, /* C1, coarse guide CG                            -> C0 | dC0 -> dC1                   */
  HUSH_TWIN_PASSES = 10
} hush_twin_pass;

/* The trainer's buffers (device memory owned by the trainer, valid until hush_trainer_destroy; OUT / OUT_PREV swap at
 * hush_trainer_end_frame). Element types: THETA f32, GRAD and LOSS f64, the rest f32. */
typedef enum {
  HUSH_TB_THETA = 0,    /* 812 x 1 x 1: FP32 master weights (W1 b1 W2 b2 W3 b3)                      */
  HUSH_TB_GRAD = 1,     /* 812 x 1 x 1: weight-gradient accumulator                                  */
  HUSH_TB_LOSS = 2,     /* 1 x 1 x 1: the last loss                                                  */
  HUSH_TB_PAR = 3,      /* W2 x H2 x 12: alpha gamma beta kappa, s0..s3, c0..c3 per half-res pixel   */
  HUSH_TB_DPAR = 4,     /* W2 x H2 x 12                                                              */
  HUSH_TB_B1 = 5, HUSH_TB_B2 = 6, HUSH_TB_B3 = 7,     /* W2 x H2 x 4: mid levels (rgb, variance)      */
  HUSH_TB_DB1 = 8, HUSH_TB_DB2 = 9, HUSH_TB_DB3 = 10, /* W2 x H2 x 4                                 */
  HUSH_TB_A1 = 11,      /* W x H x 4: fine level                                                     */
  HUSH_TB_X = 12,       /* W x H x 4: recombined colour (the TAA input)                              */
  HUSH_TB_DX = 13,      /* W x H x 4                                                                 */
  HUSH_TB_OUT = 14,     /* W x H x 4: TAA output of this frame                                       */
  HUSH_TB_OUT_PREV = 15, /* W x H x 4: TAA output of the previous frame (the temporal loss term)     */
  HUSH_TB_DOUT = 16,    /* W x H x 4                                                                 */
  HUSH_TB_DA0 = 17,     /* W x H x 4: dL/d TEMPORAL's colour + variance (the fine adjoint adds into it) */
  HUSH_TB_DA1 = 18,     /* W x H x 4: dL/d the fine level through the colour history (a fine seed)    */
  HUSH_TB_DMOM = 19,    /* W x H x 4: dL/d this frame's moments (a TEMPORAL seed)                     */
  HUSH_TB_DHIST = 20,   /* W x H x 4: dL/d the previous frame's colour history (TEMPORAL adds into it) */
  HUSH_TB_DMOM_PREV = 21, /* W x H x 4: dL/d the previous frame's moments                             */
  HUSH_TB_DAG = 22,     /* W2 x H2 x 2: dL/d the previous frame's alpha, gamma per half-res pixel     */
  HUSH_TB_AH = 23,      /* W2 x H2 x 4: COARSE1's input, the block means (F2.zw) as FP32              */
  HUSH_TB_DAH = 24,     /* W2 x H2 x 4                                                               */
  HUSH_TB_C1 = 25,      /* W4 x H4 x 4: coarse level 1 (COARSE1's output, coarse2's input), FP32      */
  HUSH_TB_DC1 = 26,     /* W4 x H4 x 4                                                               */
  HUSH_TB_C0 = 27,      /* W4 x H4 x 4: coarse level 2 (coarse2's output), FP32                       */
  HUSH_TB_DC0 = 28,     /* W4 x H4 x 4                                                               */
  HUSH_TB_COUNT = 29
} hush_trainer_buf;

/* TEMPORAL and the coarse levels for the frame's inputs, and the frame context for the pass calls (clean: dense f32
 * rgb, required; clean_prev may be NULL). */
int hush_trainer_begin(hush_trainer_t *t, const hush_inputs *in, const float *clean, const float *clean_prev,
                       float lambda_t, void *stream);
int hush_trainer_zero_adjoints(hush_trainer_t *t, void *stream);
int hush_trainer_buffer(hush_trainer_t *t, int which, void **ptr, int *width, int *height, int *channels);
/* pass: a hush_twin_pass; backward != 0 runs its adjoint. The named pairs below are the same calls. */
int hush_trainer_pass(hush_trainer_t *t, int pass, int backward, void *stream);
int hush_mlp_fwd(hush_trainer_t *t, void *stream);
int hush_mlp_bwd(hush_trainer_t *t, void *stream);
int hush_mid1_fwd(hush_trainer_t *t, void *stream);
int hush_mid1_bwd(hush_trainer_t *t, void *stream);
int hush_mid2_fwd(hush_trainer_t *t, void *stream);
int hush_mid2_bwd(hush_trainer_t *t, void *stream);
int hush_mid3_fwd(hush_trainer_t *t, void *stream);
int hush_mid3_bwd(hush_trainer_t *t, void *stream);
int hush_fine_fwd(hush_trainer_t *t, void *stream);
int hush_fine_bwd(hush_trainer_t *t, void *stream);
int hush_taa_fwd(hush_trainer_t *t, void *stream);
int hush_taa_bwd(hush_trainer_t *t, void *stream);
int hush_loss_fwd(hush_trainer_t *t, void *stream);
int hush_loss_bwd(hush_trainer_t *t, void *stream);
/* TEMPORAL (hush.js:111-223) as a pass: the forward reruns the reference pass on the begun frame; the adjoint takes
 * dA0 and dMOM (the gradients of TEMPORAL's colour + variance and moments) back through the anti-lag clamp, the blend
 * a = max(alpha, 1 / len), the moment updates, the variance lerp and the bilinear (or 3x3 fallback) reprojection,
 * ADDING into dHIST, dMOM_PREV and dAG. The f16 storage of the history counts as the identity; the lag metric and the
 * block features are not differentiated (the MLP's inputs are held fixed). */
int hush_temporal_fwd(hush_trainer_t *t, void *stream);
int hush_temporal_bwd(hush_trainer_t *t, void *stream);
/* COARSE1 (hush.js:372-421: down() of the block means weighted by their pixel counts, then the 5x5 a-trous with
 * step 1) and coarse2 (hush.js:752: the 5x5 a-trous with step 2), both with the variance prefilter, s = COARSE_S and
 * c = 1, in FP32 over the trainer's AH / C1 / C0 (hush_trainer_begin fills AH from the frame's F2.zw). The levels have
 * no learnable input; each adjoint ADDS dL/d(its input level) (dAH, dC1) from dL/d(its output level) (dC1, dC0):
 * the direct taps, every tap's and the centre's luminance edge-stopping term, and the prefiltered variance through
 * s / sd. The guide (the coarse guide CG, normals and depths) is geometry and carries no gradient. */
int hush_coarse1_fwd(hush_trainer_t *t, void *stream);
int hush_coarse1_bwd(hush_trainer_t *t, void *stream);
int hush_coarse2_fwd(hush_trainer_t *t, void *stream);
int hush_coarse2_bwd(hush_trainer_t *t, void *stream);

/* Backpropagation through time over one window of n_frames frames (frames[] / cleans[] as in hush_train_step): the
 * window starts without history, every frame runs forward with its state kept, then the frames run backward from the
 * last one. Besides each frame's own loss gradient (what hush_trainer_frame takes), the gradient flows across frames
 * through TEMPORAL (hush_temporal_bwd): from a frame's colour + variance A0 and moments into the previous frame's
 * colour history (its fine level), moments and alpha / gamma, so the alpha and gamma heads of the MLP train. A0
 * reaches the loss directly (the fine level) and through the block means (block(), hush.js:241-244), which feed mid1,
 * the recombination and the coarse levels COARSE1 / coarse2; both paths are followed. The block features and the TAA
 * history are held fixed (truncated there). Adds into the gradient and loss accumulators,
 * like hush_trainer_windows; allocates the window's per-frame records (about 11 MB per frame at 384 x 384) on first
 * use. The trainer's own Hush history is not touched. */
int hush_trainer_window_bptt(hush_trainer_t *t, const hush_inputs *frames, const float *const *cleans, int n_frames,
                             float lambda_t, void *stream);

/* hush_trainer_window_bptt over the training windows of the analytic scene generator, as hush_trainer_windows runs
 * them: for each of n_windows seeds the n_frames frames of *sc are generated on the device into trainer-owned buffers
 * and the window runs forward and backward through time. Up to eight windows run concurrently on the same lanes
 * (each lane its own records), summed into this trainer's accumulators in lane order; each window's forward + reverse
 * sweep replays as a cached CUDA graph. No optimiser step; sc's size must be the trainer's. The trainer's own Hush
 * history is not touched. */
int hush_trainer_windows_bptt(hush_trainer_t *t, const struct hush_scene_s *sc, const uint32_t *seeds, int n_windows,
                              int n_frames, float lambda_t, void *stream);

/* Weight gradient of the parameter MLP (812 doubles in dtheta, overwritten) from a half-resolution image of rows:
 * packed features F0..F3 (16-byte texels, width2 x height2, as hush_buffer returns them), dL/dpar (12 floats per
 * row, as hush_trainer_par lays them out, all 12 channels honoured) and FP32 weights theta (812). The same
 * computation as hush_mlp_bwd's weight gradient, but it allocates nothing: no counterpart in the reference. It
 * exists for callers that cannot allocate device memory after start-up (a render or training loop with a fixed
 * memory budget, where an allocation would synchronise the device or fail mid-frame) or that only lend the library
 * buffers they own. Rows are summed in FP32 over chunks of 64 and the chunks in FP64, so the rounding error stays
 * that of a 64-row FP32 sum at every size. Its scratch is a fixed 3.33 MB device array (512 FP64 partial sums) that
 * every GPU loading the library holds until exit;
 * at most 16,777,216 rows (4096 x 4096) are accepted, larger sizes fail with HUSH_ERR_ARG. The first call on a device
 * looks up that array's device address, so make it before any stream capture. Calls share the array: calls that
 * overlap on the GPU (different streams, or different threads) race. Errors: hush_global_error(). */
int hush_mlp_grad_noalloc(const void *F0, const void *F1, const void *F2, const void *F3, const float *dpar,
                          const float *theta, int width2, int height2, double *dtheta, void *stream);

/* ---- SVGF baseline (src/denoise/svgf.js) ---------------------------------------------------------------------- */
/* SVGFOptions (src/index.d.ts:63-72, svgf.js:278-281). iterations must be 1..5 (the reference's uniform array
 * holds 5 a-trous iterations, svgf.js:294). */
typedef struct {
  int iterations;
  float sigma_l, sigma_n, sigma_z, alpha_color, alpha_moments, taa_alpha;
  int taa;
} svgf_options;
/* Inputs: HushInputs plus last frame's normalDepth / motion (svgf.js:341). */
typedef struct {
  const void *radiance, *normal_depth, *motion, *material, *emission, *prev_normal_depth, *prev_motion;
  size_t pitch[7];
} svgf_inputs;

svgf_options svgf_options_default(void);
/* new SVGF(device, width, height, options) (svgf.js:273-300). */
int svgf_create(int width, int height, const svgf_options *opts, int device, svgf_t **out);
void svgf_destroy(svgf_t *s);
int svgf_resize(svgf_t *s, int width, int height);
int svgf_reset(svgf_t *s);
/* encode(encoder, inputs) (svgf.js:343-378): one frame; *out = this frame's output image. */
int svgf_encode(svgf_t *s, const svgf_inputs *in, void *stream, const void **out);
const void *svgf_output(const svgf_t *s);
const char *svgf_last_error(const svgf_t *s);

/* ---- path tracer (src/pt): scene buffers, BVH, 1 spp + G-buffer frames -----------------------------------------
 * SceneGPU (src/pt/scene.js:22-344) without three.js: meshes arrive as world-space arrays grouped into at most 8
 * BLAS (group flags: dynamic = re-posed by hush_pt_scene_update with exact previous positions, no shadow = skipped by
 * shadow rays). PathTracer (src/pt/pathtracer.js:14-162): two G-buffer slots of five dense rgba16float images
 * (radiance, normalDepth, motion, material, emission: exactly the Hush inputs) or a float4 accumulation buffer. */
#define HUSH_PT_MAX_BLAS 8
#define HUSH_PT_MAX_LIGHTS 8
#define HUSH_PT_TEX_SIZE 1024
#define HUSH_PT_TEX_MIPS 11
#define HUSH_PT_ENV_GW 256
#define HUSH_PT_ENV_GH 128
#define HUSH_PT_GROUP_DYNAMIC 1
#define HUSH_PT_GROUP_NO_SHADOW 2
typedef struct hush_pt_scene_s hush_pt_scene_t;
typedef struct hush_pt_s hush_pt_t;
/* Material record in the reference's GPU layout (scene.js:50-56, 305-310): base rgb + alpha cutoff, emissive rgb,
 * (roughness, metalness, transmission, ior), texture layers (base, normal, arm; -1 = none), (uv scale xy, normal
 * scale, 0). */
typedef struct {
  float base[4], emissive[4], pbr[4];
  int32_t tex[4];
  float uv[4];
} hush_pt_material;
typedef struct { uint32_t node_offset, tri_offset, node_count, flags; } hush_pt_blas;
typedef struct { float pos[4], prev_pos[4], radiance[4], params[4]; } hush_pt_light; /* params.x: 0 sun, 1 sphere */
/* Frame uniforms, the 960-byte layout of the reference's uniform buffer (pathtracer.wgsl.js:22-46, written by
 * writeUniforms, pathtracer.js:105-149); matrices column-major. */
typedef struct {
  float cam_pos[4], cam_right[4], cam_up[4], cam_fwd[4];
  float view_proj[16], prev_view_proj[16];
  uint32_t size[2], frame, mode;
  float jitter[2];
  uint32_t spp, max_bounces;
  float sky_zenith[4], sky_horizon[4], ground[4];
  uint32_t counts[4];
  float clamp_lum, pixel_angle, shadow_tau, clamp_direct;
  float env[4];
  hush_pt_blas blas[HUSH_PT_MAX_BLAS];
  hush_pt_light lights[HUSH_PT_MAX_LIGHTS];
} hush_pt_frame;

hush_pt_material hush_pt_material_default(void);
int hush_pt_scene_create(int device, hush_pt_scene_t **out);
void hush_pt_scene_destroy(hush_pt_scene_t *s);
/* Returns the material id (>= 0; it is also the object id the G-buffer reports) or -1. */
int hush_pt_scene_add_material(hush_pt_scene_t *s, const hush_pt_material *m);
/* rgba8 image (any size; resampled to 1024^2, 11 box-filtered mips); returns the texture layer or -1. */
int hush_pt_scene_add_texture(hush_pt_scene_t *s, const uint8_t *rgba, int width, int height);
/* One BLAS from world-space vertices (pos: 3 floats, nrm: 3 floats or NULL = +y, uv: 2 floats or NULL = 0) and
 * triangles (idx: 3 vertex indices, mat: material id per triangle). Returns the group id or -1. */
int hush_pt_scene_add_group(hush_pt_scene_t *s, int flags, const float *pos, const float *nrm, const float *uv,
                            int n_verts, const uint32_t *idx, const uint32_t *mat, int n_tris);
/* Builds every group's BVH (binned SAH, bvh.js:12-143), packs it (bvh.js:186-210) and uploads the scene. */
int hush_pt_scene_build(hush_pt_scene_t *s);
/* SceneGPU.update for one dynamic group (scene.js:225-270): the current positions become the previous ones, pos
 * (and nrm, or area-weighted smooth normals when NULL) become current, the BVH is refitted and re-uploaded. */
int hush_pt_scene_update(hush_pt_scene_t *s, int group, const float *pos, const float *nrm, void *stream);
/* The BLAS table for the frame uniforms (scene.js:338-343); returns the group count. */
int hush_pt_scene_blas(const hush_pt_scene_t *s, hush_pt_blas *out, int max);
/* Sizes and device buffers (packed nodes, triangles, triangle indices, vertices, materials) for inspection. */
int hush_pt_scene_info(const hush_pt_scene_t *s, int *tri_total, int *node_total, int *vert_total, int *max_depth);
int hush_pt_scene_device(const hush_pt_scene_t *s, const void **nodes, const void **tris, const void **tri_idx,
                         const void **verts, const void **mats, const void **tex);
/* The BVH builder alone (host; bvh.js:12-143): nodes (8 floats per node, room for 2 * max(1, n) nodes), order;
 * returns the node count. */
int hush_pt_bvh_build(const float *pos, int tri_count, float *nodes, uint32_t *order, int *max_depth);
/* prepareEnvMap (src/pt/envmap.js:85-105), host: cuts the sun out of rgba (w x h x 4 floats, row 0 = up; in place),
 * writes the rgba16float map (w x h x 4) and the alias table (256 x 128 cells x 4 floats); returns 1 when a sun was
 * cut (its direction and irradiance in sun_dir / sun_irr). */
int hush_pt_env_prepare(float *rgba, int width, int height, int sun, double sun_cone_deg, uint16_t *half_out,
                        float *table_out, double sun_dir[3], double sun_irr[3]);
/* JITTER (pathtracer.js:6-12): 16 Halton(2, 3) subpixel offsets in pixels, x y pairs. */
void hush_pt_jitter(float out[32]);

int hush_pt_create(hush_pt_scene_t *scene, int width, int height, hush_pt_t **out);
void hush_pt_destroy(hush_pt_t *p);
int hush_pt_resize(hush_pt_t *p, int width, int height);
/* The environment map (host rgba16float w x h and its alias table) or NULL to unbind (analytic sky). */
int hush_pt_set_envmap(hush_pt_t *p, const uint16_t *half_rgba, int width, int height, const float *table);
/* One dispatch (pathtracer.js:152-159): mode 0 writes G-buffer slot `slot`, mode 1 adds spp paths per pixel to the
 * accumulation buffer. f->size must equal the tracer's size. */
int hush_pt_encode(hush_pt_t *p, const hush_pt_frame *f, int slot, void *stream);
/* which: 0 radiance, 1 normalDepth, 2 motion, 3 material, 4 emission. */
const void *hush_pt_gbuffer(const hush_pt_t *p, int slot, int which);
float *hush_pt_accum(const hush_pt_t *p);
int hush_pt_clear_accum(hush_pt_t *p, void *stream);
const char *hush_pt_last_error(void);

/* ---- display post of the demo (src/demo/post.js) on a headless target ------------------------------------------
 * new Post(device, format, {bloom, vignette}) (post.js:137-156) and Post.encode (post.js:191-210): split-screen
 * composite of left | mid | right (linear HDR rgba16float, dense, width x height), six-level bloom, vignette, AgX,
 * sRGB and divider line. The canvas is replaced by a caller-owned device buffer of target_width x target_height
 * texels in `format` (the bloom / vignette strengths are instance state as in the reference). */
#define HUSH_POST_LEVELS 6
#define HUSH_POST_RGBA8 0   /* 4 x u8 unorm, r g b a */
#define HUSH_POST_BGRA8 1   /* 4 x u8 unorm, b g r a (the usual canvas format) */
#define HUSH_POST_RGBA32F 2 /* 4 x f32: the colour before 8-bit quantisation */
typedef struct hush_post_s hush_post_t;
typedef struct {
  int device, format;
  float bloom, vignette; /* defaults 0.03 and 0.35 (post.js:138) */
} hush_post_desc;
typedef struct {
  const void *left, *right, *mid; /* mid NULL = right (post.js:191) */
  int width, height;
  float split, split2, exposure, line; /* defaults 0.5, 0.5 (= split), 1, 1.5 */
  int same;                            /* 1: every third shows the middle third of its own image */
} hush_post_inputs;
hush_post_desc hush_post_desc_default(void);
hush_post_inputs hush_post_inputs_default(void);
int hush_post_create(const hush_post_desc *desc, hush_post_t **out);
void hush_post_destroy(hush_post_t *p);
int hush_post_set(hush_post_t *p, float bloom, float vignette);
/* Enqueues the 13 passes on `stream`; target_pitch in bytes (0 = dense). */
int hush_post_encode(hush_post_t *p, const hush_post_inputs *in, void *target, int target_width, int target_height,
                     size_t target_pitch, void *stream);
/* level 0: the composited HDR image; 1..6: the bloom levels as the last encode left them (rgba16float). */
const void *hush_post_buffer(const hush_post_t *p, int level, int *width, int *height);
const char *hush_post_last_error(const hush_post_t *p);

/* ---- synthetic G-buffer scenes (benchmark / test / training inputs) ------------------------------------------ */
typedef struct hush_scene_s {
  int width, height, n_objects, n_moving;
  float sky_frac, pan_min, pan_max, yaw_deg, firefly_rate, firefly_scale;
  int cut_frame;
  uint32_t seed;
} hush_scene;
/* One frame on the host: five dense rgba16float images (may be NULL) and the noise-free radiance + emission as
 * f32 rgb (may be NULL). */
int hush_scene_frame_host(const hush_scene *sc, int frame, uint16_t *radiance, uint16_t *normal_depth,
                          uint16_t *motion, uint16_t *material, uint16_t *emission, float *clean);
/* The same on the device, enqueued on `stream`. */
int hush_scene_frame_device(const hush_scene *sc, int frame, void *radiance, void *normal_depth, void *motion,
                            void *material, void *emission, void *clean, void *stream);

#ifdef __cplusplus
}
#endif
#endif
