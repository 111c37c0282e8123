/* CPU oracle for the Hush denoise path: TEST INFRASTRUCTURE ONLY.
 *
 * A scalar restatement of the reference's WGSL passes (src/denoise/hush.js:28-678, MLP order hush.js:681-704,
 * weight decoding hush.js:706-744) and of the SVGF baseline (src/denoise/svgf.js:12-271). It exists to check the
 * CUDA path: only the tests, the smoke check and the CPU-baseline leg of the benchmark load it. The product path
 * never calls it.
 *
 * Parity status: the reference ships no golden vectors, known-answer tests or fixtures for this path and cannot
 * run here (JavaScript + WGSL on WebGPU). The oracle is pinned only by invariants of the WGSL (known-answer tests in
 * tests/test_oracle_kat.py) and by the byte-exact weight blob: parity unpinned by reference outputs.
 *
 * Arithmetic: mode 0 ("ref") computes in f32 with the WGSL's operation order (no FMA contraction); mode 1 ("fp64")
 * computes in double. Both quantise at exactly the points where the WGSL writes an rgba16float / rgba32uint texture
 * (round toward zero to f16, hush.js:98-101) or applies qf16.
 *
 * Buffers are dense row-major rgba16float images (4 x u16 per texel); the packed feature textures F0..F3 are
 * 8 x u16 per texel (pack2x16float pairs, low half first).
 */
#ifndef HUSH_ORACLE_H
#define HUSH_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ho_hush ho_hush;
typedef struct ho_svgf ho_svgf;

/* Buffer ids, shared with the CUDA library's debug accessors (include/hush.h HUSH_BUF_*). */
enum {
  HO_BUF_A0 = 0, HO_BUF_X, HO_BUF_BH0, HO_BUF_BH1, HO_BUF_MOM0, HO_BUF_MOM1, HO_BUF_KEY0, HO_BUF_KEY1,
  HO_BUF_HIST0, HO_BUF_HIST1, HO_BUF_TAA0, HO_BUF_TAA1, HO_BUF_PAR0_0, HO_BUF_PAR0_1, HO_BUF_PAR1, HO_BUF_PAR2,
  HO_BUF_F0, HO_BUF_F1, HO_BUF_F2, HO_BUF_F3, HO_BUF_C0, HO_BUF_C1, HO_BUF_CG, HO_BUF_COUNT
};

/* Pass ids in the reference's dispatch order (hush.js:858-870). */
enum {
  HO_PASS_TEMPORAL = 0, HO_PASS_INFER, HO_PASS_MID2, HO_PASS_MID3, HO_PASS_COARSE1, HO_PASS_COARSE2,
  HO_PASS_FINE_FINAL, HO_PASS_TAA, HO_PASS_COUNT
};

/* Frame inputs: five dense rgba16float images of the instance's size. */
typedef struct {
  const uint16_t *radiance, *normal_depth, *motion, *material, *emission;
} ho_inputs;

int ho_hidden_of(long n);
ho_hush *ho_hush_create(int width, int height, float exposure, const uint16_t *weights, long n_weights, int fp64);
void ho_hush_destroy(ho_hush *h);
void ho_hush_reset(ho_hush *h);
void ho_hush_set_exposure(ho_hush *h, float e);
int ho_hush_frame(const ho_hush *h);
/* One full frame (all 8 passes), then frame++ and reset cleared; returns the output image (taa[cur]). */
const uint16_t *ho_hush_denoise(ho_hush *h, const ho_inputs *in);
/* One pass on the current frame's buffers; ho_hush_end_frame() does the frame++ / reset bookkeeping. */
int ho_hush_pass(ho_hush *h, int pass, const ho_inputs *in);
void ho_hush_end_frame(ho_hush *h);
/* Direct access to a state buffer (texels x channels u16), for pass-level tests. */
uint16_t *ho_hush_buffer(ho_hush *h, int id, int *w, int *hgt, int *channels);
/* Threads used by the row-parallel loops (OpenMP); 0 = all. */
void ho_set_threads(int n);

/* f16 helpers used by the tests. */
uint16_t ho_f2h_rz(float f);
float ho_h2f(uint16_t h);
float ho_qf16(float x);

/* MLP on one feature row (20 inputs) with f16 weights, outputs 12 raw values (mode 0 f32, 1 f64). */
void ho_mlp(const uint16_t *weights, long n_weights, const float *features, float *out, int fp64);

/* SVGF baseline (svgf.js). */
typedef struct {
  int iterations;
  float sigma_l, sigma_n, sigma_z, alpha_color, alpha_moments, taa_alpha;
  int taa;
} ho_svgf_opts;
typedef struct {
  const uint16_t *radiance, *normal_depth, *motion, *material, *emission, *prev_normal_depth, *prev_motion;
} ho_svgf_inputs;
ho_svgf *ho_svgf_create(int width, int height, const ho_svgf_opts *opts, int fp64);
void ho_svgf_destroy(ho_svgf *s);
void ho_svgf_reset(ho_svgf *s);
const uint16_t *ho_svgf_encode(ho_svgf *s, const ho_svgf_inputs *in);

/* ---- display post (src/demo/post.js), post_oracle.cpp ---------------------------------------------------------
 * Post.encode (post.js:191-210) over dense rgba16float images left / right / mid (mid NULL = right) of
 * width x height, into an out_width x out_height target. hdr_out (width x height x 4 u16), levels_out (the six bloom
 * levels, level 1 first, max(1, size >> i) each, 4 u16 per texel), out_f32 (the FINAL colour before 8-bit
 * quantisation) and out_rgba8 may each be NULL. */
#define HO_POST_LEVELS 6
typedef struct {
  const uint16_t *left, *right, *mid;
  int width, height, out_width, out_height;
  float split, split2, exposure, line, bloom, vignette;
  int same;
} ho_post_args;
int ho_post_level_size(int width, int height, int level, int *w, int *h);
int ho_post(const ho_post_args *a, uint16_t *hdr_out, uint16_t *levels_out, float *out_f32, uint8_t *out_rgba8);

#ifdef __cplusplus
}
#endif
#endif
