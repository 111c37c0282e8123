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

/* MLP on one feature row (20 inputs) with f16 weights, outputs 12 raw values (mode 0 f32, 1 f64, 2 the reference's
 * f16 arithmetic of the `f16` option, hush.js:683-703). */
void ho_mlp(const uint16_t *weights, long n_weights, const float *features, float *out, int fp64);
/* The `f16` option (hush.js:740): INFER's MLP in f16 arithmetic (mode 2 of ho_mlp); the rest of the frame unchanged. */
void ho_hush_set_mlp_half(ho_hush *h, int on);

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

/* ---- path tracer (src/pt/pathtracer.wgsl.js, bvh.js, scene.js, envmap.js), pt_oracle.cpp -----------------------
 * Frame uniforms in the byte layout of the reference's uniform buffer (pathtracer.wgsl.js:22-46, written by
 * pathtracer.js:105-149): 960 bytes. Matrices are column-major (three.js elements order). */
#define HO_PT_MAX_BLAS 8
#define HO_PT_MAX_LIGHTS 8
#define HO_PT_ENV_GW 256
#define HO_PT_ENV_GH 128
#define HO_PT_TEX_SIZE 1024
#define HO_PT_TEX_MIPS 11
typedef struct { uint32_t node_offset, tri_offset, node_count, flags; } ho_pt_blas; /* flags: 1 dynamic, 2 no shadow */
typedef struct { float pos[4], prev_pos[4], radiance[4], params[4]; } ho_pt_light;
typedef struct {
  float cam_pos[4], cam_right[4], cam_up[4], cam_fwd[4];
  float view_proj[16], prev_view_proj[16];
  uint32_t size[2], frame, mode;
  float jitter[2];
  uint32_t spp, max_bounces;
  float sky_zenith[4], sky_horizon[4], ground[4];
  uint32_t counts[4]; /* blas count, light count, sample offset, 0 */
  float clamp_lum, pixel_angle, shadow_tau, clamp_direct;
  float env[4]; /* intensity, cos / sin of the rotation about +y, 1 if a map is bound */
  ho_pt_blas blas[HO_PT_MAX_BLAS];
  ho_pt_light lights[HO_PT_MAX_LIGHTS];
} ho_pt_frame;
/* Scene buffers in the reference's GPU layouts (scene.js:167-171, 210-222, 294-311): packed BVH nodes (16 floats),
 * triangles (12 floats), triangle indices (4 u32: a, b, c, material | f16 texture LOD << 16), vertices (12 floats:
 * pos.xyz, u, prev.xyz, 0, normal.xyz, v), materials (20 x 4 bytes, tex as int32), the rgba8 texture array
 * (layers x 11 mips from 1024^2, level-major inside a layer) and the equirect environment map (rgba16float) with its
 * alias table (4 floats per cell of the 256 x 128 grid). */
typedef struct {
  const float *nodes, *tris, *verts, *mats;
  const uint32_t *tri_idx;
  const uint8_t *tex;
  int tex_layers;
  const uint16_t *env;
  int env_w, env_h;
  const float *env_table;
} ho_pt_scene;
/* main() of pathtracer.wgsl.js:648-672 over the whole image: mode 0 writes the five rgba16float G-buffer images
 * (radiance, normalDepth, motion, material, emission; dense), mode 1 adds to accum (4 floats per pixel). */
int ho_pt_render(const ho_pt_scene *s, const ho_pt_frame *f, uint16_t *const gbuf[5], float *accum);
/* One path of tracePath (pathtracer.wgsl.js:511-646) for pixel (x, y) with the RNG seeded as main() does; out:
 * radiance rgb, primary emission rgb, normal xyz, depth, motion xy, object id, previous depth, albedo rgb, rough. */
void ho_pt_pixel(const ho_pt_scene *s, const ho_pt_frame *f, int x, int y, float out[18]);
/* Closest hit of a ray through the BVHs and sphere lights (traceScene, 212-221): t, triangle (or -1), light, u, v. */
void ho_pt_trace(const ho_pt_scene *s, const ho_pt_frame *f, const float o[3], const float d[3], float out[5]);
/* bvh.js: buildBVH (12-143; nodes: 8 floats per node, room for 2 * max(1, n) nodes; returns the node count),
 * refitBVH (147-171), packedCount (178-183), packBVH (186-210). */
int ho_bvh_build(const float *pos, int tri_count, float *nodes, uint32_t *order, int *max_depth);
void ho_bvh_refit(float *nodes, int node_count, const float *tri_pos);
int ho_bvh_packed_count(const float *nodes, int node_count);
void ho_bvh_pack(const float *nodes, int node_count, float *out);
/* scene.js computeTriLod (178-208): the f16 bits of log2(texels per world unit) for one triangle. */
uint16_t ho_tri_lod(const float *va, const float *vb, const float *vc, int tex_size);
/* envmap.js prepareEnvMap (85-105): cuts the sun out of rgba (in place), writes the rgba16float map and the alias
 * table; returns 1 and the sun's direction / irradiance if one was cut. */
int ho_env_prepare(float *rgba, int w, int h, int sun, double sun_cone_deg, uint16_t *half_out, float *table_out,
                   double sun_dir[3], double sun_irr[3]);
/* pathtracer.js JITTER (6-12): 16 Halton(2, 3) phases in pixels. */
void ho_pt_jitter(float out[32]);

#ifdef __cplusplus
}
#endif
#endif
