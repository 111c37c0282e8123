// Synthetic G-buffer frames (scene.h) on the host (OpenMP over rows) and on the device (one thread per pixel).
// Inputs are stored as rgba16float with round-to-nearest (a renderer's output; the denoiser never sees the f32).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstring>

#include "hush.h"
#include "scene.h"

static hs_desc to_desc(const hush_scene *s) {
  hs_desc d;
  d.width = s->width; d.height = s->height; d.n_objects = s->n_objects; d.n_moving = s->n_moving;
  d.sky_frac = s->sky_frac; d.pan_min = s->pan_min; d.pan_max = s->pan_max; d.yaw_deg = s->yaw_deg;
  d.firefly_rate = s->firefly_rate; d.firefly_scale = s->firefly_scale; d.cut_frame = s->cut_frame; d.seed = s->seed;
  return d;
}

__host__ __device__ static inline void store4(uint16_t *p, size_t i, float a, float b, float c, float d) {
  p[i * 4 + 0] = __half_as_ushort(__float2half_rn(a));
  p[i * 4 + 1] = __half_as_ushort(__float2half_rn(b));
  p[i * 4 + 2] = __half_as_ushort(__float2half_rn(c));
  p[i * 4 + 3] = __half_as_ushort(__float2half_rn(d));
}

__host__ __device__ static inline void gen_pixel(const hs_desc &d, const hs_scene &sc, const hs_camera &cam,
                                                 const hs_camera &pcam, int frame, int x, int y, uint16_t *rad,
                                                 uint16_t *nd, uint16_t *mv, uint16_t *mat, uint16_t *emi,
                                                 float *clean) {
  float r[3], n[4], m[4], a[4], e[3], c[3];
  hs_shade_pixel(&d, &sc, &cam, &pcam, frame, x, y, r, n, m, a, e, c);
  const size_t i = (size_t)y * d.width + x;
  if (rad) store4(rad, i, r[0], r[1], r[2], 1.0f);
  if (nd) store4(nd, i, n[0], n[1], n[2], n[3]);
  if (mv) store4(mv, i, m[0], m[1], m[2], m[3]);
  if (mat) store4(mat, i, a[0], a[1], a[2], a[3]);
  if (emi) store4(emi, i, e[0], e[1], e[2], 0.0f);
  if (clean) { clean[i * 3 + 0] = c[0]; clean[i * 3 + 1] = c[1]; clean[i * 3 + 2] = c[2]; }
}

extern "C" int hush_scene_frame_host(const hush_scene *s, int frame, uint16_t *radiance, uint16_t *normal_depth,
                                     uint16_t *motion, uint16_t *material, uint16_t *emission, float *clean) {
  if (!s || s->width <= 0 || s->height <= 0) return HUSH_ERR_ARG;
  const hs_desc d = to_desc(s);
  hs_scene sc;
  hs_build_scene(&d, &sc);
  hs_camera cam, pcam;
  hs_camera_at(&d, &sc, frame, &cam);
  hs_camera_at(&d, &sc, frame - 1, &pcam);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < d.height; y++)
    for (int x = 0; x < d.width; x++)
      gen_pixel(d, sc, cam, pcam, frame, x, y, radiance, normal_depth, motion, material, emission, clean);
  return HUSH_OK;
}

__global__ void k_scene(const hs_desc d, const hs_scene sc, const hs_camera cam, const hs_camera pcam, int frame,
                        uint16_t *rad, uint16_t *nd, uint16_t *mv, uint16_t *mat, uint16_t *emi, float *clean) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= d.width || y >= d.height) return;
  gen_pixel(d, sc, cam, pcam, frame, x, y, rad, nd, mv, mat, emi, clean);
}

extern "C" int hush_scene_frame_device(const hush_scene *s, int frame, void *radiance, void *normal_depth,
                                       void *motion, void *material, void *emission, void *clean, void *stream) {
  if (!s || s->width <= 0 || s->height <= 0) return HUSH_ERR_ARG;
  const hs_desc d = to_desc(s);
  hs_scene sc;
  hs_build_scene(&d, &sc);
  hs_camera cam, pcam;
  hs_camera_at(&d, &sc, frame, &cam);
  hs_camera_at(&d, &sc, frame - 1, &pcam);
  const dim3 blk(16, 8), grd((d.width + 15) / 16, (d.height + 7) / 8);
  k_scene<<<grd, blk, 0, (cudaStream_t)stream>>>(d, sc, cam, pcam, frame, (uint16_t *)radiance,
                                                 (uint16_t *)normal_depth, (uint16_t *)motion, (uint16_t *)material,
                                                 (uint16_t *)emission, (float *)clean);
  return cudaGetLastError() == cudaSuccess ? HUSH_OK : HUSH_ERR_CUDA;
}
