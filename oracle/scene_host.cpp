// Host build of the synthetic G-buffer generator, for the CPU side of the measurements and for CPU tests.
//
// TEST INFRASTRUCTURE. The generator's arithmetic lives in one header (hush_b200/csrc/scene.h) that the product's
// device and host generators include too; compiling it here as well lets the CPU timing arm produce its input frames
// without loading the product library. Storage is rgba16float with round-to-nearest-even, as the product's
// generator stores it (__float2half_rn); tests/test_oracle_kat.py checks the two frame for frame, bit for bit.
#include <stdint.h>
#include <string.h>

#include "../hush_b200/csrc/scene.h"

// f32 -> f16, IEEE 754 round to nearest, ties to even (subnormals, overflow to infinity, NaN kept quiet).
static uint16_t f2h_rne(float f) {
  uint32_t x;
  memcpy(&x, &f, 4);
  const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
  const uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u);
  if (ax >= 0x477ff000u) return sign | 0x7c00u;  // >= 65520 rounds past the largest finite f16 (65504)
  const uint32_t e = ax >> 23;
  const uint32_t m = ax & 0x7fffffu;
  uint32_t q, r, half;
  if (e < 113) {  // below 2^-14: an f16 subnormal (or zero) in units of 2^-24
    const uint32_t M = m | 0x800000u;
    const uint32_t shift = 126 - e;
    if (shift > 31) return sign;
    q = M >> shift;
    r = M & ((1u << shift) - 1u);
    half = 1u << (shift - 1);
  } else {
    q = ((e - 112) << 10) | (m >> 13);
    r = m & 0x1fffu;
    half = 0x1000u;
  }
  if (r > half || (r == half && (q & 1u))) q++;
  return sign | (uint16_t)q;
}

static void put4(uint16_t *p, size_t i, float a, float b, float c, float d) {
  p[i * 4 + 0] = f2h_rne(a);
  p[i * 4 + 1] = f2h_rne(b);
  p[i * 4 + 2] = f2h_rne(c);
  p[i * 4 + 3] = f2h_rne(d);
}

extern "C" uint16_t ho_f2h_rne(float f) { return f2h_rne(f); }

// One frame of the sequence `d` into five W x H rgba16float images (any may be NULL) and the noise-free radiance
// (W x H x 3 floats, may be NULL). Returns 0, or 1 for a bad size.
extern "C" int ho_scene_frame(const hs_desc *d, int frame, uint16_t *rad, uint16_t *nd, uint16_t *mv, uint16_t *mat,
                              uint16_t *emi, float *clean) {
  if (!d || d->width <= 0 || d->height <= 0) return 1;
  hs_scene sc;
  hs_build_scene(d, &sc);
  hs_camera cam, pcam;
  hs_camera_at(d, &sc, frame, &cam);
  hs_camera_at(d, &sc, frame - 1, &pcam);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < d->height; y++)
    for (int x = 0; x < d->width; x++) {
      float r[3], n[4], m[4], a[4], e[3], c[3];
      hs_shade_pixel(d, &sc, &cam, &pcam, frame, x, y, r, n, m, a, e, c);
      const size_t i = (size_t)y * d->width + x;
      if (rad) put4(rad, i, r[0], r[1], r[2], 1.0f);
      if (nd) put4(nd, i, n[0], n[1], n[2], n[3]);
      if (mv) put4(mv, i, m[0], m[1], m[2], m[3]);
      if (mat) put4(mat, i, a[0], a[1], a[2], a[3]);
      if (emi) put4(emi, i, e[0], e[1], e[2], 0.0f);
      if (clean) {
        clean[i * 3 + 0] = c[0];
        clean[i * 3 + 1] = c[1];
        clean[i * 3 + 2] = c[2];
      }
    }
  return 0;
}
