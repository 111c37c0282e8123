// Analytic synthetic G-buffer scenes: a ground plane plus spheres and y-rotated boxes, ray-cast per pixel.
//
// Shared by the host generator and the device generator (gbuffer_gen.cu). Every frame
// buffer follows the reference's G-buffer layout (src/index.d.ts:1-17, src/denoise/hush.js:9-13):
//   radiance     rgb noisy 1 spp radiance without the primary emission, a = 1
//   normalDepth  world normal xyz, linear view depth w (< 0 = sky)
//   motion       xy = previous pixel - current pixel, z = object id (< 2048), w = linear depth in the previous camera
//   material     albedo rgb, roughness a
//   emission     primary emission rgb
// The projection follows the reference path tracer's conventions (src/pt/pathtracer.wgsl.js:505-509, 520-528,
// 560-562): ray d = normalize(fwd + right * ndc.x - up * ndc.y), pixel = ((ndc.x + 1) / 2 * W, (1 - ndc.y) / 2 * H),
// motion = prevPixel - curPixel, previous depth = clip w of the point in the previous camera.
#ifndef HUSH_SCENE_H
#define HUSH_SCENE_H

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define HS_HD __host__ __device__ __forceinline__
#else
#define HS_HD inline
#endif

#define HS_MAX_OBJECTS 64

typedef struct {
  int width, height;
  int n_objects;       // spheres + boxes besides the ground plane (<= HS_MAX_OBJECTS - 1)
  int n_moving;        // objects with their own velocity
  float sky_frac;      // target fraction of sky pixels (sets the camera pitch)
  float pan_min, pan_max;  // camera pan speed U[pan_min, pan_max] px/frame (drawn once per sequence)
  float yaw_deg;       // camera yaw per frame, degrees
  float firefly_rate, firefly_scale;
  int cut_frame;       // frame at which the camera jumps to a new pose (< 0: never)
  uint32_t seed;
} hs_desc;

typedef struct {
  float cx, cy, cz;    // centre
  float r;             // sphere radius / box half extent (x, z), box half height = 0.75 r
  float vx, vz;        // velocity per frame (world units)
  float cosr, sinr;    // box rotation about y
  float ar, ag, ab;    // albedo
  float rough;
  float emit;
  int type;            // 0 sphere, 1 box
  int id;              // object id (< 2048)
} hs_object;

typedef struct {
  int n;
  hs_object o[HS_MAX_OBJECTS];
  int ground_id;
  float ground_r, ground_g, ground_b, ground_rough;
  float lx, ly, lz;    // direction to the light (unit)
  float pan_px;        // pan speed for this sequence
  float tan_y;         // tan(fovy / 2)
  float pitch;         // camera pitch down (radians)
  float cam_h;         // camera height
  float depth_ref;     // depth at which the pan moves pan_px pixels per frame
} hs_scene;

typedef struct {
  float px, py, pz;
  float fx, fy, fz, rx, ry, rz, ux, uy, uz;  // unit forward / right / up
  float tan_x, tan_y;
} hs_camera;

// ------------------------------------------------------------------------------------------------ RNG
// PCG hash (Jarzynski & Olano, "Hash Functions for GPU Rendering", JCGT 2020): counter-based, one 32-bit state.
HS_HD uint32_t hs_pcg(uint32_t v) {
  uint32_t s = v * 747796405u + 2891336453u;
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
HS_HD float hs_u01(uint32_t a, uint32_t b, uint32_t c) {  // uniform in [0, 1)
  uint32_t h = hs_pcg(a ^ hs_pcg(b ^ hs_pcg(c)));
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

// ------------------------------------------------------------------------------------------------ scene setup
HS_HD void hs_build_scene(const hs_desc *d, hs_scene *s) {
  const uint32_t sd = d->seed * 0x9E3779B9u + 0x1234567u;
  s->n = d->n_objects < HS_MAX_OBJECTS - 1 ? d->n_objects : HS_MAX_OBJECTS - 1;
  s->tan_y = 0.57735026f;  // fovy = 60 degrees
  s->cam_h = 2.5f;
  // pitch so that the horizon sits sky_frac of the way down the image: tan(pitch) = tan_y (1 - 2 sky_frac)
  s->pitch = atanf(s->tan_y * (1.0f - 2.0f * d->sky_frac));
  s->depth_ref = 10.0f;
  s->pan_px = d->pan_min + (d->pan_max - d->pan_min) * hs_u01(sd, 1u, 0u);
  float lx = 0.45f, ly = 0.8f, lz = -0.35f;
  float ll = sqrtf(lx * lx + ly * ly + lz * lz);
  s->lx = lx / ll; s->ly = ly / ll; s->lz = lz / ll;
  s->ground_id = 1 + (int)(hs_u01(sd, 2u, 0u) * 2000.0f);
  s->ground_r = 0.05f + 0.85f * hs_u01(sd, 3u, 0u);
  s->ground_g = 0.05f + 0.85f * hs_u01(sd, 3u, 1u);
  s->ground_b = 0.05f + 0.85f * hs_u01(sd, 3u, 2u);
  s->ground_rough = hs_u01(sd, 3u, 3u);
  for (int i = 0; i < s->n; i++) {
    hs_object *o = &s->o[i];
    const uint32_t k = 100u + (uint32_t)i;
    o->type = hs_u01(sd, k, 0u) < 0.5f ? 0 : 1;
    o->r = 0.2f + 1.3f * hs_u01(sd, k, 1u);
    // scattered over the region the camera sees (heading +z, x in [-9, 9], z in [3, 22])
    o->cx = -9.0f + 18.0f * hs_u01(sd, k, 2u);
    o->cz = 3.0f + 19.0f * hs_u01(sd, k, 3u);
    float lift = hs_u01(sd, k, 4u) < 0.25f ? 1.5f * hs_u01(sd, k, 5u) : 0.0f;
    o->cy = (o->type == 0 ? o->r : 0.75f * o->r) + lift;
    float ang = 6.2831853f * hs_u01(sd, k, 6u);
    o->cosr = cosf(ang); o->sinr = sinf(ang);
    o->ar = 0.05f + 0.85f * hs_u01(sd, k, 7u);
    o->ag = 0.05f + 0.85f * hs_u01(sd, k, 8u);
    o->ab = 0.05f + 0.85f * hs_u01(sd, k, 9u);
    o->rough = hs_u01(sd, k, 10u);
    o->emit = 0.0f;
    o->vx = o->vz = 0.0f;
    // distinct ids < 2048, away from the ground's id
    o->id = 2 + (int)(((uint32_t)(s->ground_id + 37 * (i + 1))) % 2040u);
  }
  // one emissive sphere (the first sphere found)
  for (int i = 0; i < s->n; i++) {
    if (s->o[i].type == 0) { s->o[i].emit = 5.0f; break; }
  }
  for (int i = 0; i < s->n && i < d->n_moving; i++) {
    float a = 6.2831853f * hs_u01(sd, 500u + (uint32_t)i, 0u);
    float v = 0.02f + 0.06f * hs_u01(sd, 500u + (uint32_t)i, 1u);
    s->o[s->n - 1 - i].vx = v * cosf(a);
    s->o[s->n - 1 - i].vz = v * sinf(a);
  }
}

// Camera at a frame: yaw per frame plus a lateral pan so points at depth_ref move pan_px pixels per frame. A cut
// frame and every later frame use a second pose (turned 35 degrees, moved sideways).
HS_HD void hs_camera_at(const hs_desc *d, const hs_scene *s, int frame, hs_camera *c) {
  float tf = (float)frame;
  float yaw = tf * d->yaw_deg * 0.017453292f;
  float tan_x = s->tan_y * (float)d->width / (float)d->height;
  float px_world = s->depth_ref * 2.0f * tan_x / (float)d->width;  // world units per pixel at depth_ref
  float side = tf * s->pan_px * px_world;
  float ox = 0.0f, oz = -6.0f;
  if (d->cut_frame >= 0 && frame >= d->cut_frame) {
    yaw += 0.61086524f;
    ox += -4.0f;
    oz += 3.0f;
  }
  float hx = sinf(yaw), hz = cosf(yaw);     // heading
  float cp = cosf(s->pitch), sp = sinf(s->pitch);
  c->fx = hx * cp; c->fy = -sp; c->fz = hz * cp;
  c->rx = hz; c->ry = 0.0f; c->rz = -hx;    // right = heading x up
  c->ux = hx * sp; c->uy = cp; c->uz = hz * sp;
  c->px = ox + side * c->rx;
  c->py = s->cam_h;
  c->pz = oz + side * c->rz;
  c->tan_x = tan_x;
  c->tan_y = s->tan_y;
}

HS_HD void hs_object_pos(const hs_object *o, int frame, float *x, float *y, float *z) {
  *x = o->cx + o->vx * (float)frame;
  *y = o->cy;
  *z = o->cz + o->vz * (float)frame;
}

// Nearest hit along o + t d (t > tmin): returns the object index (-1 ground, -2 none), t and the normal.
HS_HD int hs_trace(const hs_scene *s, int frame, float ox, float oy, float oz, float dx, float dy, float dz,
                   float tmin, float *t_out, float *nx, float *ny, float *nz, int skip_ground) {
  float tbest = 1e30f;
  int hit = -2;
  float bnx = 0.0f, bny = 1.0f, bnz = 0.0f;
  if (!skip_ground && dy < -1e-6f) {
    float t = -oy / dy;
    if (t > tmin && t < tbest) { tbest = t; hit = -1; bnx = 0.0f; bny = 1.0f; bnz = 0.0f; }
  }
  for (int i = 0; i < s->n; i++) {
    const hs_object *o = &s->o[i];
    float cx, cy, cz;
    hs_object_pos(o, frame, &cx, &cy, &cz);
    float lx = ox - cx, ly = oy - cy, lz = oz - cz;
    if (o->type == 0) {
      float b = lx * dx + ly * dy + lz * dz;
      float c = lx * lx + ly * ly + lz * lz - o->r * o->r;
      float disc = b * b - c;
      if (disc < 0.0f) continue;
      float sq = sqrtf(disc);
      float t = -b - sq;
      if (t <= tmin) t = -b + sq;
      if (t > tmin && t < tbest) {
        tbest = t; hit = i;
        float inv = 1.0f / o->r;
        bnx = (lx + t * dx) * inv; bny = (ly + t * dy) * inv; bnz = (lz + t * dz) * inv;
      }
    } else {
      // slab test in the box frame (rotation about y)
      float qx = o->cosr * lx + o->sinr * lz, qz = -o->sinr * lx + o->cosr * lz, qy = ly;
      float ex = o->cosr * dx + o->sinr * dz, ez = -o->sinr * dx + o->cosr * dz, ey = dy;
      float hx = o->r, hy = 0.75f * o->r, hz = o->r;
      float t0 = -1e30f, t1 = 1e30f;
      int axis = 0;
      float sgn = 1.0f;
      float qv[3] = {qx, qy, qz}, ev[3] = {ex, ey, ez}, hv[3] = {hx, hy, hz};
      int ok = 1;
      for (int a = 0; a < 3; a++) {
        if (fabsf(ev[a]) < 1e-12f) {
          if (qv[a] < -hv[a] || qv[a] > hv[a]) { ok = 0; break; }
          continue;
        }
        float inv = 1.0f / ev[a];
        float ta = (-hv[a] - qv[a]) * inv, tb = (hv[a] - qv[a]) * inv;
        float sa = -1.0f;
        if (ta > tb) { float tmp = ta; ta = tb; tb = tmp; sa = 1.0f; }
        if (ta > t0) { t0 = ta; axis = a; sgn = sa; }
        if (tb < t1) t1 = tb;
      }
      if (!ok || t0 > t1 || t0 <= tmin || t0 >= tbest) continue;
      tbest = t0; hit = i;
      float ln[3] = {0.0f, 0.0f, 0.0f};
      ln[axis] = sgn;
      // back to world: inverse rotation
      bnx = o->cosr * ln[0] - o->sinr * ln[2];
      bny = ln[1];
      bnz = o->sinr * ln[0] + o->cosr * ln[2];
    }
  }
  *t_out = tbest;
  *nx = bnx; *ny = bny; *nz = bnz;
  return hit;
}

HS_HD void hs_project(const hs_camera *c, int W, int H, float x, float y, float z, float *pxo, float *pyo,
                      float *depth) {
  float vx = x - c->px, vy = y - c->py, vz = z - c->pz;
  float zc = vx * c->fx + vy * c->fy + vz * c->fz;
  float ndx = (vx * c->rx + vy * c->ry + vz * c->rz) / (zc * c->tan_x);
  float ndy = (vx * c->ux + vy * c->uy + vz * c->uz) / (zc * c->tan_y);  // clip-space y (up)
  *pxo = (ndx * 0.5f + 0.5f) * (float)W;
  *pyo = (0.5f - ndy * 0.5f) * (float)H;
  *depth = zc;
}

// Per-pixel outputs in f32: rad[3], nd[4], mv[4], mat[4], emi[3], clean[3] (noise-free radiance + emission).
HS_HD void hs_shade_pixel(const hs_desc *d, const hs_scene *s, const hs_camera *cam, const hs_camera *pcam,
                          int frame, int x, int y, float *rad, float *nd, float *mv, float *mat, float *emi,
                          float *clean) {
  const int W = d->width, H = d->height;
  float ndcx = ((float)x + 0.5f) / (float)W * 2.0f - 1.0f;
  float ndcy = ((float)y + 0.5f) / (float)H * 2.0f - 1.0f;
  float dx = cam->fx + cam->rx * cam->tan_x * ndcx - cam->ux * cam->tan_y * ndcy;
  float dy = cam->fy + cam->ry * cam->tan_x * ndcx - cam->uy * cam->tan_y * ndcy;
  float dz = cam->fz + cam->rz * cam->tan_x * ndcx - cam->uz * cam->tan_y * ndcy;
  float dl = sqrtf(dx * dx + dy * dy + dz * dz);
  dx /= dl; dy /= dl; dz /= dl;
  float t, nx, ny, nz;
  int hit = hs_trace(s, frame, cam->px, cam->py, cam->pz, dx, dy, dz, 1e-4f, &t, &nx, &ny, &nz, 0);
  const float cpx = (float)x + 0.5f, cpy = (float)y + 0.5f;
  if (hit == -2 || t > 400.0f) {
    // sky: depth -1, normal -d, motion of the direction (rotation only), albedo 1, no emission or radiance
    rad[0] = rad[1] = rad[2] = 0.0f;
    nd[0] = -dx; nd[1] = -dy; nd[2] = -dz; nd[3] = -1.0f;
    float far = 1e4f, ppx, ppy, pd;
    hs_project(pcam, W, H, pcam->px + dx * far, pcam->py + dy * far, pcam->pz + dz * far, &ppx, &ppy, &pd);
    mv[0] = ppx - cpx; mv[1] = ppy - cpy; mv[2] = 0.0f; mv[3] = -1.0f;
    mat[0] = mat[1] = mat[2] = 1.0f; mat[3] = 1.0f;
    emi[0] = emi[1] = emi[2] = 0.0f;
    clean[0] = clean[1] = clean[2] = 0.0f;
    return;
  }
  float hx = cam->px + t * dx, hy = cam->py + t * dy, hz = cam->pz + t * dz;
  float ar, ag, ab, rough, emit = 0.0f;
  int id;
  float vx = 0.0f, vz = 0.0f;
  int cell;
  if (hit == -1) {
    ar = s->ground_r; ag = s->ground_g; ab = s->ground_b; rough = s->ground_rough; id = s->ground_id;
    cell = (int)floorf(hx + 0.25f) + (int)floorf(hz + 0.25f);  // unit cells on the plane (y = 0 is the surface)
  } else {
    const hs_object *o = &s->o[hit];
    ar = o->ar; ag = o->ag; ab = o->ab; rough = o->rough; id = o->id; emit = o->emit;
    vx = o->vx; vz = o->vz;
    // 8 cells across the object, in coordinates relative to its centre, offset by a quarter cell so that no face
    // of a box lies on a cell boundary (host and device rounding would pick different cells there)
    float cx, cy, cz;
    hs_object_pos(o, frame, &cx, &cy, &cz);
    const float k = 8.0f / (2.0f * o->r);
    cell = (int)floorf((hx - cx) * k + 0.25f) + (int)floorf((hy - cy) * k + 0.25f) + (int)floorf((hz - cz) * k + 0.25f);
  }
  float chk = (cell & 1) ? 0.6f : 1.0f;
  ar *= chk; ag *= chk; ab *= chk;
  // Lambert under one directional light (hard shadow) + 0.1 ambient
  float ndl = nx * s->lx + ny * s->ly + nz * s->lz;
  float vis = 0.0f;
  if (ndl > 0.0f) {
    float st, snx, sny, snz;
    int sh = hs_trace(s, frame, hx + nx * 1e-3f, hy + ny * 1e-3f, hz + nz * 1e-3f, s->lx, s->ly, s->lz, 1e-4f, &st,
                      &snx, &sny, &snz, 1);
    vis = sh == -2 ? 1.0f : 0.0f;
  }
  float shade = (ndl > 0.0f ? ndl * vis : 0.0f) + 0.1f;
  float cr = ar * shade, cg = ag * shade, cb = ab * shade;
  // 1 spp noise: clean x Exp(1) per channel, fireflies
  const uint32_t pix = (uint32_t)(y * W + x);
  const uint32_t fs = d->seed * 0x85EBCA6Bu + (uint32_t)frame * 0xC2B2AE35u;
  float e0 = -logf(1.0f - hs_u01(fs, pix, 0u));
  float e1 = -logf(1.0f - hs_u01(fs, pix, 1u));
  float e2 = -logf(1.0f - hs_u01(fs, pix, 2u));
  float ff = hs_u01(fs, pix, 3u) < d->firefly_rate ? d->firefly_scale : 1.0f;
  rad[0] = cr * e0 * ff; rad[1] = cg * e1 * ff; rad[2] = cb * e2 * ff;
  float depth = (hx - cam->px) * cam->fx + (hy - cam->py) * cam->fy + (hz - cam->pz) * cam->fz;
  nd[0] = nx; nd[1] = ny; nd[2] = nz; nd[3] = depth;
  // motion: where this surface point was one frame earlier, seen by the previous camera
  float ppx, ppy, pdepth;
  hs_project(pcam, W, H, hx - vx, hy, hz - vz, &ppx, &ppy, &pdepth);
  float cpx2, cpy2, cd;
  hs_project(cam, W, H, hx, hy, hz, &cpx2, &cpy2, &cd);
  mv[0] = ppx - cpx2; mv[1] = ppy - cpy2; mv[2] = (float)id; mv[3] = pdepth;
  mat[0] = ar; mat[1] = ag; mat[2] = ab; mat[3] = rough;
  emi[0] = emi[1] = emi[2] = emit;
  clean[0] = cr + emit; clean[1] = cg + emit; clean[2] = cb + emit;
}

#endif
