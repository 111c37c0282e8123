/* N-API addon over the C ABI of include/hush.h: the native half of the drop-in `Hush` / `SVGF` classes that
 * node/index.js exposes with the reference's surface (src/index.d.ts:36-83).
 *
 * Build (node-gyp, see binding.gyp): the addon links libhush_b200.so built by `python -m hush_b200.build`.
 * Device buffers cross the JS boundary as BigInt device addresses of rgba16float images (a WebGPU -> CUDA
 * external-memory import, or any CUDA allocator, supplies them); a CUDA stream is a BigInt handle, 0n being the
 * default stream. Every failing call throws a JS Error carrying the library's message, which reuses the reference's
 * error texts (hush.js:735, 743, 765, 816, 818).
 *
 * Exports: hushCreate, hushDenoise, hushOutput, hushReset, hushResize, hushSetExposure, hushSetWeights, hushDestroy,
 * hiddenOf, requiredLimits, svgfCreate, svgfEncode, svgfOutput, svgfReset, svgfResize, svgfDestroy. */
#include <node_api.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "hush.h"

#define CHECK_NAPI(env, call)                                   \
  do {                                                          \
    if ((call) != napi_ok) {                                    \
      napi_throw_error((env), NULL, "hush addon: " #call);      \
      return NULL;                                              \
    }                                                           \
  } while (0)

static napi_value throw_msg(napi_env env, const char *msg) {
  napi_throw_error(env, NULL, msg && msg[0] ? msg : "hush: unknown error");
  return NULL;
}

/* The handle objects: an external wrapping the instance, released by its finalizer or by destroy(). */
typedef struct {
  hush_t *h;
} hush_box;
typedef struct {
  svgf_t *s;
} svgf_box;

static void hush_finalize(napi_env env, void *data, void *hint) {
  (void)env; (void)hint;
  hush_box *b = (hush_box *)data;
  if (b->h) hush_destroy(b->h);
  free(b);
}
static void svgf_finalize(napi_env env, void *data, void *hint) {
  (void)env; (void)hint;
  svgf_box *b = (svgf_box *)data;
  if (b->s) svgf_destroy(b->s);
  free(b);
}

static hush_box *get_hush(napi_env env, napi_value v) {
  void *p = NULL;
  if (napi_get_value_external(env, v, &p) != napi_ok || !p || !((hush_box *)p)->h) {
    napi_throw_error(env, NULL, "Hush: instance destroyed or invalid");
    return NULL;
  }
  return (hush_box *)p;
}
static svgf_box *get_svgf(napi_env env, napi_value v) {
  void *p = NULL;
  if (napi_get_value_external(env, v, &p) != napi_ok || !p || !((svgf_box *)p)->s) {
    napi_throw_error(env, NULL, "SVGF: instance destroyed or invalid");
    return NULL;
  }
  return (svgf_box *)p;
}

/* Optional named properties of an options object. */
static bool opt_double(napi_env env, napi_value obj, const char *name, double *out) {
  bool has = false;
  napi_value v;
  napi_valuetype t;
  if (napi_has_named_property(env, obj, name, &has) != napi_ok || !has) return false;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok) return false;
  if (napi_typeof(env, v, &t) != napi_ok || t != napi_number) return false;
  return napi_get_value_double(env, v, out) == napi_ok;
}
static bool opt_bool(napi_env env, napi_value obj, const char *name, bool *out) {
  bool has = false;
  napi_value v;
  napi_valuetype t;
  if (napi_has_named_property(env, obj, name, &has) != napi_ok || !has) return false;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok) return false;
  if (napi_typeof(env, v, &t) != napi_ok || t != napi_boolean) return false;
  return napi_get_value_bool(env, v, out) == napi_ok; /* a C bool, never written through a wider pointer */
}
/* A BigInt device address or stream handle (0 when absent or undefined). */
static uint64_t bigint_or_zero(napi_env env, napi_value v) {
  napi_valuetype t;
  uint64_t x = 0;
  bool lossless = true;
  if (napi_typeof(env, v, &t) != napi_ok || t != napi_bigint) return 0;
  napi_get_value_bigint_uint64(env, v, &x, &lossless);
  return x;
}
static uint64_t named_bigint(napi_env env, napi_value obj, const char *name) {
  bool has = false;
  napi_value v;
  if (napi_has_named_property(env, obj, name, &has) != napi_ok || !has) return 0;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok) return 0;
  return bigint_or_zero(env, v);
}
static napi_value make_bigint(napi_env env, const void *p) {
  napi_value r;
  CHECK_NAPI(env, napi_create_bigint_uint64(env, (uint64_t)(uintptr_t)p, &r));
  return r;
}

/* Weights as a Uint16Array of f16 bits (index.js decodes ArrayBuffer / typed arrays / base64 into one). */
static bool get_u16(napi_env env, napi_value v, const uint16_t **data, size_t *n) {
  napi_typedarray_type type;
  size_t length = 0, offset = 0;
  void *p = NULL;
  napi_value ab;
  bool is = false;
  if (napi_is_typedarray(env, v, &is) != napi_ok || !is) return false;
  if (napi_get_typedarray_info(env, v, &type, &length, &p, &ab, &offset) != napi_ok) return false;
  if (type != napi_uint16_array) return false;
  *data = (const uint16_t *)p;
  *n = length;
  return true;
}

/* hushCreate({width, height, exposure?, f16?, weights?: Uint16Array, device?}) -> handle (hush.js:731-761) */
static napi_value hush_create_js(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc < 1) return throw_msg(env, "Hush: options required");
  double w = 0, h = 0, e = 1.0, dev = -1;
  bool f16 = false;
  opt_double(env, argv[0], "width", &w);
  opt_double(env, argv[0], "height", &h);
  opt_double(env, argv[0], "exposure", &e);
  opt_double(env, argv[0], "device", &dev);
  opt_bool(env, argv[0], "f16", &f16);
  hush_desc d = hush_desc_default((int)w, (int)h);
  d.exposure = (float)e;
  d.f16 = f16 ? 1 : 0;
  d.device = (int)dev;
  bool has = false;
  napi_value wv;
  if (napi_has_named_property(env, argv[0], "weights", &has) == napi_ok && has &&
      napi_get_named_property(env, argv[0], "weights", &wv) == napi_ok) {
    napi_valuetype t;
    napi_typeof(env, wv, &t);
    if (t != napi_undefined && t != napi_null) {
      if (!get_u16(env, wv, &d.weights, &d.n_weights)) return throw_msg(env, "Hush: weights must be a Uint16Array");
    }
  }
  hush_t *inst = NULL;
  if (hush_create(&d, &inst) != HUSH_OK) return throw_msg(env, hush_global_error());
  hush_box *b = (hush_box *)malloc(sizeof(hush_box));
  if (!b) {
    hush_destroy(inst);
    return throw_msg(env, "Hush: out of host memory");
  }
  b->h = inst;
  napi_value ext;
  CHECK_NAPI(env, napi_create_external(env, b, hush_finalize, NULL, &ext));
  return ext;
}

static const char *INPUT_NAMES[7] = {"radiance", "normalDepth", "motion", "material", "emission", "prevNormalDepth",
                                     "prevMotion"};

/* hushDenoise(handle, inputs {radiance, normalDepth, motion, material, emission}: BigInt, stream?: BigInt)
 * -> BigInt output address (hush.js:813-822) */
static napi_value hush_denoise_js(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc < 2) return throw_msg(env, "Hush.denoise: inputs required");
  hush_box *b = get_hush(env, argv[0]);
  if (!b) return NULL;
  hush_inputs in;
  memset(&in, 0, sizeof in);
  const void **slot[5] = {&in.radiance, &in.normal_depth, &in.motion, &in.material, &in.emission};
  for (int k = 0; k < 5; k++) *slot[k] = (const void *)(uintptr_t)named_bigint(env, argv[1], INPUT_NAMES[k]);
  const uint64_t stream = argc > 2 ? bigint_or_zero(env, argv[2]) : 0;
  const void *out = NULL;
  if (hush_denoise(b->h, &in, (void *)(uintptr_t)stream, &out) != HUSH_OK) return throw_msg(env, hush_last_error(b->h));
  return make_bigint(env, out);
}

static napi_value hush_output_js(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  hush_box *b = argc ? get_hush(env, argv[0]) : NULL;
  if (!b) return NULL;
  return make_bigint(env, hush_output(b->h));
}

static napi_value hush_reset_js(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  hush_box *b = argc ? get_hush(env, argv[0]) : NULL;
  if (!b) return NULL;
  if (hush_reset(b->h) != HUSH_OK) return throw_msg(env, hush_last_error(b->h));
  return NULL;
}

static napi_value hush_resize_js(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  double w = 0, h = 0;
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  hush_box *b = argc ? get_hush(env, argv[0]) : NULL;
  if (!b) return NULL;
  if (argc < 3 || napi_get_value_double(env, argv[1], &w) != napi_ok || napi_get_value_double(env, argv[2], &h) != napi_ok)
    return throw_msg(env, "Hush.resize: width and height required");
  if (hush_resize(b->h, (int)w, (int)h) != HUSH_OK) return throw_msg(env, hush_last_error(b->h));
  return NULL;
}

static napi_value hush_set_exposure_js(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  double e = 1.0;
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  hush_box *b = argc ? get_hush(env, argv[0]) : NULL;
  if (!b) return NULL;
  if (argc < 2 || napi_get_value_double(env, argv[1], &e) != napi_ok) return throw_msg(env, "Hush: exposure must be a number");
  if (hush_set_exposure(b->h, (float)e) != HUSH_OK) return throw_msg(env, hush_last_error(b->h));
  return NULL;
}

static napi_value hush_set_weights_js(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  const uint16_t *w = NULL;
  size_t n = 0;
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  hush_box *b = argc ? get_hush(env, argv[0]) : NULL;
  if (!b) return NULL;
  if (argc < 2 || !get_u16(env, argv[1], &w, &n)) return throw_msg(env, "Hush: weights must be a Uint16Array");
  if (hush_set_weights(b->h, w, n) != HUSH_OK) return throw_msg(env, hush_last_error(b->h));
  return NULL;
}

static napi_value hush_destroy_js(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  void *p = NULL;
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc && napi_get_value_external(env, argv[0], &p) == napi_ok && p) {
    hush_box *b = (hush_box *)p;
    if (b->h) hush_destroy(b->h);
    b->h = NULL; /* the finalizer then frees only the box */
  }
  return NULL;
}

/* hiddenOf(count) (hush.js:22-25) */
static napi_value hidden_of_js(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1], r;
  double n = 0;
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc) napi_get_value_double(env, argv[0], &n);
  CHECK_NAPI(env, napi_create_int32(env, hush_hidden_of((long)n), &r));
  return r;
}

/* requiredLimits() -> {computeCapability, maxSharedMemoryPerBlock} (hush.js:721, 726) */
static napi_value required_limits_js(napi_env env, napi_callback_info info) {
  (void)info;
  int major = 0, minor = 0;
  size_t smem = 0;
  hush_required_limits(&major, &minor, &smem);
  napi_value o, v;
  CHECK_NAPI(env, napi_create_object(env, &o));
  CHECK_NAPI(env, napi_create_double(env, major + minor / 10.0, &v));
  CHECK_NAPI(env, napi_set_named_property(env, o, "computeCapability", v));
  CHECK_NAPI(env, napi_create_double(env, (double)smem, &v));
  CHECK_NAPI(env, napi_set_named_property(env, o, "maxSharedMemoryPerBlock", v));
  return o;
}

/* svgfCreate(width, height, {iterations, sigmaL, sigmaN, sigmaZ, alphaColor, alphaMoments, taaAlpha, taa}, device?)
 * (svgf.js:273-300) */
static napi_value svgf_create_js(napi_env env, napi_callback_info info) {
  size_t argc = 4;
  napi_value argv[4];
  double w = 0, h = 0, dev = -1, x;
  bool taa;
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc < 2) return throw_msg(env, "SVGF: width and height required");
  napi_get_value_double(env, argv[0], &w);
  napi_get_value_double(env, argv[1], &h);
  svgf_options o = svgf_options_default();
  if (argc > 2) {
    napi_valuetype t;
    napi_typeof(env, argv[2], &t);
    if (t == napi_object) {
      if (opt_double(env, argv[2], "iterations", &x)) o.iterations = (int)x;
      if (opt_double(env, argv[2], "sigmaL", &x)) o.sigma_l = (float)x;
      if (opt_double(env, argv[2], "sigmaN", &x)) o.sigma_n = (float)x;
      if (opt_double(env, argv[2], "sigmaZ", &x)) o.sigma_z = (float)x;
      if (opt_double(env, argv[2], "alphaColor", &x)) o.alpha_color = (float)x;
      if (opt_double(env, argv[2], "alphaMoments", &x)) o.alpha_moments = (float)x;
      if (opt_double(env, argv[2], "taaAlpha", &x)) o.taa_alpha = (float)x;
      if (opt_bool(env, argv[2], "taa", &taa)) o.taa = taa ? 1 : 0;
    }
  }
  if (argc > 3) napi_get_value_double(env, argv[3], &dev);
  svgf_t *s = NULL;
  if (svgf_create((int)w, (int)h, &o, (int)dev, &s) != HUSH_OK) return throw_msg(env, hush_global_error());
  svgf_box *b = (svgf_box *)malloc(sizeof(svgf_box));
  if (!b) {
    svgf_destroy(s);
    return throw_msg(env, "SVGF: out of host memory");
  }
  b->s = s;
  napi_value ext;
  CHECK_NAPI(env, napi_create_external(env, b, svgf_finalize, NULL, &ext));
  return ext;
}

/* svgfEncode(handle, inputs + {prevNormalDepth, prevMotion}: BigInt, stream?: BigInt) -> BigInt (svgf.js:343-378) */
static napi_value svgf_encode_js(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc < 2) return throw_msg(env, "SVGF.encode: inputs required");
  svgf_box *b = get_svgf(env, argv[0]);
  if (!b) return NULL;
  svgf_inputs in;
  memset(&in, 0, sizeof in);
  const void **slot[7] = {&in.radiance, &in.normal_depth, &in.motion, &in.material, &in.emission,
                          &in.prev_normal_depth, &in.prev_motion};
  for (int k = 0; k < 7; k++) *slot[k] = (const void *)(uintptr_t)named_bigint(env, argv[1], INPUT_NAMES[k]);
  const uint64_t stream = argc > 2 ? bigint_or_zero(env, argv[2]) : 0;
  const void *out = NULL;
  if (svgf_encode(b->s, &in, (void *)(uintptr_t)stream, &out) != HUSH_OK) return throw_msg(env, svgf_last_error(b->s));
  return make_bigint(env, out);
}

static napi_value svgf_output_js(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  svgf_box *b = argc ? get_svgf(env, argv[0]) : NULL;
  if (!b) return NULL;
  return make_bigint(env, svgf_output(b->s));
}

static napi_value svgf_reset_js(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  svgf_box *b = argc ? get_svgf(env, argv[0]) : NULL;
  if (!b) return NULL;
  if (svgf_reset(b->s) != HUSH_OK) return throw_msg(env, svgf_last_error(b->s));
  return NULL;
}

static napi_value svgf_resize_js(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  double w = 0, h = 0;
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  svgf_box *b = argc ? get_svgf(env, argv[0]) : NULL;
  if (!b) return NULL;
  if (argc < 3 || napi_get_value_double(env, argv[1], &w) != napi_ok || napi_get_value_double(env, argv[2], &h) != napi_ok)
    return throw_msg(env, "SVGF.resize: width and height required");
  if (svgf_resize(b->s, (int)w, (int)h) != HUSH_OK) return throw_msg(env, svgf_last_error(b->s));
  return NULL;
}

static napi_value svgf_destroy_js(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  void *p = NULL;
  CHECK_NAPI(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc && napi_get_value_external(env, argv[0], &p) == napi_ok && p) {
    svgf_box *b = (svgf_box *)p;
    if (b->s) svgf_destroy(b->s);
    b->s = NULL;
  }
  return NULL;
}

static napi_value init(napi_env env, napi_value exports) {
  napi_property_descriptor p[] = {
      {"hushCreate", NULL, hush_create_js, NULL, NULL, NULL, napi_default, NULL},
      {"hushDenoise", NULL, hush_denoise_js, NULL, NULL, NULL, napi_default, NULL},
      {"hushOutput", NULL, hush_output_js, NULL, NULL, NULL, napi_default, NULL},
      {"hushReset", NULL, hush_reset_js, NULL, NULL, NULL, napi_default, NULL},
      {"hushResize", NULL, hush_resize_js, NULL, NULL, NULL, napi_default, NULL},
      {"hushSetExposure", NULL, hush_set_exposure_js, NULL, NULL, NULL, napi_default, NULL},
      {"hushSetWeights", NULL, hush_set_weights_js, NULL, NULL, NULL, napi_default, NULL},
      {"hushDestroy", NULL, hush_destroy_js, NULL, NULL, NULL, napi_default, NULL},
      {"hiddenOf", NULL, hidden_of_js, NULL, NULL, NULL, napi_default, NULL},
      {"requiredLimits", NULL, required_limits_js, NULL, NULL, NULL, napi_default, NULL},
      {"svgfCreate", NULL, svgf_create_js, NULL, NULL, NULL, napi_default, NULL},
      {"svgfEncode", NULL, svgf_encode_js, NULL, NULL, NULL, napi_default, NULL},
      {"svgfOutput", NULL, svgf_output_js, NULL, NULL, NULL, napi_default, NULL},
      {"svgfReset", NULL, svgf_reset_js, NULL, NULL, NULL, napi_default, NULL},
      {"svgfResize", NULL, svgf_resize_js, NULL, NULL, NULL, napi_default, NULL},
      {"svgfDestroy", NULL, svgf_destroy_js, NULL, NULL, NULL, napi_default, NULL},
  };
  if (napi_define_properties(env, exports, sizeof p / sizeof p[0], p) != napi_ok) return NULL;
  return exports;
}

NAPI_MODULE(NODE_GYP_MODULE_NAME, init)
