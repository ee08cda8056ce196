/*
 * kraken_napi.c -- Node.js N-API addon over the drop-in C ABI
 * (include/kraken_b200.h), so that the reference's JavaScript keeps its
 * src/gpu/gpuworld.js surface with CUDA behind it.
 *
 * Exports (each maps one call of gpuworld.js onto the C ABI; a non-zero
 * status becomes a thrown Error carrying kr_last_error's message, as
 * gpuworld.js throws Error with a message, gpuworld.js:43-55, 224-229,
 * 269-271):
 *   deviceCount()                                  isAvailable, gpuworld.js:30-32
 *   create(params, nB, nC, rects, collData, collRange) -> handle
 *                                                  create + writeStatic, gpuworld.js:34-171, 209-247
 *       params: {h, substeps, iterations, linDrag, angDrag, maxSpeed, maxAngSpeed}
 *       rects Float32Array (x y w h), collData Uint32Array (groupCollPoints
 *       order, 4 words per point), collRange Uint32Array (2 x nB)
 *   upload(handle, bodyData, consData, forceData, colorInfo|null)
 *                                                  upload, gpuworld.js:250-298
 *   uploadControls(handle, consData)               uploadControls, gpuworld.js:312-315
 *   step(handle[, n])                              step, gpuworld.js:374-382 (n env steps, default 1)
 *   download(handle, bodyData, consData)           download without the mirror, gpuworld.js:385-396
 *   destroy(handle)                                destroy, gpuworld.js:466-472 (never throws)
 * bodyData / forceData are Float32Array, consData a Float32Array or
 * Uint32Array over the 80 B constraint blocks -- the same buffers the
 * reference's pure packControls / mirrorInto read and write.
 *
 * The handle is a JS External owning one kr_world; a world that JS drops
 * without destroy() is freed by its finalizer.  One JS thread per handle,
 * as in the reference.
 *
 * Build: node-gyp with binding.gyp next to this file (Node's node_api.h),
 * or any C compiler with node_api_decls.h (the declarations of the Node-API
 * functions used here); link against libkraken_b200.so.
 */
#if defined(__has_include)
#if __has_include(<node_api.h>)
#include <node_api.h>
#define KRAKEN_HAVE_NODE_API_H 1
#endif
#endif
#ifndef KRAKEN_HAVE_NODE_API_H
#include "node_api_decls.h"
#endif

#include <stdio.h>
#include <stdlib.h>

#include "kraken_b200.h"

typedef struct {
  kr_world *w;
  uint32_t nB, nC;
} kr_handle;

#define MAX_ARGS 6

/* Throws and returns NULL (the JS call then sees the pending exception). */
static napi_value fail(napi_env env, const char *msg) {
  napi_throw_error(env, NULL, msg);
  return NULL;
}

static napi_value fail_kr(napi_env env, const kr_world *w, int rc) {
  char buf[512];
  snprintf(buf, sizeof(buf), "kraken_b200 status %d: %s", rc, kr_last_error(w));
  return fail(env, buf);
}

static napi_value undefined(napi_env env) {
  napi_value u;
  napi_get_undefined(env, &u);
  return u;
}

static int args(napi_env env, napi_callback_info info, size_t want, napi_value *argv, size_t *argc) {
  *argc = MAX_ARGS;
  if (napi_get_cb_info(env, info, argc, argv, NULL, NULL) != napi_ok) return 0;
  return *argc >= want;
}

/* A typed array of the given element type(s) with at least `min_len`
 * elements: 1 with *data (NULL for an empty array) and *len, or 0 with a
 * thrown Error. */
static int typed(napi_env env, napi_value v, napi_typedarray_type t1, napi_typedarray_type t2, size_t min_len,
                 void **data, size_t *len, const char *what) {
  bool is = false;
  char buf[160];
  if (napi_is_typedarray(env, v, &is) != napi_ok || !is) {
    snprintf(buf, sizeof(buf), "%s: typed array expected", what);
    fail(env, buf);
    return 0;
  }
  napi_typedarray_type t;
  size_t n = 0;
  void *d = NULL;
  if (napi_get_typedarray_info(env, v, &t, &n, &d, NULL, NULL) != napi_ok || (t != t1 && t != t2) || n < min_len ||
      (!d && n)) {
    snprintf(buf, sizeof(buf), "%s: wrong element type or fewer than %zu elements", what, min_len);
    fail(env, buf);
    return 0;
  }
  *data = n ? d : NULL;
  if (len) *len = n;
  return 1;
}

static kr_handle *handle_of(napi_env env, napi_value v) {
  void *p = NULL;
  napi_valuetype t;
  if (napi_typeof(env, v, &t) != napi_ok || t != napi_external || napi_get_value_external(env, v, &p) != napi_ok ||
      !p) {
    fail(env, "not a kraken world handle");
    return NULL;
  }
  return (kr_handle *)p;
}

static kr_handle *live_handle(napi_env env, napi_value v) {
  kr_handle *h = handle_of(env, v);
  if (h && !h->w) {
    fail(env, "kraken world already destroyed");
    return NULL;
  }
  return h;
}

static void finalize_handle(napi_env env, void *data, void *hint) {
  (void)env;
  (void)hint;
  kr_handle *h = (kr_handle *)data;
  if (!h) return;
  kr_destroy(h->w);
  free(h);
}

static int get_num(napi_env env, napi_value obj, const char *name, double *out) {
  napi_value v;
  return napi_get_named_property(env, obj, name, &v) == napi_ok && napi_get_value_double(env, v, out) == napi_ok;
}

static napi_value DeviceCount(napi_env env, napi_callback_info info) {
  (void)info;
  napi_value r;
  napi_create_int32(env, kr_device_count(), &r);
  return r;
}

static napi_value Create(napi_env env, napi_callback_info info) {
  napi_value argv[MAX_ARGS];
  size_t argc;
  if (!args(env, info, 6, argv, &argc)) return fail(env, "create(params, nB, nC, rects, collData, collRange)");
  double h, sub, it, ld, ad, ms, mas;
  if (!get_num(env, argv[0], "h", &h) || !get_num(env, argv[0], "substeps", &sub) ||
      !get_num(env, argv[0], "iterations", &it) || !get_num(env, argv[0], "linDrag", &ld) ||
      !get_num(env, argv[0], "angDrag", &ad) || !get_num(env, argv[0], "maxSpeed", &ms) ||
      !get_num(env, argv[0], "maxAngSpeed", &mas))
    return fail(env, "create: params needs h, substeps, iterations, linDrag, angDrag, maxSpeed, maxAngSpeed");
  uint32_t nB = 0, nC = 0;
  if (napi_get_value_uint32(env, argv[1], &nB) != napi_ok || napi_get_value_uint32(env, argv[2], &nC) != napi_ok)
    return fail(env, "create: nB and nC must be numbers");
  size_t n_rect = 0, n_coll = 0;
  void *rects = NULL, *coll = NULL, *range = NULL;
  if (!typed(env, argv[3], napi_float32_array, napi_float32_array, 4, &rects, &n_rect, "rects") ||
      !typed(env, argv[4], napi_uint32_array, napi_uint32_array, 0, &coll, &n_coll, "collData") ||
      !typed(env, argv[5], napi_uint32_array, napi_uint32_array, 2 * (size_t)nB, &range, NULL, "collRange"))
    return NULL;
  kr_solver_params p;
  p.h = h;
  p.substeps = (int32_t)sub;
  p.iterations = (int32_t)it;
  p.lin_drag = ld;
  p.ang_drag = ad;
  p.max_speed = ms;
  p.max_ang_speed = mas;
  kr_world *w = NULL;
  int rc = kr_create(&p, nB, nC, (const float *)rects, (uint32_t)(n_rect / 4), (const uint32_t *)coll,
                     (uint32_t)(n_coll / 4), (const uint32_t *)range, &w);
  if (rc != KR_OK) return fail_kr(env, NULL, rc);
  kr_handle *hd = (kr_handle *)calloc(1, sizeof(kr_handle));
  if (!hd) {
    kr_destroy(w);
    return fail(env, "create: out of host memory");
  }
  hd->w = w;
  hd->nB = nB;
  hd->nC = nC;
  napi_value ext;
  if (napi_create_external(env, hd, finalize_handle, NULL, &ext) != napi_ok) {
    finalize_handle(env, hd, NULL);
    return fail(env, "create: napi_create_external failed");
  }
  return ext;
}

static napi_value Upload(napi_env env, napi_callback_info info) {
  napi_value argv[MAX_ARGS];
  size_t argc;
  if (!args(env, info, 4, argv, &argc)) return fail(env, "upload(handle, bodyData, consData, forceData, colorInfo)");
  kr_handle *h = live_handle(env, argv[0]);
  if (!h) return NULL;
  void *bd = NULL, *cd = NULL, *fd = NULL, *ci = NULL;
  if (!typed(env, argv[1], napi_float32_array, napi_float32_array, 12 * (size_t)h->nB, &bd, NULL, "bodyData") ||
      !typed(env, argv[2], napi_float32_array, napi_uint32_array, 20 * (size_t)h->nC, &cd, NULL, "consData") ||
      !typed(env, argv[3], napi_float32_array, napi_float32_array, 4 * (size_t)h->nB, &fd, NULL, "forceData"))
    return NULL;
  if (argc > 4) {
    napi_valuetype t;
    napi_typeof(env, argv[4], &t);
    if (t != napi_null && t != napi_undefined &&
        !typed(env, argv[4], napi_uint32_array, napi_uint32_array, 33, &ci, NULL, "colorInfo"))
      return NULL;
  }
  int rc = kr_upload(h->w, (const float *)bd, (const uint32_t *)cd, (const float *)fd, (const uint32_t *)ci);
  if (rc != KR_OK) return fail_kr(env, h->w, rc);
  return undefined(env);
}

static napi_value UploadControls(napi_env env, napi_callback_info info) {
  napi_value argv[MAX_ARGS];
  size_t argc;
  if (!args(env, info, 2, argv, &argc)) return fail(env, "uploadControls(handle, consData)");
  kr_handle *h = live_handle(env, argv[0]);
  if (!h) return NULL;
  if (!h->nC) return undefined(env);
  void *cd = NULL;
  if (!typed(env, argv[1], napi_float32_array, napi_uint32_array, 20 * (size_t)h->nC, &cd, NULL, "consData"))
    return NULL;
  int rc = kr_upload_controls(h->w, (const uint32_t *)cd);
  if (rc != KR_OK) return fail_kr(env, h->w, rc);
  return undefined(env);
}

static napi_value Step(napi_env env, napi_callback_info info) {
  napi_value argv[MAX_ARGS];
  size_t argc;
  if (!args(env, info, 1, argv, &argc)) return fail(env, "step(handle[, n])");
  kr_handle *h = live_handle(env, argv[0]);
  if (!h) return NULL;
  int32_t n = 1;
  if (argc > 1 && napi_get_value_int32(env, argv[1], &n) != napi_ok) return fail(env, "step: n must be a number");
  int rc = kr_step(h->w, n);
  if (rc != KR_OK) return fail_kr(env, h->w, rc);
  return undefined(env);
}

static napi_value Download(napi_env env, napi_callback_info info) {
  napi_value argv[MAX_ARGS];
  size_t argc;
  if (!args(env, info, 3, argv, &argc)) return fail(env, "download(handle, bodyData, consData)");
  kr_handle *h = live_handle(env, argv[0]);
  if (!h) return NULL;
  void *bd = NULL, *cd = NULL;
  if (!typed(env, argv[1], napi_float32_array, napi_float32_array, 12 * (size_t)h->nB, &bd, NULL, "bodyData") ||
      !typed(env, argv[2], napi_float32_array, napi_uint32_array, 20 * (size_t)h->nC, &cd, NULL, "consData"))
    return NULL;
  int rc = kr_download(h->w, (float *)bd, (uint32_t *)cd);
  if (rc != KR_OK) return fail_kr(env, h->w, rc);
  return undefined(env);
}

static napi_value Destroy(napi_env env, napi_callback_info info) {
  napi_value argv[MAX_ARGS];
  size_t argc;
  /* destroy never throws (gpuworld.js:466-472 swallows errors) */
  if (args(env, info, 1, argv, &argc)) {
    void *p = NULL;
    napi_valuetype t;
    if (napi_typeof(env, argv[0], &t) == napi_ok && t == napi_external &&
        napi_get_value_external(env, argv[0], &p) == napi_ok && p) {
      kr_handle *h = (kr_handle *)p;
      kr_destroy(h->w);
      h->w = NULL;
    }
  }
  return undefined(env);
}

static int export_fn(napi_env env, napi_value exports, const char *name, napi_callback cb) {
  napi_value f;
  return napi_create_function(env, name, (size_t)-1, cb, NULL, &f) == napi_ok &&
         napi_set_named_property(env, exports, name, f) == napi_ok;
}

/* The module's entry point (what NAPI_MODULE_INIT defines in node_api.h). */
#ifdef __cplusplus
extern "C"
#endif
__attribute__((visibility("default"))) napi_value napi_register_module_v1(napi_env env, napi_value exports) {
  if (!export_fn(env, exports, "deviceCount", DeviceCount) || !export_fn(env, exports, "create", Create) ||
      !export_fn(env, exports, "upload", Upload) || !export_fn(env, exports, "uploadControls", UploadControls) ||
      !export_fn(env, exports, "step", Step) || !export_fn(env, exports, "download", Download) ||
      !export_fn(env, exports, "destroy", Destroy))
    return fail(env, "kraken_napi: registering the exports failed");
  return exports;
}
