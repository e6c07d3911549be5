// gtrace_napi.cc — N-API addon: the TypeScript host's binding of the C ABI.
//
// The reference's TypeScript host keeps its PLY loader (src/GS_ply.ts), packer
// (src/GS_packing.ts) and camera (src/camera.ts) and replaces the WebGPU
// ray-tracing pipeline (src/main.ts:469-577) with these calls:
//
//   const gt = require('./build/Release/gtrace_napi.node');
//   const ctx = gt.createContext(0);
//   const scene = gt.createScene(ctx, gsData.gaussiansBuffer, gsData.numGaussians,
//                                gsData.gaussianArrayLayout.size / gsData.numGaussians, alpha_min);
//   gt.traceRays(ctx, scene, uniformData /* the 112-byte ArrayBuffer */, width, height,
//                pixels /* Float32Array(width*height*4) */);
//
// or loads the PLY natively and shows the frame without WebGPU:
//
//   const scene = gt.createSceneFromPly(ctx, plyArrayBuffer, alpha_min);
//   gt.traceRays(ctx, scene, uniformData, width, height, pixels, /*antialias=*/false);
//   gt.toneMap(ctx, pixels, imageData.data /* Uint8ClampedArray */, 0, 1.66);
//
// Only plain N-API (node_api.h) is used.  Errors become JS exceptions carrying
// gt_last_error().  Build with binding.gyp next to this file (node-gyp).
#include <node_api.h>
#include <stdint.h>
#include <string.h>

#include <string>

#include "../../include/gtrace.h"

namespace {

napi_value throw_error(napi_env env, const char* what) {
  napi_throw_error(env, nullptr, what);
  return nullptr;
}

napi_value throw_status(napi_env env, gt_context* ctx, gt_status st) {
  char buf[512];
  gt_last_error(ctx, buf, sizeof buf);
  std::string msg = "gtrace error " + std::to_string(st) + ": " + buf;
  napi_throw_error(env, nullptr, msg.c_str());
  return nullptr;
}

bool get_args(napi_env env, napi_callback_info info, size_t want, napi_value* argv) {
  size_t argc = want;
  if (napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr) != napi_ok || argc < want) {
    napi_throw_type_error(env, nullptr, "wrong number of arguments");
    return false;
  }
  return true;
}

template <class T>
T* get_external(napi_env env, napi_value v) {
  void* p = nullptr;
  if (napi_get_value_external(env, v, &p) != napi_ok) return nullptr;
  return static_cast<T*>(p);
}

// Returns the data pointer and byte length of an ArrayBuffer or TypedArray.
bool get_bytes(napi_env env, napi_value v, void** data, size_t* len) {
  bool is_ab = false, is_ta = false;
  napi_is_arraybuffer(env, v, &is_ab);
  if (is_ab) return napi_get_arraybuffer_info(env, v, data, len) == napi_ok;
  napi_is_typedarray(env, v, &is_ta);
  if (is_ta) {
    napi_typedarray_type type;
    size_t length = 0, offset = 0;
    napi_value ab;
    void* base = nullptr;
    if (napi_get_typedarray_info(env, v, &type, &length, &base, &ab, &offset) != napi_ok) return false;
    size_t elem = (type == napi_float64_array || type == napi_bigint64_array || type == napi_biguint64_array) ? 8
                  : (type == napi_int16_array || type == napi_uint16_array)                                   ? 2
                  : (type == napi_int8_array || type == napi_uint8_array || type == napi_uint8_clamped_array) ? 1
                                                                                                               : 4;
    *data = base;
    *len = length * elem;
    return true;
  }
  return false;
}

uint32_t get_u32(napi_env env, napi_value v) {
  uint32_t x = 0;
  napi_get_value_uint32(env, v, &x);
  return x;
}

napi_value CreateContext(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!get_args(env, info, 1, argv)) return nullptr;
  gt_context* ctx = nullptr;
  gt_status st = gt_context_create((int)get_u32(env, argv[0]), &ctx);
  if (st != GT_OK) return throw_status(env, nullptr, st);
  napi_value out;
  napi_create_external(env, ctx, nullptr, nullptr, &out);
  return out;
}

napi_value DestroyContext(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!get_args(env, info, 1, argv)) return nullptr;
  gt_context_destroy(get_external<gt_context>(env, argv[0]));
  return nullptr;
}

// createScene(ctx, gaussiansBuffer, numGaussians, strideBytes, alphaMin[, activated])
// activated: Float64Array of 8 numbers per Gaussian (opacity, scale xyz,
// rotation wxyz from gsData.gaussianData): the proxies are then built from the
// same double values as the reference's gaussianSceneToBvh.
napi_value CreateScene(napi_env env, napi_callback_info info) {
  napi_value argv[6];
  size_t argc = 6;
  if (napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr) != napi_ok || argc < 5) {
    napi_throw_type_error(env, nullptr, "wrong number of arguments");
    return nullptr;
  }
  gt_context* ctx = get_external<gt_context>(env, argv[0]);
  void* data = nullptr;
  size_t len = 0;
  if (!ctx || !get_bytes(env, argv[1], &data, &len)) return throw_error(env, "createScene: bad arguments");
  uint32_t n = get_u32(env, argv[2]), stride = get_u32(env, argv[3]);
  double alpha_min = 0.0;
  napi_get_value_double(env, argv[4], &alpha_min);
  if ((uint64_t)n * stride > len) return throw_error(env, "createScene: buffer smaller than n * stride");
  void* act = nullptr;
  size_t alen = 0;
  if (argc >= 6 && !get_bytes(env, argv[5], &act, &alen)) return throw_error(env, "createScene: bad activated");
  if (act && alen < (uint64_t)n * 8 * sizeof(double)) return throw_error(env, "createScene: activated too small");
  gt_scene* scene = nullptr;
  gt_status st = gt_scene_create_ex(ctx, data, n, stride, alpha_min, static_cast<const double*>(act), 0, &scene);
  if (st != GT_OK) return throw_status(env, ctx, st);
  napi_value out;
  napi_create_external(env, scene, nullptr, nullptr, &out);
  return out;
}

napi_value DestroyScene(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!get_args(env, info, 1, argv)) return nullptr;
  gt_scene_destroy(get_external<gt_scene>(env, argv[0]));
  return nullptr;
}

// createSceneFromPly(ctx, plyArrayBuffer, alphaMin): loadGaussianSplatting +
// PackedGaussians + gaussianSceneToBvh, decoded and packed natively.
napi_value CreateSceneFromPly(napi_env env, napi_callback_info info) {
  napi_value argv[3];
  if (!get_args(env, info, 3, argv)) return nullptr;
  gt_context* ctx = get_external<gt_context>(env, argv[0]);
  void* data = nullptr;
  size_t len = 0;
  if (!ctx || !get_bytes(env, argv[1], &data, &len)) return throw_error(env, "createSceneFromPly: bad arguments");
  double alpha_min = 0.0;
  napi_get_value_double(env, argv[2], &alpha_min);
  gt_scene* scene = nullptr;
  gt_ply_info pi;
  gt_status st = gt_scene_create_from_ply(ctx, data, len, alpha_min, 0, &scene, &pi);
  if (st != GT_OK) return throw_status(env, ctx, st);
  napi_value out;
  napi_create_external(env, scene, nullptr, nullptr, &out);
  return out;
}

// toneMap(ctx, pixels(Float32Array w*h*4), rgba8(Uint8ClampedArray w*h*4), mode, exposure):
// the display pass of src/toneMapper.ts; rgba8 can back a canvas ImageData.
napi_value ToneMap(napi_env env, napi_callback_info info) {
  napi_value argv[5];
  if (!get_args(env, info, 5, argv)) return nullptr;
  gt_context* ctx = get_external<gt_context>(env, argv[0]);
  void *pix = nullptr, *out = nullptr;
  size_t plen = 0, olen = 0;
  if (!ctx || !get_bytes(env, argv[1], &pix, &plen) || !get_bytes(env, argv[2], &out, &olen))
    return throw_error(env, "toneMap: bad arguments");
  double exposure = 1.66;
  napi_get_value_double(env, argv[4], &exposure);
  const uint64_t n = plen / 16;
  if (n * 4 > olen) return throw_error(env, "toneMap: output buffer too small");
  gt_status st = gt_tonemap(ctx, static_cast<const float*>(pix), n, get_u32(env, argv[3]), (float)exposure,
                            static_cast<uint8_t*>(out), 0);
  if (st != GT_OK) return throw_status(env, ctx, st);
  return nullptr;
}

// traceRays(ctx, scene, uniforms(112 bytes), width, height, pixels(Float32Array w*h*4)[, antialias])
// With antialias true the pixels keep the running average of the frames
// (uniforms.accumulatedFrames counts them), as the reference's shader does
// when its `antialiasing` constant is true.
napi_value TraceRays(napi_env env, napi_callback_info info) {
  napi_value argv[7];
  size_t argc = 7;
  if (napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr) != napi_ok || argc < 6) {
    napi_throw_type_error(env, nullptr, "wrong number of arguments");
    return nullptr;
  }
  bool antialias = false;
  if (argc >= 7) napi_get_value_bool(env, argv[6], &antialias);
  gt_context* ctx = get_external<gt_context>(env, argv[0]);
  gt_scene* scene = get_external<gt_scene>(env, argv[1]);
  void *ub = nullptr, *pix = nullptr;
  size_t ulen = 0, plen = 0;
  if (!ctx || !scene || !get_bytes(env, argv[2], &ub, &ulen) || ulen < sizeof(gt_uniforms) ||
      !get_bytes(env, argv[5], &pix, &plen))
    return throw_error(env, "traceRays: bad arguments");
  uint32_t w = get_u32(env, argv[3]), h = get_u32(env, argv[4]);
  if ((uint64_t)w * h * 16 > plen) return throw_error(env, "traceRays: pixel buffer too small");
  gt_uniforms u;
  memcpy(&u, ub, sizeof u);
  gt_status st = gt_render(ctx, scene, &u, w, h, static_cast<float*>(pix), antialias ? GT_FLAG_ANTIALIAS : 0u,
                           nullptr);
  if (st != GT_OK) return throw_status(env, ctx, st);
  return nullptr;
}

// backward(ctx, scene, uniforms, width, height, dLdrgba(Float32Array), dLdparams(Float32Array 59*n))
napi_value Backward(napi_env env, napi_callback_info info) {
  napi_value argv[7];
  if (!get_args(env, info, 7, argv)) return nullptr;
  gt_context* ctx = get_external<gt_context>(env, argv[0]);
  gt_scene* scene = get_external<gt_scene>(env, argv[1]);
  void *ub = nullptr, *g = nullptr, *out = nullptr;
  size_t ulen = 0, glen = 0, olen = 0;
  if (!ctx || !scene || !get_bytes(env, argv[2], &ub, &ulen) || ulen < sizeof(gt_uniforms) ||
      !get_bytes(env, argv[5], &g, &glen) || !get_bytes(env, argv[6], &out, &olen))
    return throw_error(env, "backward: bad arguments");
  uint32_t w = get_u32(env, argv[3]), h = get_u32(env, argv[4]);
  if ((uint64_t)w * h * 16 > glen) return throw_error(env, "backward: gradient buffer too small");
  gt_scene_info si;
  gt_scene_get_info(scene, &si);
  if (si.n_particles * GT_PARAMS_PER_PARTICLE * 4 > olen) return throw_error(env, "backward: output too small");
  gt_uniforms u;
  memcpy(&u, ub, sizeof u);
  gt_status st = gt_backward(ctx, scene, &u, w, h, static_cast<const float*>(g), static_cast<float*>(out), 0,
                             nullptr, nullptr);
  if (st != GT_OK) return throw_status(env, ctx, st);
  return nullptr;
}

napi_value Init(napi_env env, napi_value exports) {
  napi_property_descriptor props[] = {
      {"createContext", nullptr, CreateContext, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"destroyContext", nullptr, DestroyContext, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"createScene", nullptr, CreateScene, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"destroyScene", nullptr, DestroyScene, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"createSceneFromPly", nullptr, CreateSceneFromPly, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"traceRays", nullptr, TraceRays, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"toneMap", nullptr, ToneMap, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"backward", nullptr, Backward, nullptr, nullptr, nullptr, napi_default, nullptr},
  };
  napi_define_properties(env, exports, sizeof props / sizeof props[0], props);
  return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, Init)
