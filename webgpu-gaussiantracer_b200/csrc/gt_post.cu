// gt_post.cu — display post-process: the reference's tone-map render pass as
// a CUDA kernel writing a headless RGBA8 buffer.
//
// The reference displays its RGBA-f32 pixel buffer with a full-screen
// fragment shader (src/toneMapper.ts:15-24) into an 8-bit swap-chain texture:
//   hdr = pixelBuffer[x + y * width].xyz
//   ldr = 1 - exp(-exposure * hdr)            (exposure = 1.66)
//   return vec4(hdr, 1)                       (the exposure and the gamma line,
//                                              pow(ldr, 1/2.2), are unused)
// and the swap chain's unorm8 format clamps each channel to [0, 1] and rounds
// c * 255 to the nearest integer.  Three modes cover the shader's active
// path and its two written-out variants:
//   GT_TONEMAP_HDR            unorm8(hdr)                 (what the reference shows)
//   GT_TONEMAP_EXPOSURE       unorm8(1 - exp(-exposure hdr))
//   GT_TONEMAP_EXPOSURE_GAMMA unorm8((1 - exp(-exposure hdr))^(1/2.2))
// exp is this library's deterministic det_expf and x^(1/2.2) is
// det_expf(det_log(x) / 2.2), so the bytes are reproducible on the CPU.
// Alpha is 255.  NaN channels give 0 (unorm conversion of NaN).
//
// One thread per pixel: a 16-byte load and a 4-byte store, both coalesced;
// the kernel is bound by HBM bandwidth (20 bytes per pixel).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "gt_device.cuh"
#include "gt_handles.h"
#include "gt_internal.cuh"

namespace gt {

__device__ __forceinline__ uint32_t to_unorm8(float c) {
  if (!(c > 0.0f)) return 0u;  // also NaN
  if (c >= 1.0f) return 255u;
  return __float2uint_rn(c * 255.0f);
}

__device__ __forceinline__ float tone(float hdr, uint32_t mode, float exposure) {
  if (mode == GT_TONEMAP_HDR) return hdr;
  float ldr = 1.0f - det_expf(-(exposure * hdr));
  if (mode == GT_TONEMAP_EXPOSURE) return ldr;
  if (!(ldr > 0.0f)) return ldr;
  return det_expf((float)(det_log((double)ldr) / 2.2));
}

__global__ void k_tonemap(const float4* __restrict__ rgba, uint64_t n, uint32_t mode, float exposure,
                          uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float4 p = __ldg(rgba + i);
    const uint32_t r = to_unorm8(tone(p.x, mode, exposure));
    const uint32_t g = to_unorm8(tone(p.y, mode, exposure));
    const uint32_t b = to_unorm8(tone(p.z, mode, exposure));
    out[i] = r | (g << 8) | (b << 16) | (255u << 24);
  }
}

}  // namespace gt

using namespace gt;

extern "C" gt_status gt_tonemap(gt_context* ctx, const float* rgba, uint64_t n_pixels, uint32_t mode, float exposure,
                                uint8_t* out_rgba8, uint32_t flags) {
  if (!ctx) return api_fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (n_pixels == 0) return GT_OK;
  if (!rgba || !out_rgba8) return api_fail(ctx, GT_ERR_INVALID_ARG, "rgba or out_rgba8 is NULL");
  if (mode > GT_TONEMAP_EXPOSURE_GAMMA) return api_fail(ctx, GT_ERR_INVALID_ARG, "unknown tone-map mode");
  if ((flags & GT_FLAG_ASYNC) && !((flags & GT_FLAG_INPUT_DEVICE) && (flags & GT_FLAG_OUTPUT_DEVICE)))
    return api_fail(ctx, GT_ERR_INVALID_ARG, "GT_FLAG_ASYNC needs device buffers");
  if ((flags & GT_FLAG_INPUT_DEVICE) && ((uintptr_t)rgba & 15u))
    return api_fail(ctx, GT_ERR_INVALID_ARG, "a device rgba buffer must be 16-byte aligned");
  if ((flags & GT_FLAG_OUTPUT_DEVICE) && ((uintptr_t)out_rgba8 & 3u))
    return api_fail(ctx, GT_ERR_INVALID_ARG, "a device out_rgba8 buffer must be 4-byte aligned");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return api_fail(ctx, GT_ERR_CUDA, cudaGetErrorString(e));
  const float4* src = reinterpret_cast<const float4*>(rgba);
  uint32_t* dst = reinterpret_cast<uint32_t*>(out_rgba8);
  float4* in_tmp = nullptr;
  uint32_t* out_tmp = nullptr;
  auto cleanup = [&]() {
    if (in_tmp) cudaFreeAsync(in_tmp, ctx->stream);
    if (out_tmp) cudaFreeAsync(out_tmp, ctx->stream);
  };
  if (!(flags & GT_FLAG_INPUT_DEVICE)) {
    e = cudaMallocAsync(&in_tmp, n_pixels * sizeof(float4), ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(in_tmp, rgba, n_pixels * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream);
    src = in_tmp;
  }
  if (e == cudaSuccess && !(flags & GT_FLAG_OUTPUT_DEVICE)) {
    e = cudaMallocAsync(&out_tmp, n_pixels * sizeof(uint32_t), ctx->stream);
    dst = out_tmp;
  }
  if (e != cudaSuccess) {
    cleanup();
    cudaStreamSynchronize(ctx->stream);
    return api_fail(ctx, e == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA,
                    std::string("tone map buffers: ") + cudaGetErrorString(e));
  }
  const uint64_t blocks = std::min<uint64_t>((n_pixels + 255) / 256, (uint64_t)ctx->num_sms * 16u);
  k_tonemap<<<(unsigned)blocks, 256, 0, ctx->stream>>>(src, n_pixels, mode, exposure, dst);
  ++ctx->launches;
  e = cudaGetLastError();
  if (e == cudaSuccess && !(flags & GT_FLAG_OUTPUT_DEVICE))
    e = cudaMemcpyAsync(out_rgba8, out_tmp, n_pixels * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream);
  cleanup();
  if (e == cudaSuccess && !(flags & GT_FLAG_ASYNC)) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return api_fail(ctx, GT_ERR_CUDA, std::string("tone map: ") + cudaGetErrorString(e));
  return GT_OK;
}
