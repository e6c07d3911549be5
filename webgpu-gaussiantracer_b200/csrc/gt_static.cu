// gt_static.cu — batched render that allocates no memory.
//
// gt_render_batch keeps its per-launch scratch (the tile counter, the
// statistics counters and the device copy of the view table) in buffers the
// context grows with cudaMalloc/cudaHostAlloc on demand.  Some hosts cannot
// allocate while they render: an engine whose frame loop must never stall on
// cudaMalloc/cudaFree (both synchronise the whole device), or a process whose
// GPU memory is owned by another allocator and capped at start-up.  For them,
// gt_render_batch_noalloc runs the same persistent trace kernel with that
// scratch in a fixed array in the library's own device image, so a call
// issues only copies, a memset and the kernel launch.
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>
#include <string>

#include "gt_handles.h"
#include "gt_internal.cuh"

using namespace gt;

namespace {

// Layout of the static scratch: DevCounters at offset 0 (256-byte slot),
// then the view table of up to kNoallocMaxViews entries.
constexpr uint32_t kNoallocMaxViews = 256;
constexpr size_t kCounterSlot = 256;
constexpr size_t kNoallocBytes = kCounterSlot + sizeof(ViewDev) * kNoallocMaxViews;
static_assert(sizeof(DevCounters) <= kCounterSlot, "counter slot too small");
static_assert(kCounterSlot % alignof(ViewDev) == 0, "view table alignment");

// One copy per device that loads the library, held until the process exits.
// In host code this name is only a handle for cudaGetSymbolAddress; kernels
// receive the device address returned by it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on `device` (which must be current).
// The first call per device resolves it with cudaGetSymbolAddress.
cudaError_t noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_ptr[device];
  return cudaSuccess;
}

}  // namespace

extern "C" gt_status gt_render_batch_noalloc(gt_context* ctx, const gt_batch_item* items, uint32_t count,
                                             uint32_t flags, gt_render_stats* stats) {
  if (!ctx) return api_fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (count == 0) return GT_OK;
  if (!items) return api_fail(ctx, GT_ERR_INVALID_ARG, "items is NULL");
  if (count > kNoallocMaxViews)
    return api_fail(ctx, GT_ERR_INVALID_ARG,
                    "gt_render_batch_noalloc takes at most " + std::to_string(kNoallocMaxViews) + " views per call");
  if (!(flags & GT_FLAG_OUTPUT_DEVICE))
    return api_fail(ctx, GT_ERR_INVALID_ARG,
                    "gt_render_batch_noalloc needs device output buffers (GT_FLAG_OUTPUT_DEVICE): host outputs "
                    "would need a staging allocation");
  if (flags & GT_FLAG_CHECKPOINT)
    return api_fail(ctx, GT_ERR_INVALID_ARG,
                    "gt_render_batch_noalloc does not checkpoint: the checkpoint records need an allocation");
  const bool aa = (flags & GT_FLAG_ANTIALIAS) != 0;
  uint32_t total_tiles = 0;
  uint64_t slots_all = 0;
  ViewDev views[kNoallocMaxViews];
  for (uint32_t i = 0; i < count; ++i) {
    const gt_batch_item& it = items[i];
    if (!it.scene || it.scene->ctx != ctx) return api_fail(ctx, GT_ERR_INVALID_ARG, "batch item scene invalid");
    gt_status st = api_check_uniforms(ctx, &it.u);
    if (st != GT_OK) return st;
    if (!it.out_rgba || it.w == 0 || it.h == 0 || (uint64_t)it.w * it.h > (1ull << 31))
      return api_fail(ctx, GT_ERR_INVALID_ARG, "batch item image invalid");
    slots_all += view_slots(it.w, it.h);
    if (slots_all > kMaxSlots) return api_fail(ctx, GT_ERR_INVALID_ARG, "batch larger than 2^31 work slots");
    if (((uintptr_t)it.out_rgba % 16) != 0)
      return api_fail(ctx, GT_ERR_INVALID_ARG, "device out_rgba must be 16-byte aligned");
    views[i] = api_make_view(it.scene, it.u, it.w, it.h, reinterpret_cast<float4*>(it.out_rgba), total_tiles);
    views[i].u.aa = aa ? 1u : 0u;  // jittered sample blended into out_rgba, as gt_render_batch does
    total_tiles += views[i].n_tiles;
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  unsigned char* scratch = nullptr;
  if (e == cudaSuccess) e = noalloc_scratch(ctx->device, &scratch);
  if (e != cudaSuccess)
    return api_fail(ctx, GT_ERR_CUDA, std::string("gt_render_batch_noalloc set-up: ") + cudaGetErrorString(e));
  DevCounters* d_ctr = reinterpret_cast<DevCounters*>(scratch);
  ViewDev* d_views = reinterpret_cast<ViewDev*>(scratch + kCounterSlot);
  // the array keeps the previous call's contents: the counters must start at zero
  e = cudaEventRecord(ctx->call0, ctx->stream);  // the context's own timing events
  if (e == cudaSuccess) e = cudaMemsetAsync(d_ctr, 0, sizeof(DevCounters), ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->int0, ctx->stream);
  if (e != cudaSuccess) return api_fail(ctx, GT_ERR_CUDA, cudaGetErrorString(e));
  LaunchShape shape = api_shape_for(ctx, items[0].scene, items[0].w, items[0].h, items[0].u.k);
  Err err = launch_trace(views, count, total_tiles, d_ctr, ctx->faces, shape, ctx->num_sms, ctx->stream,
                         &ctx->launches, d_views);
  if (err.code != GT_OK) return api_fail(ctx, err.code, err.msg);
  e = cudaEventRecord(ctx->int1, ctx->stream);
  if (e != cudaSuccess) return api_fail(ctx, GT_ERR_CUDA, cudaGetErrorString(e));
  if (flags & GT_FLAG_ASYNC) return GT_OK;
  e = cudaMemcpyAsync(ctx->h_ctr, d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->call1, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return api_fail(ctx, GT_ERR_CUDA, cudaGetErrorString(e));
  if (stats) {
    memset(stats, 0, sizeof *stats);
    api_fill_stats(*ctx->h_ctr, stats);
    cudaEventElapsedTime(&stats->kernel_ms, ctx->int0, ctx->int1);
    cudaEventElapsedTime(&stats->total_ms, ctx->call0, ctx->call1);
  }
  return api_status_to_error(ctx, ctx->h_ctr->status);
}
