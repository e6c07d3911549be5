// gt_handles.h — the library's definitions of the opaque C-ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "gt_internal.cuh"

namespace gt {
constexpr int kEventRing = 256;

struct GraphEntry {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};
}  // namespace gt

namespace gt {
// Checkpoint of the last checkpointing forward of a context (see gt_backward.cu).
struct CkptKey {
  const gt_scene* scene;
  gt_uniforms u;
  uint32_t w, h;
};
struct CkptStore {
  uint32_t* head = nullptr;       // [slots]
  uint32_t* pool = nullptr;       // checkpoint records
  uint32_t* pool_next = nullptr;  // device allocation counter
  size_t head_bytes = 0, pool_bytes = 0;
  uint64_t slots = 0;
  uint32_t pool_cap = 0;          // records that fit
  uint32_t kc = 0;                // particle indices per record (0: replay mode)
  uint32_t mode = 0;              // 1 checkpoint, 2 replay
  uint64_t last_records = 0;      // records the last forward needed
  uint32_t total_tiles = 0;
  bool valid = false;
  std::vector<CkptKey> key;
  float fwd_ms = 0.f;
};
}  // namespace gt

struct gt_context {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  std::string err;
  gt::FaceTable faces;
  gt::DevCounters* d_ctr = nullptr;
  gt::DevCounters* h_ctr = nullptr;  // pinned
  gt::ViewDev* d_views = nullptr;
  uint32_t d_views_cap = 0;
  gt::ViewDev* h_views = nullptr;    // pinned staging for view tables
  uint32_t h_views_cap = 0;
  float4* staging = nullptr;
  size_t staging_bytes = 0;
  // per-view particle colour tables of the render calls (ViewDev::rgb)
  float4* colours = nullptr;
  uint64_t colours_cap = 0;  // float4 entries
  // pinned chunks through which host records are uploaded (double-buffered)
  struct CopyPool* copy_pool = nullptr;  // host threads of the pinned uploads (gt_api.cu)
  unsigned char* up_pinned[2] = {nullptr, nullptr};
  cudaEvent_t up_done[2] = {nullptr, nullptr};
  gt::HandoffRay* d_handoff = nullptr;  // rays tile packets hand to the warp-per-ray kernel
  uint32_t handoff_cap = 0;
  cudaEvent_t call0 = nullptr, call1 = nullptr, timer0 = nullptr, timer1 = nullptr;
  cudaEvent_t int0 = nullptr, int1 = nullptr;  // library-internal timing (never the user's timer)
  cudaEvent_t ring[2 * gt::kEventRing];
  uint64_t ring_head = 0, ring_tail = 0;
  uint64_t launches = 0;
  std::map<std::tuple<uint64_t, uint32_t, uint32_t, uint32_t>, gt_tune_result> tune;
  // gt_autotune_batch results by (views, tiles, k bucket) of a batch
  std::map<std::tuple<uint32_t, uint32_t, uint32_t>, gt_tune_result> batch_tune;
  // batch graphs by (views, tiles, k bucket, blocks per SM, k-buffer slots)
  std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t, uint32_t>, gt::GraphEntry> graphs;
  std::set<gt_scene*> scenes;  // live scenes; destroyed with the context
  gt::CkptStore ckpt;
};

struct gt_scene {
  gt_context* ctx = nullptr;
  gt::SceneBuffers b;
  uint64_t n = 0;
  uint32_t stride = 0;
  double alpha_min = 0.0;
  float build_ms = 0.0f;
  float upload_ms = 0.0f;
};

namespace gt {
// shared by the C-ABI translation units (gt_api.cu)
gt_status api_fail(gt_context* ctx, gt_status code, const std::string& msg);
gt_status api_status_to_error(gt_context* ctx, uint32_t status);
gt_status api_check_uniforms(gt_context* ctx, const gt_uniforms* u);
ViewDev api_make_view(const gt_scene* s, const gt_uniforms& u, uint32_t w, uint32_t h, float4* out,
                      uint32_t tile_begin);
LaunchShape api_shape_for(gt_context* ctx, const gt_scene* s, uint32_t w, uint32_t h, uint32_t k);
// The shape of a batch launch: a gt_autotune_batch result for batches of its
// shape, else the per-view choice of the first view.
LaunchShape api_batch_shape_for(gt_context* ctx, const gt_scene* const* scenes, const gt_uniforms* us,
                                const uint32_t* ws, const uint32_t* hs, uint32_t count, uint32_t total_tiles);
void api_fill_stats(const DevCounters& c, gt_render_stats* st);
gt_status api_ensure_views(gt_context* ctx, uint32_t n);
gt_status api_ensure_handoff(gt_context* ctx, uint64_t rays, Handoff* out);
// Colour tables for the plain-render views of a launch (ViewDev::rgb).
gt_status api_assign_colours(gt_context* ctx, ViewDev* views, uint32_t n);
// Checkpointing forward (gt_backward.cu): renders the views into `outs`
// (device, one per view) and keeps the round checkpoint in ctx->ckpt.
gt_status api_forward_ckpt(gt_context* ctx, const gt_scene* const* scenes, const gt_uniforms* us, const uint32_t* ws,
                           const uint32_t* hs, float4* const* outs, uint32_t count, uint32_t mode, uint32_t cap,
                           uint64_t budget, gt_render_stats* stats);
void api_free_ckpt(gt_context* ctx);
}  // namespace gt
