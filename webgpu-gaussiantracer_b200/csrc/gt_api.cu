// gt_api.cu — the C ABI (include/gtrace.h): contexts, scenes, render calls,
// batches, tuning and device helpers.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "gt_handles.h"
#include "gt_internal.cuh"

// Host threads that copy a pageable buffer into a pinned chunk together,
// kept for the context's life: starting threads for every chunk cost about as
// much as a chunk's copy.  The calling thread takes a share as well.
struct CopyPool {
  explicit CopyPool(unsigned workers) {
    for (unsigned t = 0; t < workers; ++t) th_.emplace_back([this, t] { run(t); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> l(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& x : th_) x.join();
  }
  void copy(unsigned char* dst, const unsigned char* src, size_t bytes) {
    if (th_.empty() || bytes < (4u << 20)) {
      memcpy(dst, src, bytes);
      return;
    }
    {
      std::lock_guard<std::mutex> l(m_);
      dst_ = dst;
      src_ = src;
      bytes_ = bytes;
      left_ = (unsigned)th_.size();
      ++gen_;
    }
    cv_.notify_all();
    slice((unsigned)th_.size());
    std::unique_lock<std::mutex> l(m_);
    done_.wait(l, [&] { return left_ == 0; });
  }

 private:
  void slice(unsigned t) {
    const size_t parts = th_.size() + 1, per = (bytes_ + parts - 1) / parts;
    const size_t b = t * per, e = std::min(bytes_, b + per);
    if (b < e) memcpy(dst_ + b, src_ + b, e - b);
  }
  void run(unsigned t) {
    uint64_t seen = 0;
    while (true) {
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      slice(t);
      std::lock_guard<std::mutex> l(m_);
      if (--left_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  unsigned char* dst_ = nullptr;
  const unsigned char* src_ = nullptr;
  size_t bytes_ = 0;
  unsigned left_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};


using namespace gt;

namespace {
thread_local std::string g_last_error;  // errors without a context
}  // namespace

// ----------------------------------------------------------------- helpers
static gt_status fail(gt_context* ctx, gt_status code, const std::string& msg) {
  // a failed runtime call also stays behind as the thread's last error; read
  // it here so that the next launch check does not report it a second time
  (void)cudaGetLastError();
  if (ctx)
    ctx->err = msg;
  else
    g_last_error = msg;
  return code;
}
static gt_status fail(gt_context* ctx, const Err& e) { return fail(ctx, e.code, e.msg); }

// A failing runtime call also leaves its error as the thread's last error;
// it is read back here so that a later launch check does not report it again.
#define API_CUDA(ctx, expr)                                                                        \
  do {                                                                                             \
    cudaError_t e_ = (expr);                                                                       \
    if (e_ != cudaSuccess) {                                                                       \
      (void)cudaGetLastError();                                                                    \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA,                 \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                             \
    }                                                                                              \
  } while (0)

static gt_status status_to_error(gt_context* ctx, uint32_t status) {
  if (status & kStatusStackOverflow) return fail(ctx, GT_ERR_STACK_OVERFLOW, "traversal stack overflow");
  if (status & (kStatusVisitCap | kStatusRoundCap))
    return fail(ctx, GT_ERR_DEVICE_TIMEOUT, "a device loop reached its iteration limit");
  if (status & kStatusCheckpointFull) return fail(ctx, GT_ERR_DEVICE_TIMEOUT, "checkpoint capacity exceeded");
  if (status & kStatusHitOverflow) return fail(ctx, GT_ERR_CUDA, "internal error: too many hits on one proxy");
  return GT_OK;
}

static gt_status check_uniforms(gt_context* ctx, const gt_uniforms* u) {
  if (!u) return fail(ctx, GT_ERR_INVALID_ARG, "uniforms is NULL");
  if (u->debug_mode > 2) return fail(ctx, GT_ERR_INVALID_ARG, "debug_mode must be 0, 1 or 2");
  if (u->debug_mode == 0 && (u->k == 0 || u->k > 32))
    return fail(ctx, GT_ERR_INVALID_ARG, "k (hit_array_size) must be in 1..32");
  return GT_OK;
}

static void drop_graphs(gt_context* ctx) {
  for (auto& kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->graphs.clear();
}

// Handoff buffer for a launch of `rays` rays: room for a quarter of them, at
// most 4M rays (128 MB); a packet whose rays do not fit keeps tracing them
// itself, so the cap changes only how the tail of a large batch is shared.
static gt_status ensure_handoff(gt_context* ctx, uint64_t rays, Handoff* out) {
  const uint64_t want64 = std::max<uint64_t>(4096, rays / 4);
  const uint32_t want = (uint32_t)std::min<uint64_t>(want64, 1u << 22);
  if (want > ctx->handoff_cap) {
    // captured graphs hold the old buffer address
    cudaStreamSynchronize(ctx->stream);
    drop_graphs(ctx);
    cudaFree(ctx->d_handoff);
    ctx->d_handoff = nullptr;
    ctx->handoff_cap = 0;
    API_CUDA(ctx, cudaMalloc(&ctx->d_handoff, sizeof(HandoffRay) * (size_t)want));
    ctx->handoff_cap = want;
  }
  out->rays = ctx->d_handoff;
  out->cap = ctx->handoff_cap;
  return GT_OK;
}

static gt_status ensure_views(gt_context* ctx, uint32_t n) {
  if (n > ctx->d_views_cap || n > ctx->h_views_cap) {
    // captured graphs hold the old table addresses
    cudaStreamSynchronize(ctx->stream);
    drop_graphs(ctx);
  }
  if (n > ctx->d_views_cap) {
    cudaFree(ctx->d_views);
    ctx->d_views = nullptr;
    uint32_t cap = std::max<uint32_t>(n, 2 * ctx->d_views_cap);
    API_CUDA(ctx, cudaMalloc(&ctx->d_views, sizeof(ViewDev) * cap));
    ctx->d_views_cap = cap;
  }
  if (n > ctx->h_views_cap) {
    cudaFreeHost(ctx->h_views);
    ctx->h_views = nullptr;
    uint32_t cap = std::max<uint32_t>(n, 2 * ctx->h_views_cap);
    API_CUDA(ctx, cudaHostAlloc((void**)&ctx->h_views, sizeof(ViewDev) * cap, cudaHostAllocDefault));
    ctx->h_views_cap = cap;
  }
  return GT_OK;
}

static gt_status ensure_staging(gt_context* ctx, size_t bytes) {
  if (bytes > ctx->staging_bytes) {
    cudaFree(ctx->staging);
    ctx->staging = nullptr;
    ctx->staging_bytes = 0;
    API_CUDA(ctx, cudaMalloc(&ctx->staging, bytes));
    ctx->staging_bytes = bytes;
  }
  return GT_OK;
}

// Gives every plain-render view of a launch its own particle colour table
// (ViewDev::rgb, filled by k_view_colours before the trace kernels) in the
// context's colour buffer, grown as needed.  A launch whose tables would
// take more than kColourBudget bytes, or that has more views than a grid has
// rows, keeps the per-entry evaluation (same image bits either way).
constexpr uint64_t kColourBudget = 2ull << 30;
static gt_status assign_colours(gt_context* ctx, ViewDev* views, uint32_t n) {
  uint64_t need = 0;
  for (uint32_t i = 0; i < n; ++i) {
    views[i].rgb = nullptr;
    if (views[i].u.debug == 0) need += views[i].n_particles;
  }
  if (need == 0 || n > 65535u || need * sizeof(float4) > kColourBudget) return GT_OK;
  if (need > ctx->colours_cap) {
    API_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->colours);
    ctx->colours = nullptr;
    ctx->colours_cap = 0;
    if (cudaMalloc(&ctx->colours, need * sizeof(float4)) != cudaSuccess) {
      (void)cudaGetLastError();
      ctx->colours = nullptr;
      return GT_OK;  // (no room: the per-entry evaluation)
    }
    ctx->colours_cap = need;
  }
  uint64_t at = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (views[i].u.debug != 0) continue;
    views[i].rgb = ctx->colours + at;
    at += views[i].n_particles;
  }
  return GT_OK;
}

static SceneDev scene_dev(const gt_scene* s) {
  SceneDev d;
  d.nodes8 = s->b.nodes8;
  d.w2o = s->b.w2o;
  d.leaf_pidx = s->b.leaf_pidx;
  d.shade = s->b.shade;
  d.sh = s->b.sh;
  d.params = s->b.params;
  d.root = s->b.root;
  d.n_kept = (uint32_t)s->b.n_kept;
  d.n_sh = s->b.n_sh;
  d.scene_mag = s->b.scene_mag;
  return d;
}

static ViewDev make_view(const gt_scene* s, const gt_uniforms& u, uint32_t w, uint32_t h, float4* out,
                         uint32_t tile_begin) {
  ViewDev v;
  memset(&v, 0, sizeof v);
  v.u = to_ray_uniforms(u);
  v.s = scene_dev(s);
  v.out = out;
  v.w = w;
  v.h = h;
  // the tile grid in whole blocks of 16 x 16 tiles (see tile_pixel)
  v.tiles_x = ((w + 7) / 8 + 15) / 16 * 16;
  v.n_tiles = v.tiles_x * (((h + 3) / 4 + 15) / 16 * 16);
  v.tile_begin = tile_begin;
  v.n_particles = s->n;
  v.kbuf = 32;
  v.leaf_batch = 32;
  return v;
}

namespace gt {
gt_status api_fail(gt_context* ctx, gt_status code, const std::string& msg) { return fail(ctx, code, msg); }
gt_status api_status_to_error(gt_context* ctx, uint32_t status) { return status_to_error(ctx, status); }
gt_status api_check_uniforms(gt_context* ctx, const gt_uniforms* u) { return check_uniforms(ctx, u); }
ViewDev api_make_view(const gt_scene* s, const gt_uniforms& u, uint32_t w, uint32_t h, float4* out,
                      uint32_t tile_begin) {
  return make_view(s, u, w, h, out, tile_begin);
}
}  // namespace gt

static uint64_t ring_slot(gt_context* ctx) { return (ctx->ring_head++) % kEventRing; }

static void fill_stats(const DevCounters& c, gt_render_stats* st) {
  st->rays = c.rays;
  st->rounds = c.rounds;
  st->entries = c.entries;
  st->contributing = c.contributing;
  st->proxy_tests = c.proxy_tests;
  st->node_visits = c.node_visits;
  st->anyhits = c.anyhits;
  st->status_flags = c.status;
  st->handed = c.handoff;
}

static std::tuple<uint64_t, uint32_t, uint32_t, uint32_t> tune_key(const gt_scene* s, uint32_t w, uint32_t h,
                                                                   uint32_t k) {
  return std::make_tuple((uint64_t)(s ? (uint64_t)log2((double)std::max<uint64_t>(s->b.n_kept, 1)) : 0),
                         (uint32_t)log2((double)std::max<uint64_t>((uint64_t)w * h, 1)), kmax_for(k), 0u);
}

// The launch shape a tuning result stands for.
static LaunchShape shape_of(const gt_tune_result& r) {
  LaunchShape sh;
  // block_threads 32: tile packets with this k-buffer; 128: a warp per ray
  sh.packet = r.block_threads == 32 ? 1u : 0u;
  if (sh.packet)
    sh.packet_kbuf = r.kbuf;
  else
    sh.kbuf = r.kbuf;
  sh.blocks_per_sm = r.blocks_per_sm;
  sh.leaf_batch = r.leaf_batch;
  if (r.handoff_after) sh.handoff_after = r.handoff_after;
  return sh;
}

static LaunchShape shape_for(gt_context* ctx, const gt_scene* s, uint32_t w, uint32_t h, uint32_t k) {
  auto it = ctx->tune.find(tune_key(s, w, h, k));
  return it != ctx->tune.end() ? shape_of(it->second) : LaunchShape();
}

namespace gt {
LaunchShape api_shape_for(gt_context* ctx, const gt_scene* s, uint32_t w, uint32_t h, uint32_t k) {
  return shape_for(ctx, s, w, h, k);
}
LaunchShape api_batch_shape_for(gt_context* ctx, const gt_scene* const* scenes, const gt_uniforms* us,
                                const uint32_t* ws, const uint32_t* hs, uint32_t count, uint32_t total_tiles) {
  uint32_t kmax = 8;
  for (uint32_t i = 0; i < count; ++i) kmax = std::max(kmax, kmax_for(us[i].k));
  auto bt = ctx->batch_tune.find(std::make_tuple(count, total_tiles, kmax));
  return bt != ctx->batch_tune.end() ? shape_of(bt->second) : shape_for(ctx, scenes[0], ws[0], hs[0], us[0].k);
}
void api_fill_stats(const DevCounters& c, gt_render_stats* st) { fill_stats(c, st); }
gt_status api_ensure_views(gt_context* ctx, uint32_t n) { return ensure_views(ctx, n); }
gt_status api_ensure_handoff(gt_context* ctx, uint64_t rays, Handoff* out) { return ensure_handoff(ctx, rays, out); }
gt_status api_assign_colours(gt_context* ctx, ViewDev* views, uint32_t n) { return assign_colours(ctx, views, n); }
}  // namespace gt

// ============================================================== context
extern "C" uint32_t gt_version(void) { return GT_ABI_VERSION; }

extern "C" gt_status gt_context_create(int device, gt_context** out) {
  if (!out) return fail(nullptr, GT_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(nullptr, GT_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= count) return fail(nullptr, GT_ERR_NO_DEVICE, "device ordinal out of range");
  gt_context* ctx = new gt_context();
  ctx->device = device;
  memset(ctx->ring, 0, sizeof ctx->ring);
#define CTX_TRY(expr)                                                           \
  do {                                                                          \
    cudaError_t e2 = (expr);                                                    \
    if (e2 != cudaSuccess) {                                                    \
      std::string m = std::string(#expr) + ": " + cudaGetErrorString(e2);      \
      gt_context_destroy(ctx);                                                  \
      return fail(nullptr, e2 == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA, m); \
    }                                                                           \
  } while (0)
  CTX_TRY(cudaSetDevice(device));
  CTX_TRY(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
  CTX_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  {
    // keep stream-ordered temporaries (scene builds, adjoint checkpoints) cached
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  CTX_TRY(cudaMalloc(&ctx->d_ctr, sizeof(DevCounters)));
  CTX_TRY(cudaHostAlloc((void**)&ctx->h_ctr, sizeof(DevCounters), cudaHostAllocDefault));
  CTX_TRY(cudaEventCreate(&ctx->call0));
  CTX_TRY(cudaEventCreate(&ctx->call1));
  CTX_TRY(cudaEventCreate(&ctx->timer0));
  CTX_TRY(cudaEventCreate(&ctx->timer1));
  CTX_TRY(cudaEventCreate(&ctx->int0));
  CTX_TRY(cudaEventCreate(&ctx->int1));
  for (int i = 0; i < 2 * kEventRing; ++i) CTX_TRY(cudaEventCreate(&ctx->ring[i]));
#undef CTX_TRY
  make_face_table(&ctx->faces);
  if (ctx->faces.npairs != 10) {
    gt_context_destroy(ctx);
    return fail(nullptr, GT_ERR_CUDA, "internal error: icosahedron face table has no antipodal pairing");
  }
  *out = ctx;
  return GT_OK;
}

extern "C" gt_status gt_context_destroy(gt_context* ctx) {
  if (!ctx) return GT_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  drop_graphs(ctx);
  api_free_ckpt(ctx);
  for (gt_scene* s : ctx->scenes) {
    free_scene(&s->b, ctx->stream);
    delete s;
  }
  ctx->scenes.clear();
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);  // the frees are stream-ordered
  cudaFree(ctx->d_ctr);
  cudaFreeHost(ctx->h_ctr);
  cudaFree(ctx->d_views);
  cudaFree(ctx->d_handoff);
  cudaFreeHost(ctx->h_views);
  cudaFree(ctx->staging);
  cudaFree(ctx->colours);
  delete ctx->copy_pool;
  for (int b = 0; b < 2; ++b) {
    if (ctx->up_pinned[b]) cudaFreeHost(ctx->up_pinned[b]);
    if (ctx->up_done[b]) cudaEventDestroy(ctx->up_done[b]);
  }
  for (cudaEvent_t ev : {ctx->call0, ctx->call1, ctx->timer0, ctx->timer1, ctx->int0, ctx->int1})
    if (ev) cudaEventDestroy(ev);
  for (int i = 0; i < 2 * kEventRing; ++i)
    if (ctx->ring[i]) cudaEventDestroy(ctx->ring[i]);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return GT_OK;
}

extern "C" gt_status gt_last_error(const gt_context* ctx, char* buf, size_t len) {
  if (!buf || len == 0) return GT_ERR_INVALID_ARG;
  const std::string& m = ctx ? ctx->err : g_last_error;
  size_t n = std::min(len - 1, m.size());
  memcpy(buf, m.data(), n);
  buf[n] = 0;
  return GT_OK;
}

// ================================================================ scene
// Host-to-device copy of a host buffer through two pinned 16 MB chunks of the
// context: the host copies chunk i into one pinned buffer (several threads)
// while the DMA engine moves chunk i-1 out of the other, so a pageable
// source streams at close to host memcpy speed instead of the driver's
// staged pageable copy.  Each chunk is one cudaMemcpyAsync on the context
// stream.
constexpr size_t kUploadChunk = 16u << 20;

static gt_status upload_host(gt_context* ctx, void* dst_dev, const void* src_host, size_t bytes) {
  if (bytes == 0) return GT_OK;
  if (!ctx->copy_pool) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    ctx->copy_pool = new CopyPool(std::min(hw, 8u) - 1);
  }
  for (int b = 0; b < 2; ++b) {
    if (!ctx->up_pinned[b])
      API_CUDA(ctx, cudaHostAlloc((void**)&ctx->up_pinned[b], kUploadChunk, cudaHostAllocDefault));
    if (!ctx->up_done[b]) API_CUDA(ctx, cudaEventCreateWithFlags(&ctx->up_done[b], cudaEventDisableTiming));
  }
  const unsigned char* src = static_cast<const unsigned char*>(src_host);
  unsigned char* dst = static_cast<unsigned char*>(dst_dev);
  for (size_t off = 0, i = 0; off < bytes; off += kUploadChunk, ++i) {
    const int b = (int)(i & 1);
    const size_t len = std::min(kUploadChunk, bytes - off);
    API_CUDA(ctx, cudaEventSynchronize(ctx->up_done[b]));  // the chunk's previous copy has left
    ctx->copy_pool->copy(ctx->up_pinned[b], src + off, len);
    API_CUDA(ctx, cudaMemcpyAsync(dst + off, ctx->up_pinned[b], len, cudaMemcpyHostToDevice, ctx->stream));
    API_CUDA(ctx, cudaEventRecord(ctx->up_done[b], ctx->stream));
  }
  return GT_OK;
}

extern "C" gt_status gt_scene_create(gt_context* ctx, const void* packed, uint64_t n, uint32_t stride_bytes,
                                     double alpha_min, uint32_t flags, gt_scene** out) {
  return gt_scene_create_ex(ctx, packed, n, stride_bytes, alpha_min, nullptr, flags, out);
}

extern "C" gt_status gt_scene_create_ex(gt_context* ctx, const void* packed, uint64_t n, uint32_t stride_bytes,
                                        double alpha_min, const double* activated, uint32_t flags, gt_scene** out) {
  if (!ctx) return fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (!out) return fail(ctx, GT_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (n > 0 && !packed) return fail(ctx, GT_ERR_INVALID_ARG, "packed buffer is NULL");
  if (stride_bytes < 64 || stride_bytes % 4 != 0)
    return fail(ctx, GT_ERR_INVALID_ARG, "stride_bytes must be a multiple of 4 and at least 64");
  if (!(alpha_min > 0.0) || !(alpha_min < 1.0))
    return fail(ctx, GT_ERR_INVALID_ARG, "alpha_min must be in (0, 1)");
  if (n >= (1ull << 31)) return fail(ctx, GT_ERR_INVALID_ARG, "at most 2^31 - 1 particles");
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  const void* dev = packed;
  void* tmp = nullptr;
  double* act_tmp = nullptr;
  // stream-ordered temporaries (the context's pool keeps their memory cached)
  auto drop_tmps = [&]() {
    if (tmp) cudaFreeAsync(tmp, ctx->stream);
    if (act_tmp) cudaFreeAsync(act_tmp, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
  };
  const auto up0 = std::chrono::steady_clock::now();
  if (n > 0 && !(flags & GT_FLAG_INPUT_DEVICE)) {
    API_CUDA(ctx, cudaMallocAsync(&tmp, n * (uint64_t)stride_bytes, ctx->stream));
    gt_status ust = upload_host(ctx, tmp, packed, n * (uint64_t)stride_bytes);
    if (ust != GT_OK) {
      drop_tmps();
      return ust;
    }
    dev = tmp;
  }
  const double* act = activated;
  if (n > 0 && activated && !(flags & GT_FLAG_INPUT_DEVICE)) {
    cudaError_t e = cudaMallocAsync((void**)&act_tmp, n * 8 * sizeof(double), ctx->stream);
    if (e != cudaSuccess) {
      act_tmp = nullptr;
      drop_tmps();
      return fail(ctx, e == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA,
                  std::string("upload of the activated values: ") + cudaGetErrorString(e));
    }
    gt_status ust = upload_host(ctx, act_tmp, activated, n * 8 * sizeof(double));
    if (ust != GT_OK) {
      drop_tmps();
      return ust;
    }
    act = act_tmp;
  }
  const float upload_ms =
      std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - up0).count();
  gt_scene* s = new gt_scene();
  s->ctx = ctx;
  s->n = n;
  s->stride = stride_bytes;
  s->alpha_min = alpha_min;
  cudaEventRecord(ctx->call0, ctx->stream);
  Err e = build_scene(dev, n, stride_bytes, alpha_min, ctx->stream, &s->b, &ctx->launches,
                      (flags & GT_FLAG_FAST_BUILD) != 0, act);
  cudaEventRecord(ctx->call1, ctx->stream);
  drop_tmps();
  if (e.code != GT_OK) {
    free_scene(&s->b, ctx->stream);
    delete s;
    return fail(ctx, e);
  }
  cudaEventElapsedTime(&s->build_ms, ctx->call0, ctx->call1);
  s->upload_ms = upload_ms;
  ctx->scenes.insert(s);
  *out = s;
  return GT_OK;
}

extern "C" gt_status gt_scene_destroy(gt_scene* s) {
  if (!s) return GT_OK;
  gt_context* ctx = s->ctx;
  if (!ctx->scenes.count(s)) return fail(ctx, GT_ERR_INVALID_ARG, "scene already destroyed");
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->scenes.erase(s);
  free_scene(&s->b, ctx->stream);
  delete s;
  return GT_OK;
}

extern "C" gt_status gt_scene_export_bvh(const gt_scene* s, void* nodes8, uint64_t nodes_bytes, uint32_t* leaf_pidx,
                                        uint64_t leaf_count, gt_bvh_info* info) {
  if (!s) return fail(nullptr, GT_ERR_INVALID_ARG, "scene is NULL");
  gt_context* ctx = s->ctx;
  if (!info) return fail(ctx, GT_ERR_INVALID_ARG, "info is NULL");
  memset(info, 0, sizeof *info);
  info->n_nodes8 = s->b.n_nodes8;
  info->n_leaves = (uint32_t)s->b.n_kept;
  info->root = s->b.root;
  info->depth = s->b.depth;
  const uint64_t nb = (uint64_t)s->b.n_nodes8 * 16 * sizeof(float4);
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  API_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (nodes8) {
    if (nodes_bytes < nb) return fail(ctx, GT_ERR_INVALID_ARG, "nodes8 buffer smaller than n_nodes8 * 256 bytes");
    if (nb) API_CUDA(ctx, cudaMemcpy(nodes8, s->b.nodes8, nb, cudaMemcpyDeviceToHost));
  }
  if (leaf_pidx) {
    if (leaf_count < s->b.n_kept) return fail(ctx, GT_ERR_INVALID_ARG, "leaf_pidx smaller than the leaf count");
    if (s->b.n_kept) API_CUDA(ctx, cudaMemcpy(leaf_pidx, s->b.leaf_pidx, s->b.n_kept * 4, cudaMemcpyDeviceToHost));
  }
  return GT_OK;
}

extern "C" gt_status gt_scene_get_info(const gt_scene* s, gt_scene_info* info) {
  if (!s || !info) return GT_ERR_INVALID_ARG;
  memset(info, 0, sizeof *info);
  info->n_particles = s->n;
  info->n_kept = s->b.n_kept;
  info->device_bytes = s->b.bytes;
  info->bvh_depth = s->b.depth;
  info->build_ms = s->build_ms;
  info->upload_ms = s->upload_ms;
  for (int a = 0; a < 6; ++a) info->bounds[a] = s->b.bounds[a];
  return GT_OK;
}

// =============================================================== render
static gt_status finish_call(gt_context* ctx, gt_render_stats* stats, uint64_t kslot) {
  API_CUDA(ctx, cudaMemcpyAsync(ctx->h_ctr, ctx->d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, ctx->stream));
  API_CUDA(ctx, cudaEventRecord(ctx->call1, ctx->stream));
  API_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (stats) {
    memset(stats, 0, sizeof *stats);
    fill_stats(*ctx->h_ctr, stats);
    cudaEventElapsedTime(&stats->kernel_ms, ctx->ring[2 * kslot], ctx->ring[2 * kslot + 1]);
    cudaEventElapsedTime(&stats->total_ms, ctx->call0, ctx->call1);
  }
  return status_to_error(ctx, ctx->h_ctr->status);
}

extern "C" gt_status gt_render(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u, uint32_t w, uint32_t h,
                               float* out_rgba, uint32_t flags, gt_render_stats* stats) {
  if (!ctx) return fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (!scene || scene->ctx != ctx) return fail(ctx, GT_ERR_INVALID_ARG, "scene is NULL or from another context");
  gt_status st = check_uniforms(ctx, u);
  if (st != GT_OK) return st;
  if (!out_rgba) return fail(ctx, GT_ERR_INVALID_ARG, "out_rgba is NULL");
  if (w == 0 || h == 0 || (uint64_t)w * h > (1ull << 31) || view_slots(w, h) > kMaxSlots)
    return fail(ctx, GT_ERR_INVALID_ARG, "bad image size");
  if ((flags & GT_FLAG_ASYNC) && !(flags & GT_FLAG_OUTPUT_DEVICE))
    return fail(ctx, GT_ERR_INVALID_ARG, "GT_FLAG_ASYNC needs a device output buffer");
  if ((flags & GT_FLAG_OUTPUT_DEVICE) && ((uintptr_t)out_rgba % 16) != 0)
    return fail(ctx, GT_ERR_INVALID_ARG, "device out_rgba must be 16-byte aligned");
  const bool aa = (flags & GT_FLAG_ANTIALIAS) != 0;
  if (aa && (flags & GT_FLAG_CHECKPOINT))
    return fail(ctx, GT_ERR_INVALID_ARG, "GT_FLAG_ANTIALIAS renders are not checkpointed");
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  size_t bytes = (size_t)w * h * sizeof(float4);
  float4* out = reinterpret_cast<float4*>(out_rgba);
  // A page-locked host buffer of this GPU (cudaHostAlloc, cudaMallocHost or
  // cudaHostRegister with a device mapping) is written by the trace kernels
  // directly: each tile's pixels cross the host link when the tile is done,
  // instead of the whole image in one copy after the render.  Anti-aliased
  // frames (which read the previous average) and checkpointing renders take
  // the staging buffer.
  bool direct = false;
  if (!(flags & GT_FLAG_OUTPUT_DEVICE) && !aa && !(flags & GT_FLAG_CHECKPOINT)) {
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, out_rgba) == cudaSuccess) {
      if (pa.type == cudaMemoryTypeHost && pa.device == ctx->device && pa.devicePointer &&
          (uintptr_t)pa.devicePointer % 16 == 0) {
        out = reinterpret_cast<float4*>(pa.devicePointer);
        direct = true;
      }
    } else {
      (void)cudaGetLastError();  // (an unknown pointer: the staging path)
    }
  }
  if (!(flags & GT_FLAG_OUTPUT_DEVICE) && !direct) {
    st = ensure_staging(ctx, bytes);
    if (st != GT_OK) return st;
    out = ctx->staging;
    // the running average of the earlier frames is blended on the device
    if (aa && u->accumulated_frames != 0)
      API_CUDA(ctx, cudaMemcpyAsync(out, out_rgba, bytes, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (flags & GT_FLAG_CHECKPOINT) {
    if (flags & GT_FLAG_ASYNC) return fail(ctx, GT_ERR_INVALID_ARG, "a checkpointing render is synchronous");
    if (u->debug_mode != 0) return fail(ctx, GT_ERR_INVALID_ARG, "checkpointing needs debug_mode 0");
    API_CUDA(ctx, cudaEventRecord(ctx->call0, ctx->stream));
    st = api_forward_ckpt(ctx, &scene, u, &w, &h, &out, 1, 0, 0, 0, stats);
    if (st != GT_OK) return st;
    if (!(flags & GT_FLAG_OUTPUT_DEVICE))
      API_CUDA(ctx, cudaMemcpyAsync(out_rgba, out, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    API_CUDA(ctx, cudaEventRecord(ctx->call1, ctx->stream));
    API_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (stats) cudaEventElapsedTime(&stats->total_ms, ctx->call0, ctx->call1);
    return GT_OK;
  }
  st = ensure_views(ctx, 1);
  if (st != GT_OK) return st;
  ViewDev v = make_view(scene, *u, w, h, out, 0);
  v.u.aa = aa ? 1u : 0u;
  st = assign_colours(ctx, &v, 1);
  if (st != GT_OK) return st;
  API_CUDA(ctx, cudaEventRecord(ctx->call0, ctx->stream));
  API_CUDA(ctx, cudaMemsetAsync(ctx->d_ctr, 0, sizeof(DevCounters), ctx->stream));
  uint64_t slot = ring_slot(ctx);
  API_CUDA(ctx, cudaEventRecord(ctx->ring[2 * slot], ctx->stream));
  LaunchShape shape = shape_for(ctx, scene, w, h, u->k);
  Handoff hand;
  st = ensure_handoff(ctx, (uint64_t)w * h, &hand);
  if (st != GT_OK) return st;
  Err e = launch_trace(&v, 1, v.n_tiles, ctx->d_ctr, ctx->faces, shape, ctx->num_sms, ctx->stream, &ctx->launches,
                       ctx->d_views, nullptr, &hand);
  if (e.code != GT_OK) return fail(ctx, e);
  API_CUDA(ctx, cudaEventRecord(ctx->ring[2 * slot + 1], ctx->stream));
  if (!(flags & GT_FLAG_OUTPUT_DEVICE) && !direct)
    API_CUDA(ctx, cudaMemcpyAsync(out_rgba, out, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (flags & GT_FLAG_ASYNC) return GT_OK;
  return finish_call(ctx, stats, slot);
}

extern "C" gt_status gt_render_hits(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u, uint32_t w,
                                    uint32_t h, const uint32_t* pixels, uint32_t n_pix, uint32_t max_entries,
                                    uint32_t* out_pidx, float* out_t, float* out_alpha, uint32_t* out_count,
                                    uint32_t* out_rounds, float* out_rgba) {
  if (!ctx) return fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (!scene || scene->ctx != ctx) return fail(ctx, GT_ERR_INVALID_ARG, "scene is NULL or from another context");
  gt_status st = check_uniforms(ctx, u);
  if (st != GT_OK) return st;
  if (w == 0 || h == 0 || (uint64_t)w * h > (1ull << 31) || view_slots(w, h) > kMaxSlots)
    return fail(ctx, GT_ERR_INVALID_ARG, "bad image size");
  if (n_pix == 0) return GT_OK;
  if (!pixels || !out_count || !out_rounds || (max_entries > 0 && (!out_pidx || !out_t || !out_alpha)))
    return fail(ctx, GT_ERR_INVALID_ARG, "NULL output buffer");
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  size_t me = std::max<uint32_t>(max_entries, 1);
  // one allocation cut into parts that each start on a 256-byte boundary
  // (the float4 part needs 16; n_pix is arbitrary)
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t o_rgba = 0, o_pix = up(o_rgba + (size_t)n_pix * 16), o_pidx = up(o_pix + (size_t)n_pix * 4);
  const size_t o_t = up(o_pidx + (size_t)n_pix * me * 4), o_alpha = up(o_t + (size_t)n_pix * me * 4);
  const size_t o_count = up(o_alpha + (size_t)n_pix * me * 4), o_rounds = up(o_count + (size_t)n_pix * 4);
  const size_t bytes = o_rounds + (size_t)n_pix * 4;
  uint8_t* buf = nullptr;
  API_CUDA(ctx, cudaMalloc(&buf, bytes));
  float4* d_rgba = reinterpret_cast<float4*>(buf + o_rgba);
  uint32_t* d_pix = reinterpret_cast<uint32_t*>(buf + o_pix);
  uint32_t* d_pidx = reinterpret_cast<uint32_t*>(buf + o_pidx);
  float* d_t = reinterpret_cast<float*>(buf + o_t);
  float* d_alpha = reinterpret_cast<float*>(buf + o_alpha);
  uint32_t* d_count = reinterpret_cast<uint32_t*>(buf + o_count);
  uint32_t* d_rounds = reinterpret_cast<uint32_t*>(buf + o_rounds);
  ViewDev v = make_view(scene, *u, w, h, nullptr, 0);
  gt_status rc = ensure_views(ctx, 1);
  if (rc != GT_OK) {
    cudaFree(buf);
    return rc;
  }
  do {
    cudaError_t ce = cudaMemcpyAsync(d_pix, pixels, (size_t)n_pix * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(ctx->d_ctr, 0, sizeof(DevCounters), ctx->stream);
    if (ce != cudaSuccess) {
      rc = fail(ctx, GT_ERR_CUDA, cudaGetErrorString(ce));
      break;
    }
    Err e = launch_trace_hits(v, ctx->d_views, d_pix, n_pix, (uint32_t)me, d_pidx, d_t, d_alpha, d_count, d_rounds,
                              out_rgba ? d_rgba : nullptr, ctx->d_ctr, ctx->faces, ctx->stream, &ctx->launches);
    if (e.code != GT_OK) {
      rc = fail(ctx, e);
      break;
    }
    ce = cudaMemcpyAsync(out_count, d_count, (size_t)n_pix * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(out_rounds, d_rounds, (size_t)n_pix * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (ce == cudaSuccess && out_rgba)
      ce = cudaMemcpyAsync(out_rgba, d_rgba, (size_t)n_pix * 16, cudaMemcpyDeviceToHost, ctx->stream);
    if (ce == cudaSuccess && max_entries > 0) {
      // copy row by row: device rows have `me` entries, host rows `max_entries`
      ce = cudaMemcpyAsync(out_pidx, d_pidx, (size_t)n_pix * me * 4, cudaMemcpyDeviceToHost, ctx->stream);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(out_t, d_t, (size_t)n_pix * me * 4, cudaMemcpyDeviceToHost, ctx->stream);
      if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(out_alpha, d_alpha, (size_t)n_pix * me * 4, cudaMemcpyDeviceToHost, ctx->stream);
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(ctx->h_ctr, ctx->d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, ctx->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
    if (ce != cudaSuccess) {
      rc = fail(ctx, GT_ERR_CUDA, cudaGetErrorString(ce));
      break;
    }
    rc = status_to_error(ctx, ctx->h_ctr->status);
  } while (0);
  cudaFree(buf);
  return rc;
}

// ============================================================== batches
extern "C" gt_status gt_render_batch(gt_context* ctx, const gt_batch_item* items, uint32_t count, uint32_t flags,
                                     gt_render_stats* stats) {
  if (!ctx) return fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (count == 0) return GT_OK;
  if (!items) return fail(ctx, GT_ERR_INVALID_ARG, "items is NULL");
  if ((flags & GT_FLAG_ASYNC) && !(flags & GT_FLAG_OUTPUT_DEVICE))
    return fail(ctx, GT_ERR_INVALID_ARG, "GT_FLAG_ASYNC needs device output buffers");
  const bool aa = (flags & GT_FLAG_ANTIALIAS) != 0;
  if (aa && (flags & GT_FLAG_CHECKPOINT))
    return fail(ctx, GT_ERR_INVALID_ARG, "GT_FLAG_ANTIALIAS renders are not checkpointed");
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  size_t staging = 0;
  uint64_t slots_all = 0;
  uint32_t kmax = 8, total_tiles = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const gt_batch_item& it = items[i];
    if (!it.scene || it.scene->ctx != ctx) return fail(ctx, GT_ERR_INVALID_ARG, "batch item scene invalid");
    gt_status st = check_uniforms(ctx, &it.u);
    if (st != GT_OK) return st;
    if (!it.out_rgba || it.w == 0 || it.h == 0 || (uint64_t)it.w * it.h > (1ull << 31))
      return fail(ctx, GT_ERR_INVALID_ARG, "batch item image invalid");
    slots_all += view_slots(it.w, it.h);
    if (slots_all > kMaxSlots) return fail(ctx, GT_ERR_INVALID_ARG, "batch larger than 2^31 work slots");
    if ((flags & GT_FLAG_OUTPUT_DEVICE) && ((uintptr_t)it.out_rgba % 16) != 0)
      return fail(ctx, GT_ERR_INVALID_ARG, "device out_rgba must be 16-byte aligned");
    staging += (size_t)it.w * it.h;
    kmax = std::max(kmax, kmax_for(it.u.k));
  }
  gt_status st = ensure_views(ctx, count);
  if (st != GT_OK) return st;
  if (!(flags & GT_FLAG_OUTPUT_DEVICE)) {
    st = ensure_staging(ctx, staging * sizeof(float4));
    if (st != GT_OK) return st;
  }
  if (flags & GT_FLAG_CHECKPOINT) {
    if (flags & GT_FLAG_ASYNC) return fail(ctx, GT_ERR_INVALID_ARG, "a checkpointing render is synchronous");
    std::vector<const gt_scene*> sc(count);
    std::vector<gt_uniforms> us(count);
    std::vector<uint32_t> ws(count), hs(count);
    std::vector<float4*> os(count);
    size_t o = 0;
    for (uint32_t i = 0; i < count; ++i) {
      if (items[i].u.debug_mode != 0) return fail(ctx, GT_ERR_INVALID_ARG, "checkpointing needs debug_mode 0");
      sc[i] = items[i].scene;
      us[i] = items[i].u;
      ws[i] = items[i].w;
      hs[i] = items[i].h;
      os[i] = (flags & GT_FLAG_OUTPUT_DEVICE) ? reinterpret_cast<float4*>(items[i].out_rgba) : ctx->staging + o;
      o += (size_t)items[i].w * items[i].h;
    }
    st = api_forward_ckpt(ctx, sc.data(), us.data(), ws.data(), hs.data(), os.data(), count, 0, 0, 0, stats);
    if (st != GT_OK) return st;
    if (!(flags & GT_FLAG_OUTPUT_DEVICE))
      for (uint32_t i = 0; i < count; ++i)
        API_CUDA(ctx, cudaMemcpyAsync(items[i].out_rgba, os[i], (size_t)ws[i] * hs[i] * sizeof(float4),
                                      cudaMemcpyDeviceToHost, ctx->stream));
    API_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GT_OK;
  }
  // Views of one scene run back to back (stable order by scene): its nodes
  // and records then stay in L2 from one view to the next.  Each view keeps
  // its own output, so the order does not show in the results.
  std::vector<uint32_t> order(count);
  for (uint32_t i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return items[a].scene < items[b].scene; });
  std::vector<size_t> offs(count);
  size_t all_pixels = 0;
  for (uint32_t i = 0; i < count; ++i) {
    offs[i] = all_pixels;
    all_pixels += (size_t)items[i].w * items[i].h;
  }
  // before a graph is looked up: growing the handoff buffer drops the graphs
  Handoff hand;
  st = ensure_handoff(ctx, all_pixels, &hand);
  if (st != GT_OK) return st;
  for (uint32_t q = 0; q < count; ++q) {
    const uint32_t i = order[q];
    const gt_batch_item& it = items[i];
    float4* out = (flags & GT_FLAG_OUTPUT_DEVICE) ? reinterpret_cast<float4*>(it.out_rgba) : ctx->staging + offs[i];
    ctx->h_views[q] = make_view(it.scene, it.u, it.w, it.h, out, total_tiles);
    ctx->h_views[q].u.aa = aa ? 1u : 0u;
    total_tiles += ctx->h_views[q].n_tiles;
    if (aa && it.u.accumulated_frames != 0 && !(flags & GT_FLAG_OUTPUT_DEVICE))
      API_CUDA(ctx, cudaMemcpyAsync(out, it.out_rgba, (size_t)it.w * it.h * sizeof(float4), cudaMemcpyHostToDevice,
                                    ctx->stream));
  }
  st = assign_colours(ctx, ctx->h_views, count);
  if (st != GT_OK) return st;
  bool colours = false;  // (the graph holds the colour kernel or not)
  for (uint32_t q = 0; q < count; ++q) colours = colours || ctx->h_views[q].rgb != nullptr;
  API_CUDA(ctx, cudaEventRecord(ctx->call0, ctx->stream));
  uint64_t slot = ring_slot(ctx);
  API_CUDA(ctx, cudaEventRecord(ctx->ring[2 * slot], ctx->stream));
  // One graph per batch shape: colour tables, counter reset, the trace kernels.  A
  // shape tuned for batches of this shape (gt_autotune_batch) comes first.
  auto bt = ctx->batch_tune.find(std::make_tuple(count, total_tiles, kmax));
  LaunchShape shape = bt != ctx->batch_tune.end() ? shape_of(bt->second)
                                                  : shape_for(ctx, items[0].scene, items[0].w, items[0].h, items[0].u.k);
  // the view table is rebuilt on every call: it takes the shape's k-buffer
  // size and leaf batch here, and the graph's kernel matches its slot count
  const bool packet = packet_launch(ctx->h_views, count, total_tiles, ctx->num_sms, shape, false);
  apply_shape(ctx->h_views, count, shape);
  uint32_t kb_max = 1, pkb_max = 1;
  bool any_debug = false;  // the graph's kernel is the debug-mode instantiation
  for (uint32_t q = 0; q < count; ++q) {
    kb_max = std::max(kb_max, ctx->h_views[q].kbuf);
    pkb_max = std::max(pkb_max, ctx->h_views[q].pkbuf);
    any_debug = any_debug || ctx->h_views[q].u.debug != 0;
  }
  // the kernels of the graph: warp-per-ray slots per lane, and with tile
  // packets their heap size and handoff
  auto key = std::make_tuple(count, total_tiles,
                             kmax | (any_debug ? 0x10000u : 0u) | (packet ? 0x20000u : 0u) | (colours ? 0x40000u : 0u),
                             shape.blocks_per_sm,
                             ((kb_max + 31u) / 32u) | (packet ? (pkb_max << 8) | (shape.handoff_after << 16) : 0u));
  auto it = ctx->graphs.find(key);
  if (it == ctx->graphs.end()) {
    GraphEntry g;
    cudaStream_t cs = ctx->stream;
    API_CUDA(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(ctx->d_ctr, 0, sizeof(DevCounters), cs);
    // launch_trace re-uploads the view table; inside the graph it copies from
    // the pinned staging table, which is refreshed before every replay.
    Err e = launch_trace(ctx->h_views, count, total_tiles, ctx->d_ctr, ctx->faces, shape, ctx->num_sms, cs,
                         &ctx->launches, ctx->d_views, nullptr, &hand);
    cudaError_t ce = cudaStreamEndCapture(cs, &g.graph);
    if (e.code != GT_OK) return fail(ctx, e);
    if (ce != cudaSuccess) return fail(ctx, GT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    API_CUDA(ctx, cudaGraphInstantiate(&g.exec, g.graph, 0));
    it = ctx->graphs.emplace(key, g).first;
  }
  API_CUDA(ctx, cudaGraphLaunch(it->second.exec, ctx->stream));
  ++ctx->launches;
  API_CUDA(ctx, cudaEventRecord(ctx->ring[2 * slot + 1], ctx->stream));
  if (!(flags & GT_FLAG_OUTPUT_DEVICE)) {
    size_t o2 = 0;
    for (uint32_t i = 0; i < count; ++i) {
      size_t px = (size_t)items[i].w * items[i].h;
      API_CUDA(ctx, cudaMemcpyAsync(items[i].out_rgba, ctx->staging + o2, px * sizeof(float4), cudaMemcpyDeviceToHost,
                                    ctx->stream));
      o2 += px;
    }
  }
  if (flags & GT_FLAG_ASYNC) return GT_OK;
  return finish_call(ctx, stats, slot);
}

// ======================================================== loop limits
extern "C" gt_status gt_set_limits(gt_context* ctx, uint32_t max_steps, uint32_t stack_entries,
                                   uint32_t max_rounds) {
  if (!ctx) return fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (stack_entries > (uint32_t)kWarpStack)
    return fail(ctx, GT_ERR_INVALID_ARG, "stack_entries must be at most 256");
  if (max_rounds > kMaxRounds) return fail(ctx, GT_ERR_INVALID_ARG, "max_rounds must be at most 2^22");
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  API_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->faces.lim_steps = max_steps ? max_steps : 0xFFFFFFFFu;
  ctx->faces.lim_stack = stack_entries ? stack_entries : (uint32_t)kWarpStack;
  ctx->faces.lim_rounds = max_rounds ? max_rounds : kMaxRounds;
  drop_graphs(ctx);  // captured launches hold the table by value
  return GT_OK;
}

// =============================================================== tuning
extern "C" gt_status gt_autotune(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u, uint32_t w,
                                 uint32_t h, gt_tune_result* result) {
  if (!ctx) return fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (!scene || scene->ctx != ctx) return fail(ctx, GT_ERR_INVALID_ARG, "scene is NULL or from another context");
  gt_status st = check_uniforms(ctx, u);
  if (st != GT_OK) return st;
  if (w == 0 || h == 0 || (uint64_t)w * h > (1ull << 31) || view_slots(w, h) > kMaxSlots)
    return fail(ctx, GT_ERR_INVALID_ARG, "bad image size");
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  size_t bytes = (size_t)w * h * sizeof(float4);
  st = ensure_staging(ctx, bytes);
  if (st != GT_OK) return st;
  st = ensure_views(ctx, 1);
  if (st != GT_OK) return st;
  ViewDev v = make_view(scene, *u, w, h, ctx->staging, 0);
  st = assign_colours(ctx, &v, 1);  // as gt_render renders it
  if (st != GT_OK) return st;
  Handoff hand;
  st = ensure_handoff(ctx, (uint64_t)w * h, &hand);
  if (st != GT_OK) return st;
  // fastest of `reps` launches of one shape
  auto time_shape = [&](const LaunchShape& sh, int reps, float* out_ms) -> gt_status {
    float ms_min = 1e30f;
    for (int rep = 0; rep < reps; ++rep) {
      API_CUDA(ctx, cudaMemsetAsync(ctx->d_ctr, 0, sizeof(DevCounters), ctx->stream));
      API_CUDA(ctx, cudaEventRecord(ctx->int0, ctx->stream));
      Err e = launch_trace(&v, 1, v.n_tiles, ctx->d_ctr, ctx->faces, sh, ctx->num_sms, ctx->stream, &ctx->launches,
                           ctx->d_views, nullptr, &hand);
      if (e.code != GT_OK) return fail(ctx, e);
      API_CUDA(ctx, cudaEventRecord(ctx->int1, ctx->stream));
      API_CUDA(ctx, cudaEventSynchronize(ctx->int1));
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, ctx->int0, ctx->int1);
      ms_min = std::min(ms_min, ms);
    }
    *out_ms = ms_min;
    return GT_OK;
  };
  const uint32_t k = u->k;
  LaunchShape best_sh;
  float best = 1e30f, def = 0.0f;
  st = time_shape(LaunchShape(), 3, &def);
  if (st != GT_OK) return st;
  // 1. tile packets: k-buffer entries per ray, then the hand-off point of
  // the fastest
  const uint32_t pkbufs[] = {k, 24u, 32u, 48u, 64u};
  for (int i = 0; i < 5; ++i) {
    const uint32_t kb = pkbufs[i];
    if (kb < k || (i > 0 && kb == k)) continue;  // below k, or already timed as k
    LaunchShape sh;
    sh.packet = 1;
    sh.packet_kbuf = std::min(kMaxPacketKbuf, kb);
    float ms = 0.0f;
    st = time_shape(sh, 3, &ms);
    if (st != GT_OK) return st;
    if (ms < best) {
      best = ms;
      best_sh = sh;
    }
  }
  if (best_sh.packet == 1) {
    const LaunchShape kb_sh = best_sh;
    // (64: only once every tile of the launch is taken)
    for (uint32_t ha : {2u, 4u, 6u, 8u, 64u}) {
      LaunchShape sh = kb_sh;
      sh.handoff_after = ha;
      float ms = 0.0f;
      st = time_shape(sh, 3, &ms);
      if (st != GT_OK) return st;
      if (ms < best) {
        best = ms;
        best_sh = sh;
      }
    }
  }
  // 2. a warp per ray: resident blocks per SM, then k-buffer size and leaf batch
  LaunchShape warp_sh;
  warp_sh.packet = 0;
  float warp_best = 1e30f;
  const uint32_t cands[] = {1, 2, 3, 4, 6, 8, 12, 16};
  for (uint32_t b : cands) {
    LaunchShape sh = warp_sh;
    sh.blocks_per_sm = b;
    float ms = 0.0f;
    st = time_shape(sh, 3, &ms);
    if (st != GT_OK) return st;
    if (ms < warp_best) {
      warp_best = ms;
      warp_sh = sh;
    }
  }
  const uint32_t kbufs[] = {k, 32u, 64u, 96u, 128u};
  const uint32_t batches[] = {8u, 16u, 24u, 32u};
  const LaunchShape occ_sh = warp_sh;
  for (uint32_t kb : kbufs) {
    for (uint32_t lb : batches) {
      LaunchShape sh = occ_sh;
      sh.kbuf = std::min(kMaxKbuf, kb);
      sh.leaf_batch = lb;
      if (sh.kbuf == occ_sh.kbuf && sh.leaf_batch == occ_sh.leaf_batch) continue;
      float ms = 0.0f;
      st = time_shape(sh, 2, &ms);
      if (st != GT_OK) return st;
      if (ms < warp_best) {
        warp_best = ms;
        warp_sh = sh;
      }
    }
  }
  if (warp_best < best) {
    best = warp_best;
    best_sh = warp_sh;
  }
  gt_tune_result r;
  memset(&r, 0, sizeof r);
  r.block_threads = best_sh.packet ? 32u : 128u;
  r.blocks_per_sm = best_sh.blocks_per_sm;
  r.tile_w = 8;
  r.tile_h = 4;
  r.best_ms = best;
  r.default_ms = def;
  r.kbuf = std::max(best_sh.packet ? best_sh.packet_kbuf : best_sh.kbuf, k);
  r.leaf_batch = best_sh.leaf_batch;
  r.handoff_after = best_sh.handoff_after;
  ctx->tune[tune_key(scene, w, h, k)] = r;
  if (result) *result = r;
  return GT_OK;
}

extern "C" gt_status gt_autotune_batch(gt_context* ctx, const gt_batch_item* items, uint32_t count,
                                       gt_tune_result* result) {
  if (!ctx) return fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (count == 0 || !items) return fail(ctx, GT_ERR_INVALID_ARG, "empty batch");
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  uint64_t slots_all = 0, pixels = 0;
  uint32_t kmax = 8, kmin = 32;
  for (uint32_t i = 0; i < count; ++i) {
    const gt_batch_item& it = items[i];
    if (!it.scene || it.scene->ctx != ctx) return fail(ctx, GT_ERR_INVALID_ARG, "batch item scene invalid");
    gt_status st = check_uniforms(ctx, &it.u);
    if (st != GT_OK) return st;
    if (it.w == 0 || it.h == 0 || (uint64_t)it.w * it.h > (1ull << 31))
      return fail(ctx, GT_ERR_INVALID_ARG, "batch item image invalid");
    slots_all += view_slots(it.w, it.h);
    if (slots_all > kMaxSlots) return fail(ctx, GT_ERR_INVALID_ARG, "batch larger than 2^31 work slots");
    pixels += (uint64_t)it.w * it.h;
    kmax = std::max(kmax, kmax_for(it.u.k));
    kmin = std::min(kmin, std::max(1u, it.u.k));
  }
  gt_status st = ensure_views(ctx, count);
  if (st != GT_OK) return st;
  st = ensure_staging(ctx, pixels * sizeof(float4));
  if (st != GT_OK) return st;
  Handoff hand;
  st = ensure_handoff(ctx, pixels, &hand);
  if (st != GT_OK) return st;
  // the view table as gt_render_batch builds it (views of one scene back to
  // back), images into the scratch buffer
  std::vector<uint32_t> order(count);
  for (uint32_t i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return items[a].scene < items[b].scene; });
  uint32_t total_tiles = 0;
  size_t off = 0;
  for (uint32_t q = 0; q < count; ++q) {
    const gt_batch_item& it = items[order[q]];
    ctx->h_views[q] = make_view(it.scene, it.u, it.w, it.h, ctx->staging + off, total_tiles);
    total_tiles += ctx->h_views[q].n_tiles;
    off += (size_t)it.w * it.h;
  }
  st = assign_colours(ctx, ctx->h_views, count);  // as gt_render_batch renders it
  if (st != GT_OK) return st;
  auto time_shape = [&](const LaunchShape& sh, int reps, float* out_ms) -> gt_status {
    float ms_min = 1e30f;
    for (int rep = 0; rep < reps; ++rep) {
      API_CUDA(ctx, cudaMemsetAsync(ctx->d_ctr, 0, sizeof(DevCounters), ctx->stream));
      API_CUDA(ctx, cudaEventRecord(ctx->int0, ctx->stream));
      Err e = launch_trace(ctx->h_views, count, total_tiles, ctx->d_ctr, ctx->faces, sh, ctx->num_sms, ctx->stream,
                           &ctx->launches, ctx->d_views, nullptr, &hand);
      if (e.code != GT_OK) return fail(ctx, e);
      API_CUDA(ctx, cudaEventRecord(ctx->int1, ctx->stream));
      API_CUDA(ctx, cudaEventSynchronize(ctx->int1));
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, ctx->int0, ctx->int1);
      ms_min = std::min(ms_min, ms);
    }
    *out_ms = ms_min;
    return GT_OK;
  };
  // the shape gt_render_batch takes without a batch result
  const LaunchShape def_sh = shape_for(ctx, items[0].scene, items[0].w, items[0].h, items[0].u.k);
  float def = 0.0f;
  st = time_shape(def_sh, 2, &def);  // (the first launches also warm the caches)
  if (st != GT_OK) return st;
  st = time_shape(def_sh, 2, &def);
  if (st != GT_OK) return st;
  LaunchShape best_sh = def_sh;
  float best = def;
  const uint32_t pkbufs[] = {kmin, 24u, 32u, 48u, 64u};
  const uint32_t hands[] = {2u, 3u, 4u, 6u};
  for (int i = 0; i < 5; ++i) {
    if (pkbufs[i] < kmin || (i > 0 && pkbufs[i] == kmin)) continue;
    for (uint32_t ha : hands) {
      LaunchShape sh;
      sh.packet = 1;
      sh.packet_kbuf = std::min(kMaxPacketKbuf, pkbufs[i]);
      sh.handoff_after = ha;
      float ms = 0.0f;
      st = time_shape(sh, 2, &ms);
      if (st != GT_OK) return st;
      if (ms < best) {
        best = ms;
        best_sh = sh;
      }
    }
  }
  for (uint32_t b : {4u, 8u}) {
    LaunchShape sh;
    sh.packet = 0;
    sh.blocks_per_sm = b;
    float ms = 0.0f;
    st = time_shape(sh, 2, &ms);
    if (st != GT_OK) return st;
    if (ms < best) {
      best = ms;
      best_sh = sh;
    }
  }
  gt_tune_result r;
  memset(&r, 0, sizeof r);
  const bool pk = packet_launch(ctx->h_views, count, total_tiles, ctx->num_sms, best_sh, false);
  r.block_threads = pk ? 32u : 128u;
  r.blocks_per_sm = best_sh.blocks_per_sm;
  r.tile_w = 8;
  r.tile_h = 4;
  r.best_ms = best;
  r.default_ms = def;
  r.kbuf = pk ? best_sh.packet_kbuf : best_sh.kbuf;
  r.leaf_batch = best_sh.leaf_batch;
  r.handoff_after = best_sh.handoff_after;
  ctx->batch_tune[std::make_tuple(count, total_tiles, kmax)] = r;
  if (result) *result = r;
  return GT_OK;
}

extern "C" gt_status gt_set_tune(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u, uint32_t w,
                                 uint32_t h, const gt_tune_result* shape) {
  if (!ctx) return fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (!scene || scene->ctx != ctx) return fail(ctx, GT_ERR_INVALID_ARG, "scene is NULL or from another context");
  gt_status st = check_uniforms(ctx, u);
  if (st != GT_OK) return st;
  if (!shape) return fail(ctx, GT_ERR_INVALID_ARG, "shape is NULL");
  if ((shape->block_threads != 32 && shape->block_threads != 128) || shape->tile_w != 8 || shape->tile_h != 4)
    return fail(ctx, GT_ERR_INVALID_ARG, "block_threads must be 32 or 128 and the tile 8 x 4");
  if (shape->blocks_per_sm < 1 || shape->blocks_per_sm > 32 || shape->kbuf < 1 || shape->kbuf > kMaxKbuf ||
      shape->leaf_batch < 1 || shape->leaf_batch > 32)
    return fail(ctx, GT_ERR_INVALID_ARG, "blocks_per_sm and leaf_batch must lie in 1..32, kbuf in 1..128");
  if (shape->handoff_after > 64) return fail(ctx, GT_ERR_INVALID_ARG, "handoff_after must be at most 64");
  gt_tune_result r = *shape;
  ctx->tune[tune_key(scene, w, h, u->k)] = r;
  return GT_OK;
}

extern "C" gt_status gt_autotune_reset(gt_context* ctx) {
  if (!ctx) return GT_ERR_INVALID_ARG;
  ctx->tune.clear();
  ctx->batch_tune.clear();
  return GT_OK;
}

// ======================================================= device helpers
extern "C" gt_status gt_device_alloc(gt_context* ctx, uint64_t bytes, void** out) {
  if (!ctx || !out) return fail(ctx, GT_ERR_INVALID_ARG, "NULL argument");
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  API_CUDA(ctx, cudaMalloc(out, bytes ? bytes : 1));
  return GT_OK;
}
extern "C" gt_status gt_device_free(gt_context* ctx, void* ptr) {
  if (!ctx) return GT_ERR_INVALID_ARG;
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  API_CUDA(ctx, cudaFree(ptr));
  return GT_OK;
}
extern "C" gt_status gt_host_alloc(gt_context* ctx, uint64_t bytes, void** out) {
  if (!ctx || !out) return fail(ctx, GT_ERR_INVALID_ARG, "NULL argument");
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  API_CUDA(ctx, cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault));
  return GT_OK;
}
extern "C" gt_status gt_host_free(gt_context* ctx, void* ptr) {
  if (!ctx) return GT_ERR_INVALID_ARG;
  API_CUDA(ctx, cudaFreeHost(ptr));
  return GT_OK;
}
extern "C" gt_status gt_memcpy(gt_context* ctx, void* dst, const void* src, uint64_t bytes, int kind) {
  if (!ctx || (!dst && bytes) || (!src && bytes) || kind < 0 || kind > 2)
    return fail(ctx, GT_ERR_INVALID_ARG, "bad gt_memcpy argument");
  cudaMemcpyKind k = kind == 0 ? cudaMemcpyHostToDevice : (kind == 1 ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice);
  API_CUDA(ctx, cudaSetDevice(ctx->device));
  API_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, k, ctx->stream));
  API_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GT_OK;
}
extern "C" gt_status gt_synchronize(gt_context* ctx) {
  if (!ctx) return GT_ERR_INVALID_ARG;
  API_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return GT_OK;
}
extern "C" gt_status gt_timer_start(gt_context* ctx) {
  if (!ctx) return GT_ERR_INVALID_ARG;
  API_CUDA(ctx, cudaEventRecord(ctx->timer0, ctx->stream));
  return GT_OK;
}
extern "C" gt_status gt_timer_stop(gt_context* ctx, float* ms) {
  if (!ctx || !ms) return GT_ERR_INVALID_ARG;
  API_CUDA(ctx, cudaEventRecord(ctx->timer1, ctx->stream));
  API_CUDA(ctx, cudaEventSynchronize(ctx->timer1));
  API_CUDA(ctx, cudaEventElapsedTime(ms, ctx->timer0, ctx->timer1));
  return GT_OK;
}
extern "C" gt_status gt_kernel_times(gt_context* ctx, float* out_ms, uint32_t max, uint32_t* n) {
  if (!ctx || !n || (max && !out_ms)) return GT_ERR_INVALID_ARG;
  API_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  uint64_t avail = ctx->ring_head - ctx->ring_tail;
  if (avail > kEventRing) {
    ctx->ring_tail = ctx->ring_head - kEventRing;
    avail = kEventRing;
  }
  uint32_t m = 0;
  while (ctx->ring_tail < ctx->ring_head && m < max) {
    uint64_t s = ctx->ring_tail % kEventRing;
    float ms = 0.0f;
    API_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ring[2 * s], ctx->ring[2 * s + 1]));
    out_ms[m++] = ms;
    ++ctx->ring_tail;
  }
  ctx->ring_tail = ctx->ring_head;
  *n = m;
  return GT_OK;
}
extern "C" gt_status gt_launch_count(const gt_context* ctx, uint64_t* n) {
  if (!ctx || !n) return GT_ERR_INVALID_ARG;
  *n = ctx->launches;
  return GT_OK;
}

extern "C" gt_status gt_device_attributes(const gt_context* ctx, uint32_t* sm_count, uint32_t* max_sm_khz) {
  if (!ctx) return GT_ERR_INVALID_ARG;
  if (sm_count) *sm_count = (uint32_t)ctx->num_sms;
  if (max_sm_khz) {
    int khz = 0;
    if (cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, ctx->device) != cudaSuccess) {
      (void)cudaGetLastError();
      return GT_ERR_CUDA;
    }
    *max_sm_khz = (uint32_t)khz;
  }
  return GT_OK;
}
