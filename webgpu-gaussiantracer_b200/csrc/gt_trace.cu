// gt_trace.cu — forward tracer, one warp per ray, over the 8-wide BVH.
//
// Replaces the reference's per-pixel mega compute shader (raygen + tracePath
// rounds, src/GS_shader.ts:192-309; traversal, webrtx/src/glsl/trace.glsl:42-245;
// any-hit k-buffer, src/GS_shader.ts:323-367).
//
// Why a warp per ray: rays of a Gaussian scene differ wildly in the number of
// rounds, nodes and proxies they touch, so one ray per lane leaves most lanes
// idle (2.6 of 32 active in the thread-per-ray version).  Here the 32 lanes
// of a warp cooperate on one ray and every control decision is warp-uniform:
//   * traversal: up to 4 nodes are popped at once and their 32 children are
//     box-tested by the 32 lanes; hit inner children are sorted by entry
//     distance (warp bitonic sort) and pushed far-to-near onto a per-warp
//     stack in shared memory; hit leaves go to a per-warp leaf queue;
//   * leaves: queued proxies go through the bounding-sphere filter 32 at a
//     time, and those that pass through the exact object-space face tests of
//     the reference (gt_trace_common.cuh) 24 at a time, one per lane;
//   * k-buffer: entry 32 j + i (j < NB slots) lives in lane i; a hit is
//     inserted with one ballot and shuffles.  A traversal keeps the kbuf
//     (64 by default, up to 128) closest hits beyond t_curr and feeds several
//     rounds: a round's set (the k smallest hits with t > t_curr) is certain
//     whenever it lies inside the first kbuf entries or the buffer is not full;
//   * compositing: lanes evaluate the response and SH colour of one entry
//     each; the front-to-back accumulation then runs in entry order on
//     broadcast values, so the float operations are those of the reference
//     loop (src/GS_shader.ts:250-269), in the same order.
#include <math_constants.h>

#include "gt_device.cuh"
#include "gt_internal.cuh"
#include "gt_trace_common.cuh"
#include "gt_warp.cuh"

namespace gt {

// Per-ray state (identical in all lanes).
struct WRay {
  V3 o, d;
  BoxRay br;
  float L0, L1, L2, T, t_curr;
  uint32_t step, n_entries;
};

__device__ __forceinline__ bool wray_more(const ViewDev& V, const WRay& R) {
  return V.u.T_min < R.T && R.t_curr < V.u.t_max && V.u.early_stop != R.step;
}

// tracePath (src/GS_shader.ts:192-273) for one pixel, by one warp.
// RECORD: write the composited hit sequence (gt_render_hits).
// CKPT: write the round checkpoint the adjoint replays (gt_backward).
// DEBUG: also handle debugMode 1 and 2.  Launches whose views all render
// (debugMode 0) use the instantiation without them: their extra traversal
// copies cost the render loop registers and spills (4.7 % of its time).
// init: the state of a ray handed over by a tile packet (nullptr: a new ray).
template <bool RECORD, bool CKPT, int NB, bool DEBUG>
__device__ __forceinline__ float4 trace_ray_warp(const ViewDev& V, const FaceTable& F, WarpScratch& W, uint32_t px,
                                                 uint32_t py, RayStats& st, uint32_t& status, uint32_t lane,
                                                 const HitOut& ho, uint32_t slot, const Ckpt& ck,
                                                 const HandoffRay* init) {
  WRay R;
  ray_gen(V.u, V.w, V.h, px, py, R.o, R.d);
  R.br = make_boxray(R.o, R.d, V.s.scene_mag);
  const float t_max = V.u.t_max;
  if (DEBUG && V.u.debug != 0) {
    KBuf<1> kb;
    kbuf_init(kb, t_max);
    uint32_t cnt = 0;
    if (V.u.debug == 1) {
      traverse8<kClosestAny>(V.s, F, W, R.o, R.d, R.br, V.u.t_min, t_max, kb, st, status, lane);
      float4 out = make_float4(0.f, 0.f, 0.f, 1.f);
      uint32_t p0 = __shfl_sync(kFull, kb.p[0], 0);
      if (p0 != kInvalid) {
        float c[3];
        sh_radiance(V.s.sh, p0, R.d, V.u.deg, c);
        out = make_float4(c[0] > 0.f ? c[0] : 0.f, c[1] > 0.f ? c[1] : 0.f, c[2] > 0.f ? c[2] : 0.f, 1.f);
        cnt = 1;
      }
      if (RECORD && lane == 0) {
        ho.count[slot] = cnt;
        ho.rounds[slot] = 0;
      }
      return out;
    }
    // kCountFront: the warp's anyhit counter before and after
    __syncwarp();
    const unsigned long long before = st.anyhits;
    traverse8<kCountFront>(V.s, F, W, R.o, R.d, R.br, V.u.t_min, t_max, kb, st, status, lane);
    __syncwarp();
    cnt = (uint32_t)(st.anyhits - before);
    __syncwarp();
    float r = 0.f, g = 0.f, b = 0.f;
    if (cnt == 0) {
    } else if (cnt < 20) { r = 0.5f; g = 0.5f; }
    else if (cnt < 40) { r = 0.5f; b = 0.5f; }
    else if (cnt < 60) { g = 0.5f; b = 0.5f; }
    else if (cnt < 80) { r = 0.5f; }
    else if (cnt < 100) { g = 0.5f; }
    else if (cnt < 150) { b = 0.5f; }
    else { r = 0.5f; g = 0.5f; b = 0.5f; }
    if (RECORD && lane == 0) {
      ho.count[slot] = cnt;
      ho.rounds[slot] = 0;
    }
    return make_float4(r, g, b, 1.f);
  }
  R.L0 = R.L1 = R.L2 = 0.f;
  R.T = 1.f;
  R.t_curr = V.u.t_min;
  R.step = 0;
  R.n_entries = 0;
  uint32_t ck_head = kInvalid;
  uint32_t ck_fill = ck.kc;  // entries in the open record (checkpoint mode; kc: none open)
  if (!RECORD && init) {
    R.L0 = init->L0;
    R.L1 = init->L1;
    R.L2 = init->L2;
    R.T = init->T;
    R.t_curr = init->t_curr;
    R.step = init->step;
    ck_head = init->ck_head;
    ck_fill = init->ck_fill;
  }
  const uint32_t k = V.u.k;
  while (wray_more(V, R)) {
    // one traversal: the kbuf closest front-face hits with t > t_curr
    KBuf<NB> kb;
    kbuf_init(kb, t_max);
    const int kbuf = (int)V.kbuf;
    // The ray's accumulators are warp-uniform: they wait out the traversal in
    // shared memory (volatile, so the compiler does not keep register copies),
    // which leaves the traversal and the proxy test more registers and cut
    // spilling (5% faster on the 1M-Gaussian 1080p view).
    if (lane == 0) {
      volatile float* vs = W.rs;
      volatile uint32_t* vu = W.ru;
      vs[0] = R.L0;
      vs[1] = R.L1;
      vs[2] = R.L2;
      vs[3] = R.T;
      vu[0] = R.step;
      vu[1] = R.n_entries;
      vu[2] = ck_head;
      if (CKPT) vu[3] = ck_fill;
    }
    traverse8<kCollect>(V.s, F, W, R.o, R.d, R.br, R.t_curr, t_max, kb, st, status, lane, kbuf, V.leaf_batch);
    {
      __syncwarp();
      volatile float* vs = W.rs;
      volatile uint32_t* vu = W.ru;
      R.L0 = vs[0];
      R.L1 = vs[1];
      R.L2 = vs[2];
      R.T = vs[3];
      R.step = vu[0];
      R.n_entries = vu[1];
      ck_head = vu[2];
      if (CKPT) ck_fill = vu[3];
    }
    // status bits may be set in single lanes: reduce before branching on them
    if (__reduce_or_sync(kFull, status) & (kStatusStackOverflow | kStatusVisitCap | kStatusHitOverflow)) break;
    // only entries below kbuf are certain: the far bound was entry kbuf-1
    uint32_t cnt = 0;
#pragma unroll
    for (int j = 0; j < NB; ++j) cnt += __popc(__ballot_sync(kFull, kb.p[j] != kInvalid && 32 * j + (int)lane < kbuf));
    const bool complete = cnt < (uint32_t)kbuf;
    // rounds served from this buffer
    while (wray_more(V, R)) {
      // entries past kbuf are not counted: hits just beyond entry kbuf-1 can
      // lie below t_curr
      uint32_t skip = 0;
#pragma unroll
      for (int j = 0; j < NB; ++j)
        skip += __popc(
            __ballot_sync(kFull, kb.p[j] != kInvalid && 32 * j + (int)lane < kbuf && !(kb.t[j] > R.t_curr)));
      const uint32_t avail = cnt - skip;
      if (!complete && avail < k) break;  // the next round reaches past the buffer
      const uint32_t n = avail < k ? avail : k;
      // this round's entries, entry e in lane e
      const int pos = (int)(skip + lane);
      const int src = pos & 31;
      float et = __shfl_sync(kFull, kb.t[0], src);
      uint32_t ep = __shfl_sync(kFull, kb.p[0], src);
#pragma unroll
      for (int j = 1; j < NB; ++j) {
        const float xt = __shfl_sync(kFull, kb.t[j], src);
        const uint32_t xp = __shfl_sync(kFull, kb.p[j], src);
        if ((pos >> 5) == j) {
          et = xt;
          ep = xp;
        }
      }
      if (CKPT && ck.kc == 0) {
        // replay mode: one record a round
        uint32_t rec = 0;
        if (lane == 0) rec = atomicAdd(ck.pool_next, 1u);
        rec = __shfl_sync(kFull, rec, 0);
        if (rec < ck.pool_cap) {  // past the pool the host sizes it up and runs again
          uint32_t* r = ck.pool + (size_t)rec * (kCkptHeader + ck.kc);
          if (lane == 0) {
            r[0] = __float_as_uint(R.t_curr);
            r[1] = __float_as_uint(R.T);
            r[2] = ck_head;
            r[3] = n;
          }
          ck_head = rec;
        }
      }
      ++R.step;
      if (lane == 0) ++st.rounds;
      float new_t = n == k ? kbuf_t_at(kb, (int)(skip + k - 1)) + 1e-4f : t_max;
      const bool mine = lane < n;
      float alpha = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
      bool contrib = false;
      if (mine) {
        Shade sd = load_shade(V.s.shade, ep);
        alpha = response(sd, R.o, R.d) * sd.opacity;
        contrib = V.u.alpha_min < alpha;
        if (contrib) {
          if (V.rgb) {
            const float4 q = __ldg(V.rgb + ep);
            c0 = q.x;
            c1 = q.y;
            c2 = q.z;
          } else {
            entry_colour(V.s.sh, ep, sd.mu, R.o, V.u.deg, c0, c1, c2);
          }
        }
        if (RECORD) {
          uint32_t e = R.n_entries + lane;
          if (e < ho.max_entries) {
            size_t at = (size_t)slot * ho.max_entries + e;
            ho.pidx[at] = ep;
            ho.t[at] = et;
            ho.alpha[at] = alpha;
          }
        }
      }
      const uint32_t cmask = __ballot_sync(kFull, contrib);
      if (lane == 0) {
        st.entries += n;
        st.contributing += (unsigned)__popc(cmask);
      }
      // front-to-back accumulation in entry order
      for (uint32_t e = 0; e < n; ++e) {
        float a = __shfl_sync(kFull, alpha, (int)e);
        float x0 = __shfl_sync(kFull, c0, (int)e);
        float x1 = __shfl_sync(kFull, c1, (int)e);
        float x2 = __shfl_sync(kFull, c2, (int)e);
        if ((cmask >> e) & 1u) {
          if (CKPT && ck.kc) {
            // checkpoint mode: the entry goes to the ray's open record
            const uint32_t pe = __shfl_sync(kFull, ep, (int)e);
            if (ck_fill >= ck.kc) {
              uint32_t rec = 0;
              if (lane == 0) rec = atomicAdd(ck.pool_next, 1u);
              rec = __shfl_sync(kFull, rec, 0);
              if (lane == 0 && rec < ck.pool_cap) {  // past the pool the host sizes it up and runs again
                uint32_t* r = ck.pool + (size_t)rec * (kCkptHeader + ck.kc);
                r[0] = __float_as_uint(R.t_curr);
                r[1] = __float_as_uint(R.T);
                r[2] = ck_head;
              }
              ck_head = rec;
              ck_fill = 0;
            }
            if (lane == 0 && ck_head < ck.pool_cap) {
              uint32_t* r = ck.pool + (size_t)ck_head * (kCkptHeader + ck.kc);
              r[kCkptHeader + ck_fill] = pe;
              r[3] = ck_fill + 1;
            }
            ++ck_fill;
          }
          float ta = R.T * a;
          R.L0 = R.L0 + ta * x0;
          R.L1 = R.L1 + ta * x1;
          R.L2 = R.L2 + ta * x2;
          R.T = R.T * (1.0f - a);
        }
      }
      R.n_entries += n;
      R.t_curr = new_t;
      if (R.step >= F.lim_rounds && wray_more(V, R)) {
        status |= kStatusRoundCap;
        R.t_curr = t_max;
      }
    }
  }
  if (RECORD && lane == 0) {
    ho.count[slot] = R.n_entries;
    ho.rounds[slot] = R.step;
  }
  if (CKPT && lane == 0) ck.head[slot] = ck_head < ck.pool_cap ? ck_head : kInvalid;
  return make_float4(R.L0, R.L1, R.L2, 1.0f);
}

// Persistent kernel: each warp takes one pixel slot at a time from a global
// counter (slot = 32 * tile + position in the 8x4 tile, views back to back),
// so neighbouring pixels run on neighbouring warps at the same time.  With
// `resume`, the slots are instead the rays a tile-packet launch handed over
// (DevCounters::handoff of them, at most resume_cap), continued from their
// state.
// 8 resident blocks (32 warps per SM, 64 registers a thread) beat 4 blocks
// without spills by 12% on the 1M-Gaussian 1080p view: the kernel is bound by
// dependent latencies, and more warps hide them better than the spill loads
// cost (measured 4/5/6/8/10/12/16 blocks: 111/105/104/98/112/121/140 ms).
template <bool RECORD, bool CKPT, int NB, bool DEBUG>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 8) k_trace8(const ViewDev* __restrict__ views, uint32_t n_views,
                                                                  uint32_t total_tiles, DevCounters* ctr,
                                                                  const __grid_constant__ FaceTable F,
                                                                  const uint32_t* pixels, uint32_t n_pix,
                                                                  const HitOut ho, const Ckpt ck,
                                                                  const HandoffRay* resume, uint32_t resume_cap) {
  __shared__ WarpScratch scratch[kWarpsPerBlock];
  const uint32_t lane = threadIdx.x & 31;
  WarpScratch& W = scratch[threadIdx.x >> 5];
  RayStats& st = W.stats;
  if (lane == 0) st = RayStats{0, 0, 0, 0, 0, 0};
  __syncwarp();
  uint32_t status = 0, rays = 0;
  const uint32_t total = RECORD ? n_pix : (resume ? min(ctr->handoff, resume_cap) : total_tiles * 32u);
  while (true) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(resume ? &ctr->work2 : &ctr->work, 1u);
    item = __shfl_sync(kFull, item, 0);
    if (item >= total) break;
    const HandoffRay* init = nullptr;
    if (!RECORD && resume) {
      init = resume + item;
      item = init->item;
    }
    uint32_t vi = 0, px, py;
    if (RECORD) {
      uint32_t pix = pixels[item];
      const ViewDev& V = views[0];
      if (pix >= V.w * V.h) continue;
      px = pix % V.w;
      py = pix / V.w;
    } else {
      uint32_t tile = item >> 5, s = item & 31u;
      vi = n_views == 1 ? 0u : find_view(views, n_views, tile);
      const ViewDev& V = views[vi];
      tile_pixel(V.tiles_x, tile - V.tile_begin, s, px, py);
      if (px >= V.w || py >= V.h) continue;
    }
    // the output position waits in shared memory as well
    if (lane == 0) {
      volatile uint32_t* vu = W.ru;
      vu[4] = vi;
      vu[5] = px;
      vu[6] = py;
      vu[7] = item;
    }
    const float4 r = trace_ray_warp<RECORD, CKPT, NB, DEBUG>(views[vi], F, W, px, py, st, status, lane, ho, item,
                                                            ck, init);
    {
      __syncwarp();
      volatile uint32_t* vu = W.ru;
      vi = vu[4];
      px = vu[5];
      py = vu[6];
      item = vu[7];
    }
    const ViewDev& V = views[vi];
    if (lane == 0) {
      if (RECORD) {
        if (ho.rgba) ho.rgba[item] = r;
      } else {
        float4* dst = V.out + (size_t)py * V.w + px;
        *dst = V.u.aa ? aa_blend(*dst, r, V.u.frames) : r;
      }
      ++rays;
    }
  }
  flush_stats(ctr, st, rays, status);
}

uint32_t kmax_for(uint32_t k) { return k <= 8 ? 8u : (k <= 16 ? 16u : 32u); }

bool packet_launch(const ViewDev* views, uint32_t n_views, uint32_t total_tiles, int num_sms,
                   const LaunchShape& shape, bool ckpt) {
  (void)ckpt;  // the tile packets write the checkpoint as well
  if (!shape.packet) return false;
  for (uint32_t i = 0; i < n_views; ++i)
    if (views[i].u.debug != 0) return false;
  if (shape.packet == 1) return true;
  return (uint64_t)total_tiles >= (uint64_t)kPacketTilesPerSm * (uint64_t)std::max(1, num_sms);
}

void apply_shape(ViewDev* views, uint32_t n_views, const LaunchShape& shape) {
  for (uint32_t i = 0; i < n_views; ++i) {
    views[i].kbuf = std::max(1u, std::min(kMaxKbuf, std::max(shape.kbuf, views[i].u.k)));
    views[i].pkbuf = std::max(1u, std::min(kMaxPacketKbuf, std::max(shape.packet_kbuf, views[i].u.k)));
    views[i].leaf_batch = std::min(32u, std::max(1u, shape.leaf_batch));
  }
}

// The colour table of each view that has one: thread p of row v writes view
// v's colour of particle p (entry_colour, the arithmetic of the trace
// kernels' own evaluation, so the image bits do not depend on the table).
// (A grid-stride loop: a launch captured in a batch graph serves later
// batches of the same shape whose scenes hold more particles.)
__global__ void k_view_colours(const ViewDev* __restrict__ views) {
  const ViewDev& V = views[blockIdx.y];
  if (!V.rgb) return;
  const V3 o = mk(V.u.tw[12], V.u.tw[13], V.u.tw[14]);  // the rays' origin (ray_gen)
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < V.n_particles;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const V3 mu = load_shade(V.s.shade, (uint32_t)p).mu;
    float x0, x1, x2;
    entry_colour(V.s.sh, (uint32_t)p, mu, o, V.u.deg, x0, x1, x2);
    V.rgb[p] = make_float4(x0, x1, x2, 0.0f);
  }
}

Err launch_view_colours(const ViewDev* views, const ViewDev* d_views, uint32_t n_views, int num_sms,
                        cudaStream_t stream, uint64_t* launches) {
  uint64_t colour_rows = 0;
  for (uint32_t i = 0; i < n_views; ++i)
    if (views[i].rgb) colour_rows = std::max<uint64_t>(colour_rows, views[i].n_particles);
  if (colour_rows == 0) return Err{};
  if (n_views > 65535u) return Err{GT_ERR_INVALID_ARG, "colour tables for more than 65535 views"};
  const uint32_t cb = 256;
  const uint64_t blocks = std::min<uint64_t>((colour_rows + cb - 1) / cb, (uint64_t)num_sms * 16u);
  k_view_colours<<<dim3((unsigned)blocks, n_views), cb, 0, stream>>>(d_views);
  ++*launches;
  GT_CUDA_TRY(cudaGetLastError());
  return Err{};
}

Err launch_trace(ViewDev* views, uint32_t n_views, uint32_t total_tiles, DevCounters* counters,
                 const FaceTable& faces, const LaunchShape& shape, int num_sms, cudaStream_t stream,
                 uint64_t* launches, ViewDev* d_views, const Ckpt* ckpt, const Handoff* handoff) {
  const bool packet = packet_launch(views, n_views, total_tiles, num_sms, shape, ckpt != nullptr);
  apply_shape(views, n_views, shape);
  GT_CUDA_TRY(cudaMemcpyAsync(d_views, views, sizeof(ViewDev) * n_views, cudaMemcpyHostToDevice, stream));
  Err ce = launch_view_colours(views, d_views, n_views, num_sms, stream, launches);
  if (ce.code != GT_OK) return ce;
  const bool hand = packet && handoff && handoff->rays && handoff->cap && shape.handoff_after;
  if (packet) {
    Err e = launch_trace_packet(views, d_views, n_views, total_tiles, counters, faces, num_sms, stream, launches,
                                hand ? *handoff : Handoff{}, shape.handoff_after, ckpt);
    if (e.code != GT_OK || !hand) return e;
  }
  uint32_t block = kWarpsPerBlock * 32;
  uint32_t grid = (uint32_t)num_sms * std::max(1u, shape.blocks_per_sm);
  uint64_t warps_needed = (uint64_t)total_tiles * 32u;
  uint64_t max_grid = (warps_needed + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (grid > max_grid) grid = (uint32_t)std::max<uint64_t>(1, max_grid);
  HitOut ho{};
  // buffer slots per lane: enough for the widest k-buffer of the batch
  uint32_t kmax = 1;
  for (uint32_t i = 0; i < n_views; ++i) kmax = std::max(kmax, views[i].kbuf);
  const uint32_t nb = (kmax + 31u) / 32u;
  const Ckpt ck = ckpt ? *ckpt : Ckpt{};
  bool debug = false;
  for (uint32_t i = 0; i < n_views; ++i) debug = debug || views[i].u.debug != 0;
  const void* fn;
  if (ckpt)  // checkpointing renders have debugMode 0
    fn = nb <= 1   ? (const void*)k_trace8<false, true, 1, false>
         : nb == 2 ? (const void*)k_trace8<false, true, 2, false>
         : nb == 3 ? (const void*)k_trace8<false, true, 3, false>
                   : (const void*)k_trace8<false, true, 4, false>;
  else if (debug)
    fn = nb <= 1   ? (const void*)k_trace8<false, false, 1, true>
         : nb == 2 ? (const void*)k_trace8<false, false, 2, true>
         : nb == 3 ? (const void*)k_trace8<false, false, 3, true>
                   : (const void*)k_trace8<false, false, 4, true>;
  else
    fn = nb <= 1   ? (const void*)k_trace8<false, false, 1, false>
         : nb == 2 ? (const void*)k_trace8<false, false, 2, false>
         : nb == 3 ? (const void*)k_trace8<false, false, 3, false>
                   : (const void*)k_trace8<false, false, 4, false>;
  const ViewDev* dv = d_views;
  const uint32_t* no_pix = nullptr;
  uint32_t zero = 0;
  // after a tile-packet launch: the rays it handed over, one warp per ray
  const HandoffRay* resume = hand ? handoff->rays : nullptr;
  const uint32_t resume_cap = hand ? handoff->cap : 0u;
  if (hand) grid = (uint32_t)num_sms * std::max(1u, shape.blocks_per_sm);
  void* args[] = {(void*)&dv, (void*)&n_views, (void*)&total_tiles, (void*)&counters, (void*)&faces,
                  (void*)&no_pix, (void*)&zero, (void*)&ho, (void*)&ck, (void*)&resume, (void*)&resume_cap};
  GT_CUDA_TRY(cudaLaunchKernel(fn, dim3(grid), dim3(block), args, 0, stream));
  ++*launches;
  GT_CUDA_TRY(cudaGetLastError());
  return Err{};
}

Err launch_trace_hits(const ViewDev& view, ViewDev* d_views, const uint32_t* pixels, uint32_t n_pix,
                      uint32_t max_entries, uint32_t* out_pidx, float* out_t, float* out_alpha, uint32_t* out_count,
                      uint32_t* out_rounds, float4* out_rgba, DevCounters* counters, const FaceTable& faces,
                      cudaStream_t stream, uint64_t* launches) {
  if (n_pix == 0) return Err{};
  GT_CUDA_TRY(cudaMemcpyAsync(d_views, &view, sizeof(ViewDev), cudaMemcpyHostToDevice, stream));
  HitOut ho{out_pidx, out_t, out_alpha, out_count, out_rounds, out_rgba, max_entries};
  uint32_t grid = std::min<uint32_t>((n_pix + kWarpsPerBlock - 1) / kWarpsPerBlock, 148u * 8u);
  k_trace8<true, false, 1, true><<<grid, kWarpsPerBlock * 32, 0, stream>>>(d_views, 1, 0, counters, faces, pixels, n_pix, ho,
                                                                  Ckpt{}, nullptr, 0u);
  ++*launches;
  GT_CUDA_TRY(cudaGetLastError());
  return Err{};
}

}  // namespace gt
