// gt_backward.cu — adjoint of the tracer: dLoss/d(particle parameters) from
// dLoss/d(pixel).  No counterpart in the reference (it has no training path,
// README.md:69); the forward it differentiates is tracePath
// (src/GS_shader.ts:192-273) as implemented in gt_trace.cu.
//
// Scheme.  A forward pass writes, per ray and round, t_curr and the
// transmittance T at the round's start (and, in checkpoint mode, the round's
// particle indices).  The adjoint then walks each ray's rounds from the last
// to the first, one warp per ray:
//   * the round's entries come from the checkpoint, or are found again by a
//     traversal from the stored t_curr (replay mode; the set is the same: it is
//     the k closest front-face hits beyond t_curr);
//   * lanes recompute alpha_i and the SH colour c_i of one entry each, and the
//     transmittance before each entry, T_i, in entry order from the stored T
//     (bit-identical to the forward's);
//   * back to front, with R the radiance behind the current entry divided by
//     its transmittance (R <- a c + (1 - a) R, carried across rounds),
//     dL/dalpha_i = T_i (g.c_i - g.R) and dL/dc_i = T_i alpha_i g; no division
//     by (1 - alpha), so alpha close to 1 is harmless;
//   * alpha = opacity * exp(E), E = -(p - mu)^T A (p - mu) at the point of
//     maximum density p, where dE/dtau = 0: mu and A act only directly,
//     dE/dmu = 2 A (p - mu), dE/dA = -(p - mu)(p - mu)^T, A = R S^-2 R^T with
//     R the rotation of the stored quaternion (as computeResponse builds it,
//     src/GS_shader.ts:115-130) and S the scales;
//   * the SH direction normalize(mu - origin) (src/GS_shader.ts:264) adds its
//     own position gradient.
// Hit sets are held fixed: the proxy geometry is piecewise constant.
// Per-particle gradients accumulate with 16-byte vector atomics into a
// particle-major buffer (60 floats per particle) that a final kernel writes
// out parameter-major.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "gt_device.cuh"
#include "gt_handles.h"
#include "gt_internal.cuh"
#include "gt_trace_common.cuh"
#include "gt_warp.cuh"

namespace gt {

// Real SH basis of degree <= deg at direction d and its gradient
// (the polynomials of shToRadiance, src/GS_shader.ts:138-177).
__device__ __forceinline__ void sh_basis(V3 d, uint32_t deg, float B[16], float dB[16][3]) {
  const float x = d.x, y = d.y, z = d.z, xx = x * x, yy = y * y, zz = z * z;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    B[k] = 0.f;
    dB[k][0] = dB[k][1] = dB[k][2] = 0.f;
  }
  B[0] = GT_SH_C0;
  if (deg >= 1) {
    B[1] = -GT_SH_C1 * y; dB[1][1] = -GT_SH_C1;
    B[2] = GT_SH_C1 * z;  dB[2][2] = GT_SH_C1;
    B[3] = -GT_SH_C1 * x; dB[3][0] = -GT_SH_C1;
  }
  if (deg >= 2) {
    B[4] = GT_SH_C2_0 * x * y; dB[4][0] = GT_SH_C2_0 * y; dB[4][1] = GT_SH_C2_0 * x;
    B[5] = GT_SH_C2_1 * y * z; dB[5][1] = GT_SH_C2_1 * z; dB[5][2] = GT_SH_C2_1 * y;
    B[6] = GT_SH_C2_2 * (2.f * zz - xx - yy);
    dB[6][0] = -2.f * GT_SH_C2_2 * x; dB[6][1] = -2.f * GT_SH_C2_2 * y; dB[6][2] = 4.f * GT_SH_C2_2 * z;
    B[7] = GT_SH_C2_3 * x * z; dB[7][0] = GT_SH_C2_3 * z; dB[7][2] = GT_SH_C2_3 * x;
    B[8] = GT_SH_C2_4 * (xx - yy); dB[8][0] = 2.f * GT_SH_C2_4 * x; dB[8][1] = -2.f * GT_SH_C2_4 * y;
  }
  if (deg >= 3) {
    B[9] = GT_SH_C3_0 * y * (3.f * xx - yy);
    dB[9][0] = GT_SH_C3_0 * 6.f * x * y; dB[9][1] = GT_SH_C3_0 * (3.f * xx - 3.f * yy);
    B[10] = GT_SH_C3_1 * x * y * z;
    dB[10][0] = GT_SH_C3_1 * y * z; dB[10][1] = GT_SH_C3_1 * x * z; dB[10][2] = GT_SH_C3_1 * x * y;
    B[11] = GT_SH_C3_2 * y * (4.f * zz - xx - yy);
    dB[11][0] = -2.f * GT_SH_C3_2 * x * y; dB[11][1] = GT_SH_C3_2 * (4.f * zz - xx - 3.f * yy);
    dB[11][2] = 8.f * GT_SH_C3_2 * y * z;
    B[12] = GT_SH_C3_3 * z * (2.f * zz - 3.f * xx - 3.f * yy);
    dB[12][0] = -6.f * GT_SH_C3_3 * x * z; dB[12][1] = -6.f * GT_SH_C3_3 * y * z;
    dB[12][2] = GT_SH_C3_3 * (6.f * zz - 3.f * xx - 3.f * yy);
    B[13] = GT_SH_C3_4 * x * (4.f * zz - xx - yy);
    dB[13][0] = GT_SH_C3_4 * (4.f * zz - 3.f * xx - yy); dB[13][1] = -2.f * GT_SH_C3_4 * x * y;
    dB[13][2] = 8.f * GT_SH_C3_4 * x * z;
    B[14] = GT_SH_C3_5 * z * (xx - yy);
    dB[14][0] = 2.f * GT_SH_C3_5 * x * z; dB[14][1] = -2.f * GT_SH_C3_5 * y * z; dB[14][2] = GT_SH_C3_5 * (xx - yy);
    B[15] = GT_SH_C3_6 * x * (xx - 3.f * yy);
    dB[15][0] = GT_SH_C3_6 * (3.f * xx - 3.f * yy); dB[15][1] = -6.f * GT_SH_C3_6 * x * y;
  }
}

// Per-entry terms of the adjoint.  The 59 parameter gradients of a particle
// are linear in a few sums over its composited entries (alpha > alpha_min),
// so the adjoint adds those sums per particle and k_expand turns them into
// gradients once per particle:
//   response terms, independent of the view (v[0..15]):
//     [0..2]  gE A q                position, through the response
//     [3]     ga resp               opacity
//     [4..6]  gE u_k^2              scales
//     [7..15] gE q_r u_c            rotation (c fastest within r)
//   with q = p - mu at the point of maximum density, u = R^T q in the
//   particle's frame, gE = ga opacity resp = dL/dE;
//   colour weights, per view (v[16..18]):
//     gc = T alpha g                per channel where the SH colour is > 0
//   from which the SH coefficient gradients B_k(dir) gc and the position term
//   of the SH direction dir = normalize(mu - origin) follow; dir is the same
//   for every ray of a view (all primary rays start at the camera).
//   T: transmittance before the entry; a: its alpha; resp: exp(E); craw: SH
//   colour before the clamp; ga: dL/dalpha; g: dL/dpixel (rgb).
__device__ __forceinline__ void entry_terms(const SceneDev& S, uint32_t p, const Shade& sd, V3 o, V3 dr, float T,
                                            float a, float resp, const float craw[3], float ga, const float g[3],
                                            float v[20]) {
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) v[16 + ch] = craw[ch] > 0.f ? T * a * g[ch] : 0.f;
  v[19] = 0.f;
  const float gE = ga * sd.opacity * resp;
  v[3] = ga * resp;
  // q = p - mu is the small difference of two points about |origin - mu|
  // apart, so it is formed in double; A q is nearly orthogonal to the ray and
  // keeps its small components only so
  double aqd[3], qd[3];
  {
    const double a00 = sd.a00, a01 = sd.a01, a02 = sd.a02, a11 = sd.a11, a12 = sd.a12, a22 = sd.a22;
    const double dx = dr.x, dy = dr.y, dz = dr.z;
    const double mx = (double)sd.mu.x - (double)o.x, my = (double)sd.mu.y - (double)o.y,
                 mz = (double)sd.mu.z - (double)o.z;
    const double t0 = a00 * dx + a01 * dy + a02 * dz, t1 = a01 * dx + a11 * dy + a12 * dz,
                 t2 = a02 * dx + a12 * dy + a22 * dz;
    const double tau = (mx * t0 + my * t1 + mz * t2) / (dx * t0 + dy * t1 + dz * t2);
    qd[0] = tau * dx - mx;
    qd[1] = tau * dy - my;
    qd[2] = tau * dz - mz;
    aqd[0] = a00 * qd[0] + a01 * qd[1] + a02 * qd[2];
    aqd[1] = a01 * qd[0] + a11 * qd[1] + a12 * qd[2];
    aqd[2] = a02 * qd[0] + a12 * qd[1] + a22 * qd[2];
  }
  const float q[3] = {(float)qd[0], (float)qd[1], (float)qd[2]};
  const float4 qa = __ldg(S.params + 2 * (size_t)p + 1);
  const float qw = qa.x, qx = qa.y, qy = qa.z, qz = qa.w;
  // rotation of the quaternion (rows); computeResponse's matrix is its transpose
  const float R[3][3] = {{1.f - 2.f * (qy * qy + qz * qz), 2.f * (qx * qy - qw * qz), 2.f * (qx * qz + qw * qy)},
                         {2.f * (qx * qy + qw * qz), 1.f - 2.f * (qx * qx + qz * qz), 2.f * (qy * qz - qw * qx)},
                         {2.f * (qx * qz - qw * qy), 2.f * (qy * qz + qw * qx), 1.f - 2.f * (qx * qx + qy * qy)}};
  float u[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) u[k] = R[0][k] * q[0] + R[1][k] * q[1] + R[2][k] * q[2];
  const float gu0 = gE * u[0], gu1 = gE * u[1], gu2 = gE * u[2];
  v[0] = gE * (float)aqd[0];
  v[1] = gE * (float)aqd[1];
  v[2] = gE * (float)aqd[2];
  v[4] = gu0 * u[0];
  v[5] = gu1 * u[1];
  v[6] = gu2 * u[2];
  v[7] = gu0 * q[0];
  v[8] = gu1 * q[0];
  v[9] = gu2 * q[0];
  v[10] = gu0 * q[1];
  v[11] = gu1 * q[1];
  v[12] = gu2 * q[1];
  v[13] = gu0 * q[2];
  v[14] = gu1 * q[2];
  v[15] = gu2 * q[2];
}

// Per-warp table of per-particle sums.  The rays of one 8x4 tile composite
// mostly the same particles, so the warp adds its tile's entry terms here
// (shared-memory atomics; the entries of one round are distinct particles
// but for shared-edge duplicates) and each particle's sums reach global
// memory once per tile: 5 vector atomics per particle and tile instead of
// per entry.
constexpr int kAggSlots = 64;
struct AggTable {
  uint32_t key[kAggSlots];     // particle index, kInvalid when empty
  float val[20][kAggSlots];    // sum i of slot h at val[i][h]: the 16 response sums, the 3 colour sums, 0
};
// (component-major: lanes adding to different slots meet in one bank only
// when their slots are 32 apart)

__device__ __forceinline__ void agg_clear(AggTable& A, uint32_t lane) {
  for (uint32_t i = lane; i < (uint32_t)kAggSlots; i += 32) {
    A.key[i] = kInvalid;
#pragma unroll
    for (int c = 0; c < 20; ++c) A.val[c][i] = 0.f;
  }
  __syncwarp();
}

// Adds the terms v of particle p; returns whether p took an empty slot.  The
// caller keeps at most kAggSlots particles in the table, so the probe finds
// p or an empty slot within kAggSlots steps; past them (never) the terms go
// straight to global memory.
__device__ __forceinline__ bool agg_add(AggTable& A, uint32_t p, const float v[20], float4* G, float4* GS) {
  uint32_t h = (p * 2654435761u) >> 26;
  for (int step = 0; step < kAggSlots; ++step) {
    const uint32_t prev = atomicCAS(&A.key[h], kInvalid, p);
    if (prev == kInvalid || prev == p) {
#pragma unroll
      for (int i = 0; i < 19; ++i)
        if (v[i] != 0.f) atomicAdd(&A.val[i][h], v[i]);
      return prev == kInvalid;
    }
    h = (h + 1) & (kAggSlots - 1);
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
    atomicAdd(G + 4 * (size_t)p + c, make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]));
  atomicAdd(GS + p, make_float4(v[16], v[17], v[18], 0.f));
  return false;
}

// Adds the table to the scene's response sums G and the view's colour sums
// GS and empties it.
__device__ __forceinline__ void agg_flush(AggTable& A, float4* G, float4* GS, uint32_t lane) {
  __syncwarp();
  for (uint32_t i = lane; i < (uint32_t)kAggSlots; i += 32) {
    const uint32_t p = A.key[i];
    if (p == kInvalid) continue;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const float4 x = make_float4(A.val[4 * c][i], A.val[4 * c + 1][i], A.val[4 * c + 2][i], A.val[4 * c + 3][i]);
      if (x.x != 0.f || x.y != 0.f || x.z != 0.f || x.w != 0.f) atomicAdd(c < 4 ? G + 4 * (size_t)p + c : GS + p, x);
      A.val[4 * c][i] = 0.f;
      A.val[4 * c + 1][i] = 0.f;
      A.val[4 * c + 2][i] = 0.f;
      A.val[4 * c + 3][i] = 0.f;
    }
    A.key[i] = kInvalid;
  }
  __syncwarp();
}

// The adjoint, one warp per 8x4 tile of ray slots (the forward's slot
// numbering): the tiles [tile_begin, tile_end) of the launch's views.  The
// warp splits into 32 / SEG segments of SEG lanes, each walking one of the
// tile's rays (a record's up to SEG contributing entries across its lanes);
// the tile's per-particle sums gather in the warp's table.  Replay mode (a
// round's entries found again by a warp-wide traversal) runs with SEG = 32.
template <bool CKPT_PIDX, int SEG>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 4) k_backward(const ViewDev* __restrict__ views,
                                                                    uint32_t n_views, uint32_t tile_begin,
                                                                    uint32_t tile_end, DevCounters* ctr,
                                                                    const __grid_constant__ FaceTable F,
                                                                    const Ckpt ck) {
  static_assert(SEG == 8 || SEG == 16 || SEG == 32, "segment width");
  static_assert(CKPT_PIDX || SEG == 32, "replay traverses with the whole warp");
  constexpr uint32_t kGroups = 32 / SEG;
  __shared__ WarpScratch scratch[kWarpsPerBlock];
  __shared__ AggTable tables[kWarpsPerBlock];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t seg = lane / SEG, sl_lane = lane % SEG;
  const uint32_t seg_shift = seg * SEG;
  const uint32_t seg_bits = SEG == 32 ? kFull : ((1u << SEG) - 1u);
  WarpScratch& W = scratch[threadIdx.x >> 5];
  AggTable& A = tables[threadIdx.x >> 5];
  RayStats& st = W.stats;
  if (lane == 0) st = RayStats{0, 0, 0, 0, 0, 0};
  agg_clear(A, lane);
  uint32_t status = 0, rays = 0, n_rounds = 0, n_entries = 0, n_contrib = 0;
  while (true) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(&ctr->work, 1u);
    tile = __shfl_sync(kFull, tile, 0);
    if (tile >= tile_end - tile_begin) break;
    tile += tile_begin;
    const uint32_t vi = n_views == 1 ? 0u : find_view(views, n_views, tile);
    const ViewDev& V = views[vi];
    const uint32_t k = V.u.k;
    uint32_t nfill = 0;  // particles in the table
    for (uint32_t base = 0; base < 32; base += kGroups) {
      // this segment's ray
      const uint32_t sl = base + seg;
      const uint32_t item = 32u * tile + sl;
      uint32_t px, py;
      tile_pixel(V.tiles_x, tile - V.tile_begin, sl, px, py);
      uint32_t rec = kInvalid;
      float g[3] = {0.f, 0.f, 0.f};
      if (px < V.w && py < V.h) {
        const float4 g4 = V.dL[(size_t)py * V.w + px];
        if (g4.x != 0.f || g4.y != 0.f || g4.z != 0.f) {
          rec = ck.head[item];
          g[0] = g4.x;
          g[1] = g4.y;
          g[2] = g4.z;
        }
      }
      V3 o = mk(0.f, 0.f, 0.f), d = mk(0.f, 0.f, 1.f);
      if (rec != kInvalid) ray_gen(V.u, V.w, V.h, px, py, o, d);
      const BoxRay br = make_boxray(o, d, V.s.scene_mag);
      if (rec != kInvalid && sl_lane == 0) ++rays;
      float S = 0.f;  // g.R: the colour composited behind the current round, dotted with g
      // records from the last to the first along their links, all segments
      // in step (a segment whose ray is done idles)
      for (uint32_t guard = 0; guard < ck.pool_cap; ++guard) {
        const bool active = rec != kInvalid;
        if (!__any_sync(kFull, active)) break;
        uint32_t p = kInvalid, nrec = 0;
        float2 ri = make_float2(0.f, 0.f);
        bool valid = false;
        if (CKPT_PIDX) {
          if (active) {
            const uint32_t* rr = ck.pool + (size_t)rec * (kCkptHeader + ck.kc);
            ri = make_float2(__uint_as_float(rr[0]), __uint_as_float(rr[1]));
            nrec = rr[3];
            p = sl_lane < ck.kc ? rr[kCkptHeader + sl_lane] : kInvalid;
            valid = sl_lane < nrec && p != kInvalid;
            rec = rr[2];
          }
        } else {
          const uint32_t* rr = ck.pool + (size_t)rec * (kCkptHeader + ck.kc);
          ri = make_float2(__uint_as_float(rr[0]), __uint_as_float(rr[1]));
          nrec = rr[3];
          KBuf<1> kb;
          kbuf_init(kb, V.u.t_max);
          traverse8<kCollect>(V.s, F, W, o, d, br, ri.x, V.u.t_max, kb, st, status, lane, (int)k, V.leaf_batch);
          if (__reduce_or_sync(kFull, status) & (kStatusStackOverflow | kStatusVisitCap | kStatusHitOverflow)) {
            rec = kInvalid;
            break;
          }
          valid = lane < k && lane < nrec && kb.p[0] != kInvalid;
          p = kb.p[0];
          rec = rr[2];
        }
        const uint32_t vmask = (__ballot_sync(kFull, valid) >> seg_shift) & seg_bits;
        const int n = __popc(vmask);
        float alpha = 0.f, resp = 0.f;
        float craw[3] = {0.f, 0.f, 0.f};
        Shade sd;
        bool contrib = false;
        if (valid) {
          sd = load_shade(V.s.shade, p);
          resp = response(sd, o, d);
          alpha = resp * sd.opacity;
          contrib = V.u.alpha_min < alpha;
          if (contrib) {
            if (V.rgb) {
              // the view's colour table holds max(0, craw): the same signs
              // and clamped values, which is all the adjoint uses of craw
              const float4 q = __ldg(V.rgb + p);
              craw[0] = q.x;
              craw[1] = q.y;
              craw[2] = q.z;
            } else {
              sh_radiance(V.s.sh, p, vnorm(vsub(sd.mu, o)), V.u.deg, craw);
            }
          }
        }
        const uint32_t cballot = __ballot_sync(kFull, contrib);
        const uint32_t cmask = (cballot >> seg_shift) & seg_bits;
        // transmittance before each entry: the round's starting T times the
        // product of (1 - alpha) over the contributing entries ahead of it
        // (an exclusive product scan across the segment's lanes)
        const float keep = contrib ? 1.0f - alpha : 1.0f;
        float pre = keep;
#pragma unroll
        for (int off = 1; off < SEG; off <<= 1) {
          const float x = __shfl_up_sync(kFull, pre, off, SEG);
          if ((int)sl_lane >= off) pre *= x;
        }
        float ahead = __shfl_up_sync(kFull, pre, 1, SEG);
        if (sl_lane == 0) ahead = 1.0f;
        const float Tme = ri.y * ahead;
        // dL/dalpha of entry e: T_e (g.c_e - g.R_e), R_e the colour composited
        // behind e (normalised by T_e (1 - a_e)), i.e. the entries after e in
        // this round and the later rounds' S.  Behind-colours follow
        // x -> a_e s_e + (1 - a_e) x from the back, so they are an inclusive
        // suffix scan of these affine maps (composed through shuffles).
        float sv = 0.f;
        if (contrib) {
          const float c0 = craw[0] > 0.f ? craw[0] : 0.f, c1 = craw[1] > 0.f ? craw[1] : 0.f,
                      c2 = craw[2] > 0.f ? craw[2] : 0.f;
          sv = g[0] * c0 + g[1] * c1 + g[2] * c2;
        }
        float fm = keep, fb = contrib ? alpha * sv : 0.f;  // map of entries e.. (from e to the round's end)
#pragma unroll
        for (int off = 1; off < SEG; off <<= 1) {
          const float xm = __shfl_down_sync(kFull, fm, off, SEG);
          const float xb = __shfl_down_sync(kFull, fb, off, SEG);
          if ((int)sl_lane + off < SEG) {
            fb = __fmaf_rn(fm, xb, fb);
            fm = fm * xm;
          }
        }
        float nm = __shfl_down_sync(kFull, fm, 1, SEG), nb = __shfl_down_sync(kFull, fb, 1, SEG);
        if ((int)sl_lane + 1 >= SEG) {
          nm = 1.0f;
          nb = 0.0f;
        }
        const float ga = contrib ? Tme * (sv - __fmaf_rn(nm, S, nb)) : 0.f;
        S = __fmaf_rn(__shfl_sync(kFull, fm, 0, SEG), S, __shfl_sync(kFull, fb, 0, SEG));
        // room for this step's particles (all segments) in the table
        const uint32_t nc_all = (uint32_t)__popc(cballot);
        if (nfill + nc_all > (uint32_t)kAggSlots) {
          agg_flush(A, V.grad, V.grad_sh, lane);
          nfill = 0;
        }
        bool fresh = false;
        if (contrib) {
          float v[20];
          entry_terms(V.s, p, sd, o, d, Tme, alpha, resp, craw, ga, g, v);
          fresh = agg_add(A, p, v, V.grad, V.grad_sh);
        }
        nfill += (uint32_t)__popc(__ballot_sync(kFull, fresh));
        if (active && sl_lane == 0) {
          ++n_rounds;
          n_entries += (uint32_t)n;
          n_contrib += (uint32_t)__popc(cmask);
        }
      }
    }
    // the next tile may be another view's (other colour sums) or scene's
    agg_flush(A, V.grad, V.grad_sh, lane);
  }
  {
    const uint32_t r_ = __reduce_add_sync(kFull, n_rounds), e_ = __reduce_add_sync(kFull, n_entries),
                   c_ = __reduce_add_sync(kFull, n_contrib);
    if (lane == 0) {
      st.rounds += r_;
      st.entries += e_;
      st.contributing += c_;
    }
    __syncwarp();
  }
  flush_stats(ctr, st, __reduce_add_sync(kFull, rays), status);
}

// One view's share of the SH terms of a scene's particles: the camera
// position, the view's SH degree and its colour-weight sums (1 float4 a
// particle).
struct ExpandView {
  float ox, oy, oz;
  uint32_t deg;
  const float4* gs;
};

// The 59 gradients of particle p from its sums (entry_terms), written
// parameter-major: out[i * n + p] (+)= dL/dparam_i.
__global__ void __launch_bounds__(128) k_expand(const float4* __restrict__ G, const ExpandView* __restrict__ ev,
                                                uint32_t n_ev, SceneDev S, uint64_t n, float* __restrict__ out,
                                                bool accumulate) {
  const uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  const float4 r0 = G[4 * p], r1 = G[4 * p + 1], r2 = G[4 * p + 2], r3 = G[4 * p + 3];
  const float4 sa = __ldg(S.params + 2 * p), qa = __ldg(S.params + 2 * p + 1);
  const float s[3] = {sa.x, sa.y, sa.z};
  const float qw = qa.x, qx = qa.y, qy = qa.z, qz = qa.w;
  float head[11];
  // particles without composited entries (among them those below the opacity
  // cut, whose scales may be 0) have zero sums: their response terms are 0
  const bool any = r0.x != 0.f || r0.y != 0.f || r0.z != 0.f || r0.w != 0.f || r1.x != 0.f || r1.y != 0.f ||
                   r1.z != 0.f || r1.w != 0.f || r2.x != 0.f || r2.y != 0.f || r2.z != 0.f || r2.w != 0.f ||
                   r3.x != 0.f || r3.y != 0.f || r3.z != 0.f || r3.w != 0.f;
  head[0] = 2.f * r0.x;
  head[1] = 2.f * r0.y;
  head[2] = 2.f * r0.z;
  head[10] = r0.w;
  const float U[3] = {r1.x, r1.y, r1.z};
#pragma unroll
  for (int k = 0; k < 3; ++k) head[3 + k] = 2.f * U[k] / (s[k] * s[k] * s[k]);
  // sum gE q_r u_c, and GR = dL/dR(r, c) = -2 sum gE q_r u_c / s_c^2
  const float M[3][3] = {{r1.w, r2.x, r2.y}, {r2.z, r2.w, r3.x}, {r3.y, r3.z, r3.w}};
  float GR[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) GR[r][c] = -2.f * M[r][c] / (s[c] * s[c]);
  head[6] = 2.f * (-qz * GR[0][1] + qy * GR[0][2] + qz * GR[1][0] - qx * GR[1][2] - qy * GR[2][0] + qx * GR[2][1]);
  head[7] = 2.f * (qy * GR[0][1] + qz * GR[0][2] + qy * GR[1][0] - 2.f * qx * GR[1][1] - qw * GR[1][2] +
                   qz * GR[2][0] + qw * GR[2][1] - 2.f * qx * GR[2][2]);
  head[8] = 2.f * (-2.f * qy * GR[0][0] + qx * GR[0][1] + qw * GR[0][2] + qx * GR[1][0] + qz * GR[1][2] -
                   qw * GR[2][0] + qz * GR[2][1] - 2.f * qy * GR[2][2]);
  head[9] = 2.f * (-2.f * qz * GR[0][0] - qw * GR[0][1] + qx * GR[0][2] + qw * GR[1][0] - 2.f * qz * GR[1][1] +
                   qy * GR[1][2] + qx * GR[2][0] + qy * GR[2][1]);
  if (!any)
#pragma unroll
    for (int i = 3; i < 10; ++i) head[i] = 0.f;
  // SH coefficients, B_k(dir) sum gc, and the position term of dir
  float gsh[48];
#pragma unroll
  for (int i = 0; i < 48; ++i) gsh[i] = 0.f;
  const float4 m4 = __ldg(S.shade + 3 * p);
  const V3 mu = mk(m4.x, m4.y, m4.z);
  for (uint32_t v = 0; v < n_ev; ++v) {
    const float4 gc4 = ev[v].gs[p];
    if (gc4.x == 0.f && gc4.y == 0.f && gc4.z == 0.f) continue;
    const float gc[3] = {gc4.x, gc4.y, gc4.z};
    const V3 d0 = vsub(mu, mk(ev[v].ox, ev[v].oy, ev[v].oz));
    const float len = sqrtf(vdot(d0, d0));
    const V3 dir = mk(d0.x / len, d0.y / len, d0.z / len);
    float B[16], dB[16][3];
    sh_basis(dir, ev[v].deg, B, dB);
    const float4* shp = S.sh + 12 * p;
    float dd0 = 0.f, dd1 = 0.f, dd2 = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float4 c0 = __ldg(shp + 3 * i), c1 = __ldg(shp + 3 * i + 1), c2 = __ldg(shp + 3 * i + 2);
      const float sv[12] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w, c2.x, c2.y, c2.z, c2.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = 4 * i + j;
        const float sg = sv[3 * j] * gc[0] + sv[3 * j + 1] * gc[1] + sv[3 * j + 2] * gc[2];
        dd0 += dB[k][0] * sg;
        dd1 += dB[k][1] * sg;
        dd2 += dB[k][2] * sg;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) gsh[3 * k + ch] += B[k] * gc[ch];
      }
    }
    const float dd = dd0 * dir.x + dd1 * dir.y + dd2 * dir.z;
    head[0] += (dd0 - dir.x * dd) / len;
    head[1] += (dd1 - dir.y * dd) / len;
    head[2] += (dd2 - dir.z * dd) / len;
  }
#pragma unroll
  for (int i = 0; i < 11; ++i) {
    float* o = out + (uint64_t)i * n + p;
    *o = accumulate ? *o + head[i] : head[i];
  }
#pragma unroll
  for (int i = 0; i < 48; ++i) {
    float* o = out + (uint64_t)(11 + i) * n + p;
    *o = accumulate ? *o + gsh[i] : gsh[i];
  }
}

// Writes the L2 loss gradient and per-block partial sums of the loss.
__global__ void k_l2_loss(const float4* rgba, const float4* target, uint64_t n, float4* dL, double* partial) {
  __shared__ double red[256];
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < n) {
    float4 a = rgba[i], b = target[i];
    float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    dL[i] = make_float4(2.f * dx, 2.f * dy, 2.f * dz, 0.f);
    v = (double)dx * dx + (double)dy * dy + (double)dz * dz;
  }
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

}  // namespace gt

using namespace gt;

namespace {

struct BwdView {
  const gt_scene* scene;
  gt_uniforms u;
  uint32_t w, h;
  const float* dL;
};

#define CK_TRY(expr)                                                                                     \
  do {                                                                                                   \
    cudaError_t e_ = (expr);                                                                             \
    if (e_ != cudaSuccess)                                                                               \
      return api_fail(ctx, e_ == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA,                     \
                      std::string(#expr) + ": " + cudaGetErrorString(e_));                               \
  } while (0)

// Grows a context-owned device buffer to at least `bytes`, with a quarter
// more room so that slowly growing needs (the records of successive
// checkpointing forwards) do not free and allocate on every call.
gt_status grow(gt_context* ctx, void** p, size_t* have, size_t bytes) {
  if (*have >= bytes) return GT_OK;
  cudaFree(*p);
  *p = nullptr;
  *have = 0;
  const size_t want = bytes + bytes / 4;
  CK_TRY(cudaMalloc(p, want ? want : 16));
  *have = want;
  return GT_OK;
}

bool key_matches(const CkptStore& ck, const BwdView* v, uint32_t count) {
  if (!ck.valid || ck.key.size() != count) return false;
  for (uint32_t i = 0; i < count; ++i) {
    const CkptKey& k = ck.key[i];
    if (k.scene != v[i].scene || k.w != v[i].w || k.h != v[i].h || memcmp(&k.u, &v[i].u, sizeof(gt_uniforms)) != 0)
      return false;
  }
  return true;
}

}  // namespace

namespace gt {

void api_free_ckpt(gt_context* ctx) {
  CkptStore& c = ctx->ckpt;
  cudaFree(c.head);
  cudaFree(c.pool);
  cudaFree(c.pool_next);
  c = CkptStore{};
}

// Checkpointing forward: renders the views into `outs` and keeps one record
// per traced round (see Ckpt).  Mode 1 stores the rounds' particle indices
// (no traversal in the adjoint) when the records fit in `budget` bytes;
// mode 2 stores only (t_curr, T) and the adjoint finds each round's entries
// again.  The pool is sized from the previous call; when the rounds outgrow
// it, the forward runs again with the exact size.
gt_status api_forward_ckpt(gt_context* ctx, const gt_scene* const* scenes, const gt_uniforms* us, const uint32_t* ws,
                           const uint32_t* hs, float4* const* outs, uint32_t count, uint32_t mode, uint32_t cap,
                           uint64_t budget, gt_render_stats* stats) {
  CkptStore& ck = ctx->ckpt;
  ck.valid = false;
  cudaStream_t st = ctx->stream;
  gt_status sst = api_ensure_views(ctx, count);
  if (sst != GT_OK) return sst;
  std::vector<ViewDev> vd(count);
  uint32_t total_tiles = 0;
  uint64_t rays = 0;
  for (uint32_t i = 0; i < count; ++i) {
    vd[i] = api_make_view(scenes[i], us[i], ws[i], hs[i], outs[i], total_tiles);
    total_tiles += vd[i].n_tiles;
    rays += (uint64_t)ws[i] * hs[i];
  }
  const uint64_t slots = (uint64_t)total_tiles * 32u;
  if (budget == 0) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    budget = free_b / 2 + ck.pool_bytes;  // the pool we hold counts as available
  }
  // first guess of the records: the last call's count, else 4 a ray
  uint64_t want = ck.last_records ? ck.last_records + ck.last_records / 8 + 1024 : rays * 4 + 1024;
  if (cap) want = std::max<uint64_t>(want, rays * (uint64_t)cap);
  if (!ck.pool_next) CK_TRY(cudaMalloc(&ck.pool_next, 4));
  sst = grow(ctx, (void**)&ck.head, &ck.head_bytes, slots * 4);
  if (sst != GT_OK) return sst;
  LaunchShape shape = api_batch_shape_for(ctx, scenes, us, ws, hs, count, total_tiles);
  Handoff hand;
  sst = api_ensure_handoff(ctx, rays, &hand);
  if (sst != GT_OK) return sst;
  sst = api_assign_colours(ctx, vd.data(), count);  // as a plain render's
  if (sst != GT_OK) return sst;
  for (int attempt = 0; attempt < 3; ++attempt) {
    if (want > 0xFFFFFFF0ull) return api_fail(ctx, GT_ERR_OOM, "checkpoint needs more than 2^32 records");
    uint32_t m = mode == 1 ? 1u : (mode == 2 ? 2u : (want * (kCkptHeader + kCkptChunk) * 4 <= budget ? 1u : 2u));
    const uint32_t kc = m == 1 ? kCkptChunk : 0u;
    sst = grow(ctx, (void**)&ck.pool, &ck.pool_bytes, want * (kCkptHeader + kc) * 4);
    if (sst != GT_OK) return sst;
    Ckpt c;
    c.head = ck.head;
    c.pool = ck.pool;
    c.pool_next = ck.pool_next;
    c.pool_cap = (uint32_t)std::min<uint64_t>(ck.pool_bytes / ((kCkptHeader + kc) * 4), 0xFFFFFFF0ull);
    c.kc = kc;
    CK_TRY(cudaMemsetAsync(ck.head, 0xFF, slots * 4, st));
    CK_TRY(cudaMemsetAsync(ck.pool_next, 0, 4, st));
    CK_TRY(cudaMemsetAsync(ctx->d_ctr, 0, sizeof(DevCounters), st));
    CK_TRY(cudaEventRecord(ctx->int0, st));
    Err e = launch_trace(vd.data(), count, total_tiles, ctx->d_ctr, ctx->faces, shape, ctx->num_sms, st,
                         &ctx->launches, ctx->d_views, &c, &hand);
    if (e.code != GT_OK) return api_fail(ctx, e.code, e.msg);
    CK_TRY(cudaEventRecord(ctx->int1, st));
    uint32_t used = 0;
    CK_TRY(cudaMemcpyAsync(&used, ck.pool_next, 4, cudaMemcpyDeviceToHost, st));
    CK_TRY(cudaMemcpyAsync(ctx->h_ctr, ctx->d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, st));
    CK_TRY(cudaStreamSynchronize(st));
    cudaEventElapsedTime(&ck.fwd_ms, ctx->int0, ctx->int1);
    sst = api_status_to_error(ctx, ctx->h_ctr->status);
    if (sst != GT_OK) return sst;
    if (stats) {
      memset(stats, 0, sizeof *stats);
      api_fill_stats(*ctx->h_ctr, stats);
      stats->kernel_ms = ck.fwd_ms;
      stats->total_ms = ck.fwd_ms;
    }
    ck.last_records = used;
    if (used <= c.pool_cap) {
      ck.slots = slots;
      ck.pool_cap = c.pool_cap;
      ck.kc = kc;
      ck.mode = m;
      ck.total_tiles = total_tiles;
      ck.key.resize(count);
      for (uint32_t i = 0; i < count; ++i) ck.key[i] = CkptKey{scenes[i], us[i], ws[i], hs[i]};
      ck.valid = true;
      return GT_OK;
    }
    want = (uint64_t)used + 1024;  // exact size for the second run
  }
  return api_fail(ctx, GT_ERR_DEVICE_TIMEOUT, "checkpoint pool kept overflowing");
}

}  // namespace gt

namespace {

gt_status backward_impl(gt_context* ctx, const BwdView* views, uint32_t count, const gt_scene* const* scenes,
                        float* const* outs, uint32_t n_scenes, uint32_t flags, gt_bwd_opts* opts,
                        gt_render_stats* stats) {
  if (count == 0) return GT_OK;
  CK_TRY(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  std::vector<void*> temps;
  auto cleanup = [&]() {
    for (void* p : temps) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
  };
  auto talloc = [&](void** p, size_t bytes) -> cudaError_t {
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, st);
    if (e == cudaSuccess) temps.push_back(*p);
    return e;
  };
#define BWD_TRY(expr)                                                                                     \
  do {                                                                                                    \
    cudaError_t e_ = (expr);                                                                              \
    if (e_ != cudaSuccess) {                                                                              \
      cleanup();                                                                                          \
      return api_fail(ctx, e_ == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA,                      \
                      std::string(#expr) + ": " + cudaGetErrorString(e_));                                \
    }                                                                                                     \
  } while (0)
  size_t pixels = 0;
  for (uint32_t i = 0; i < count; ++i) pixels += (size_t)views[i].w * views[i].h;
  // 1. the checkpointing forward, unless the context holds it for these views
  float fwd_ms = 0.f;
  const bool reuse = (flags & GT_FLAG_CHECKPOINT) && key_matches(ctx->ckpt, views, count);
  if (!reuse) {
    float4* img = nullptr;
    BWD_TRY(talloc((void**)&img, pixels * sizeof(float4)));
    std::vector<const gt_scene*> sc(count);
    std::vector<gt_uniforms> us(count);
    std::vector<uint32_t> ws(count), hs(count);
    std::vector<float4*> os(count);
    size_t off = 0;
    for (uint32_t i = 0; i < count; ++i) {
      sc[i] = views[i].scene;
      us[i] = views[i].u;
      ws[i] = views[i].w;
      hs[i] = views[i].h;
      os[i] = img + off;
      off += (size_t)views[i].w * views[i].h;
    }
    gt_status sst = api_forward_ckpt(ctx, sc.data(), us.data(), ws.data(), hs.data(), os.data(), count,
                                     opts ? opts->mode : 0u, opts ? opts->max_rounds : 0u,
                                     opts ? opts->mem_budget : 0ull, nullptr);
    if (sst != GT_OK) {
      cleanup();
      return sst;
    }
    fwd_ms = ctx->ckpt.fwd_ms;
  }
  const CkptStore& cs = ctx->ckpt;
  // 2. dL on the device and the adjoint's view table
  float4* dl_dev = nullptr;
  if (!(flags & GT_FLAG_INPUT_DEVICE)) BWD_TRY(talloc((void**)&dl_dev, pixels * sizeof(float4)));
  gt_status sst = api_ensure_views(ctx, count);
  if (sst != GT_OK) {
    cleanup();
    return sst;
  }
  std::vector<ViewDev> vd(count);
  std::vector<uint32_t> vscene(count);
  uint32_t total_tiles = 0;
  size_t off = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const BwdView& bv = views[i];
    vd[i] = api_make_view(bv.scene, bv.u, bv.w, bv.h, nullptr, total_tiles);
    total_tiles += vd[i].n_tiles;
    size_t px = (size_t)bv.w * bv.h;
    if (flags & GT_FLAG_INPUT_DEVICE) {
      vd[i].dL = reinterpret_cast<const float4*>(bv.dL);
    } else {
      BWD_TRY(cudaMemcpyAsync(dl_dev + off, bv.dL, px * sizeof(float4), cudaMemcpyHostToDevice, st));
      vd[i].dL = dl_dev + off;
    }
    uint32_t s = 0;
    while (s < n_scenes && scenes[s] != bv.scene) ++s;
    vscene[i] = s;
    off += px;
  }
  // 3. per-scene sums of the response terms (4 float4 a particle) and per-view
  //    colour sums (1 float4 a particle of the view's scene).  Views go in
  //    groups whose colour sums fit the budget; each group is one adjoint
  //    launch over its tile range and one expansion per scene.
  std::vector<float4*> G(n_scenes, nullptr);
  for (uint32_t s = 0; s < n_scenes; ++s)
    BWD_TRY(talloc((void**)&G[s], (size_t)std::max<uint64_t>(scenes[s]->n, 1) * 4 * sizeof(float4)));
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t gs_budget =
      (opts && opts->mem_budget) ? (size_t)opts->mem_budget : std::max<size_t>((size_t)256 << 20, free_b / 4);
  std::vector<uint32_t> group_end;
  size_t gs_max = 0;
  {
    size_t acc = 0;
    for (uint32_t i = 0; i < count; ++i) {
      const size_t b = (size_t)std::max<uint64_t>(scenes[vscene[i]]->n, 1) * sizeof(float4);
      if (acc > 0 && acc + b > gs_budget) {
        group_end.push_back(i);
        acc = 0;
      }
      acc += b;
      gs_max = std::max(gs_max, acc);
    }
    group_end.push_back(count);
  }
  float4* gs_all = nullptr;
  BWD_TRY(talloc((void**)&gs_all, gs_max));
  ExpandView* d_ev = nullptr;
  BWD_TRY(talloc((void**)&d_ev, sizeof(ExpandView) * count));
  std::vector<ExpandView> hev(count);
  const LaunchShape shape = api_shape_for(ctx, views[0].scene, views[0].w, views[0].h, views[0].u.k);
  apply_shape(vd.data(), count, shape);
  sst = api_assign_colours(ctx, vd.data(), count);  // filled before the first adjoint launch
  if (sst != GT_OK) {
    cleanup();
    return sst;
  }
  Ckpt ck;
  ck.head = cs.head;
  ck.pool = cs.pool;
  ck.pool_next = cs.pool_next;
  ck.pool_cap = cs.pool_cap;
  ck.kc = cs.kc;
  std::vector<float*> dev_out(n_scenes, nullptr);
  for (uint32_t s = 0; s < n_scenes; ++s) {
    const uint64_t n = scenes[s]->n;
    dev_out[s] = outs[s];
    if (n == 0 || (flags & GT_FLAG_OUTPUT_DEVICE)) continue;
    BWD_TRY(talloc((void**)&dev_out[s], n * GT_PARAMS_PER_PARTICLE * 4));
    if (flags & GT_FLAG_ACCUMULATE)
      BWD_TRY(cudaMemcpyAsync(dev_out[s], outs[s], n * GT_PARAMS_PER_PARTICLE * 4, cudaMemcpyHostToDevice, st));
  }
  float bwd_ms = 0.f;
  BWD_TRY(cudaMemsetAsync(ctx->d_ctr, 0, sizeof(DevCounters), st));
  BWD_TRY(cudaEventRecord(ctx->int0, st));
  uint32_t g0 = 0;
  for (size_t gi = 0; gi < group_end.size(); ++gi) {
    const uint32_t g1 = group_end[gi];
    size_t gs_off = 0;
    for (uint32_t i = g0; i < g1; ++i) {
      const ViewDev& v = vd[i];
      const uint64_t n = std::max<uint64_t>(scenes[vscene[i]]->n, 1);
      vd[i].grad = G[vscene[i]];
      vd[i].grad_sh = gs_all + gs_off;
      hev[i] = ExpandView{v.u.tw[12], v.u.tw[13], v.u.tw[14], v.u.deg, gs_all + gs_off};
      gs_off += n;
    }
    for (uint32_t s = 0; s < n_scenes; ++s)
      BWD_TRY(cudaMemsetAsync(G[s], 0, (size_t)std::max<uint64_t>(scenes[s]->n, 1) * 4 * sizeof(float4), st));
    BWD_TRY(cudaMemsetAsync(gs_all, 0, gs_off * sizeof(float4), st));
    BWD_TRY(cudaMemcpyAsync(ctx->d_views, vd.data(), sizeof(ViewDev) * count, cudaMemcpyHostToDevice, st));
    if (gi == 0) {
      Err ce = launch_view_colours(vd.data(), ctx->d_views, count, ctx->num_sms, st, &ctx->launches);
      if (ce.code != GT_OK) {
        cleanup();
        return api_fail(ctx, ce.code, ce.msg);
      }
    }
    BWD_TRY(cudaMemsetAsync(&ctx->d_ctr->work, 0, sizeof(uint32_t), st));
    {
      const uint32_t tile0 = vd[g0].tile_begin;
      const uint32_t tile1 = vd[g1 - 1].tile_begin + vd[g1 - 1].n_tiles;
      uint32_t block = kWarpsPerBlock * 32;
      uint32_t grid = (uint32_t)ctx->num_sms * 4u;  // 4 resident blocks an SM (launch bounds)
      uint64_t max_grid = ((uint64_t)(tile1 - tile0) + kWarpsPerBlock - 1) / kWarpsPerBlock;
      if (grid > max_grid) grid = (uint32_t)std::max<uint64_t>(1, max_grid);
      // lanes per ray: the record's entry slots
      if (cs.mode == 1 && cs.kc <= 8)
        k_backward<true, 8><<<grid, block, 0, st>>>(ctx->d_views, count, tile0, tile1, ctx->d_ctr, ctx->faces, ck);
      else if (cs.mode == 1 && cs.kc <= 16)
        k_backward<true, 16><<<grid, block, 0, st>>>(ctx->d_views, count, tile0, tile1, ctx->d_ctr, ctx->faces, ck);
      else if (cs.mode == 1)
        k_backward<true, 32><<<grid, block, 0, st>>>(ctx->d_views, count, tile0, tile1, ctx->d_ctr, ctx->faces, ck);
      else
        k_backward<false, 32><<<grid, block, 0, st>>>(ctx->d_views, count, tile0, tile1, ctx->d_ctr, ctx->faces, ck);
      ++ctx->launches;
      BWD_TRY(cudaGetLastError());
    }
    // 4. parameter-major gradients of each scene from its sums and its views' colour sums
    for (uint32_t s = 0; s < n_scenes; ++s) {
      const uint64_t n = scenes[s]->n;
      if (n == 0) continue;
      // this group's views of scene s, uploaded as one run of the table
      std::vector<ExpandView> mine;
      for (uint32_t i = g0; i < g1; ++i)
        if (vscene[i] == s) mine.push_back(hev[i]);
      ExpandView* evs = d_ev + g0;
      if (!mine.empty())
        BWD_TRY(cudaMemcpyAsync(evs, mine.data(), sizeof(ExpandView) * mine.size(), cudaMemcpyHostToDevice, st));
      const bool acc = gi > 0 || (flags & GT_FLAG_ACCUMULATE);
      SceneDev sd{};
      sd.shade = scenes[s]->b.shade;
      sd.sh = scenes[s]->b.sh;
      sd.params = scenes[s]->b.params;
      k_expand<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(G[s], evs, (uint32_t)mine.size(), sd, n, dev_out[s],
                                                             acc);
      ++ctx->launches;
      BWD_TRY(cudaGetLastError());
    }
    g0 = g1;
  }
  for (uint32_t s = 0; s < n_scenes; ++s) {
    const uint64_t n = scenes[s]->n;
    if (n == 0 || (flags & GT_FLAG_OUTPUT_DEVICE)) continue;
    BWD_TRY(cudaMemcpyAsync(outs[s], dev_out[s], n * GT_PARAMS_PER_PARTICLE * 4, cudaMemcpyDeviceToHost, st));
  }
  BWD_TRY(cudaEventRecord(ctx->int1, st));
  BWD_TRY(cudaMemcpyAsync(ctx->h_ctr, ctx->d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, st));
  BWD_TRY(cudaStreamSynchronize(st));
  cudaEventElapsedTime(&bwd_ms, ctx->int0, ctx->int1);
  sst = api_status_to_error(ctx, ctx->h_ctr->status);
  if (stats) {
    memset(stats, 0, sizeof *stats);
    api_fill_stats(*ctx->h_ctr, stats);
    stats->kernel_ms = bwd_ms;
    stats->total_ms = fwd_ms + bwd_ms;
  }
  if (opts) {
    opts->used_mode = cs.mode;
    opts->fwd_ms = fwd_ms;
    opts->bwd_ms = bwd_ms;
    opts->max_rounds = (uint32_t)std::min<uint64_t>(cs.last_records, 0xFFFFFFFFull);
  }
  cleanup();
  return sst;
#undef BWD_TRY
}

gt_status check_bwd_view(gt_context* ctx, const gt_scene* s, const gt_uniforms* u, uint32_t w, uint32_t h,
                         const float* dL, uint32_t flags) {
  if (!s || s->ctx != ctx) return api_fail(ctx, GT_ERR_INVALID_ARG, "scene is NULL or from another context");
  gt_status st = api_check_uniforms(ctx, u);
  if (st != GT_OK) return st;
  if (u->debug_mode != 0) return api_fail(ctx, GT_ERR_INVALID_ARG, "backward needs debug_mode 0");
  if (!dL) return api_fail(ctx, GT_ERR_INVALID_ARG, "dL_drgba is NULL");
  if ((flags & GT_FLAG_INPUT_DEVICE) && ((uintptr_t)dL % 16) != 0)  // read as float4
    return api_fail(ctx, GT_ERR_INVALID_ARG, "device dL_drgba must be 16-byte aligned");
  if (w == 0 || h == 0 || (uint64_t)w * h > (1ull << 31) || view_slots(w, h) > kMaxSlots)
    return api_fail(ctx, GT_ERR_INVALID_ARG, "bad image size");
  return GT_OK;
}

}  // namespace

extern "C" gt_status gt_backward(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u, uint32_t w, uint32_t h,
                                 const float* dL_drgba, float* dL_dparams, uint32_t flags, gt_bwd_opts* opts,
                                 gt_render_stats* stats) {
  if (!ctx) return api_fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  gt_status st = check_bwd_view(ctx, scene, u, w, h, dL_drgba, flags);
  if (st != GT_OK) return st;
  if (!dL_dparams && scene->n > 0) return api_fail(ctx, GT_ERR_INVALID_ARG, "dL_dparams is NULL");
  if (flags & GT_FLAG_ASYNC) return api_fail(ctx, GT_ERR_INVALID_ARG, "gt_backward is synchronous");
  BwdView v{scene, *u, w, h, dL_drgba};
  return backward_impl(ctx, &v, 1, &scene, &dL_dparams, 1, flags, opts, stats);
}

extern "C" gt_status gt_backward_batch(gt_context* ctx, const gt_batch_item* items, uint32_t count,
                                       const gt_scene* const* scenes, float* const* dL_dparams, uint32_t n_scenes,
                                       uint32_t flags, gt_bwd_opts* opts, gt_render_stats* stats) {
  if (!ctx) return api_fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (count == 0) return GT_OK;
  if (!items || !scenes || !dL_dparams || n_scenes == 0) return api_fail(ctx, GT_ERR_INVALID_ARG, "NULL argument");
  if (flags & GT_FLAG_ASYNC) return api_fail(ctx, GT_ERR_INVALID_ARG, "gt_backward_batch is synchronous");
  std::vector<BwdView> v(count);
  uint64_t slots_all = 0;
  for (uint32_t i = 0; i < count; ++i) {
    gt_status st =
        check_bwd_view(ctx, items[i].scene, &items[i].u, items[i].w, items[i].h, items[i].dL_drgba, flags);
    if (st != GT_OK) return st;
    slots_all += view_slots(items[i].w, items[i].h);
    if (slots_all > kMaxSlots) return api_fail(ctx, GT_ERR_INVALID_ARG, "batch larger than 2^31 work slots");
    uint32_t s = 0;
    while (s < n_scenes && scenes[s] != items[i].scene) ++s;
    if (s == n_scenes) return api_fail(ctx, GT_ERR_INVALID_ARG, "a batch item's scene is not in `scenes`");
    v[i] = BwdView{items[i].scene, items[i].u, items[i].w, items[i].h, items[i].dL_drgba};
  }
  for (uint32_t s = 0; s < n_scenes; ++s)
    if (!scenes[s] || scenes[s]->ctx != ctx || (!dL_dparams[s] && scenes[s]->n > 0))
      return api_fail(ctx, GT_ERR_INVALID_ARG, "bad scene or gradient output");
  return backward_impl(ctx, v.data(), count, scenes, dL_dparams, n_scenes, flags, opts, stats);
}

extern "C" gt_status gt_l2_loss(gt_context* ctx, const float* rgba, const float* target, uint64_t n_pixels,
                                float* dL_drgba, double* loss) {
  if (!ctx) return api_fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (n_pixels == 0) {
    if (loss) *loss = 0.0;
    return GT_OK;
  }
  if (!rgba || !target || !dL_drgba) return api_fail(ctx, GT_ERR_INVALID_ARG, "NULL buffer");
  if (((uintptr_t)rgba | (uintptr_t)target | (uintptr_t)dL_drgba) % 16)
    return api_fail(ctx, GT_ERR_INVALID_ARG, "buffers must be 16-byte aligned");
  CK_TRY(cudaSetDevice(ctx->device));
  const unsigned blocks = (unsigned)((n_pixels + 255) / 256);
  double* partial = nullptr;
  CK_TRY(cudaMallocAsync((void**)&partial, blocks * sizeof(double), ctx->stream));
  k_l2_loss<<<blocks, 256, 0, ctx->stream>>>(reinterpret_cast<const float4*>(rgba),
                                             reinterpret_cast<const float4*>(target), n_pixels,
                                             reinterpret_cast<float4*>(dL_drgba), partial);
  ++ctx->launches;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && loss) {
    std::vector<double> h(blocks);
    e = cudaMemcpyAsync(h.data(), partial, blocks * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    double sum = 0.0;
    for (double v : h) sum += v;
    *loss = sum;
  }
  cudaFreeAsync(partial, ctx->stream);
  if (e != cudaSuccess) return api_fail(ctx, GT_ERR_CUDA, cudaGetErrorString(e));
  return GT_OK;
}
