// gt_packet.cu — forward tracer, one warp per 8x4 pixel tile (a packet of 32
// primary rays, one per lane), over the 8-wide BVH.
//
// Same output as k_trace8 (gt_trace.cu) bit for bit: the same per-round hit
// sets, the same compositing arithmetic in the same order.  What differs is
// how the work is shared out:
//   * traversal: the warp walks the hierarchy once for all its rays.  A node
//     is popped when its entry distance (a lower bound over the packet's
//     rays) is within the largest far bound of the packet; eight lanes test
//     the node's children against the whole packet at once (interval slab
//     test over the rays' common origin and range of directions, a superset
//     of the children any ray hits); inner children that pass are pushed
//     near-first, and each leaf child that passes gets the exact per-ray box
//     test, whose ballot is the leaf's ray mask.  Primary rays of one
//     tile are so coherent that the packet visits only ~1.13x the nodes of
//     one of its rays, so a node visit serves ~28 rays.  The node's 256 bytes
//     come in one coalesced load into shared memory, issued for the top of
//     the stack as soon as it is known so that it overlaps the leaf work;
//   * leaves: a leaf hit by ray r becomes a (proxy, ray) pair; pairs go 32 at
//     a time through the bounding-sphere filter and those that pass 28 at a
//     time through the exact face tests, one pair per lane.  Pairs are made
//     from a visit's hit leaves only while fewer than 32 wait, which keeps
//     the queue (and the shared memory of a warp) small: warps per SM are
//     bounded by shared memory, and more of them hide more latency;
//   * k-buffer: each ray keeps the kbuf smallest (t, particle) hits in a
//     4-ary max-heap of its own (a column of a shared-memory array of 64-bit keys
//     that order like (t, particle)); its root is the ray's far bound.  The
//     hits of one face-test batch are inserted by one lane per target ray
//     (__match_any_sync groups the lanes whose pairs test that ray);
//   * rounds and compositing: after the traversal each lane sorts its heap
//     (heapsort) and runs the rounds of its own ray serially, in entry
//     order.  Rays whose buffer ran out traverse again (with the packet's
//     other such rays) from their t_curr;
//   * handoff: a tile takes as long as its rays with the most hits, and a
//     packet traversal for a few rays costs about as much as one for all 32.
//     After handoff_after traversals (after the current one once every
//     tile is taken) a packet writes its rays that still need hits (their
//     compositing state between two rounds) to a buffer, and the
//     warp-per-ray kernel, launched next, finishes them; the arithmetic of
//     every round is the same in both kernels;
//   * checkpoint (for gt_backward): each round's record (t_curr, T, the
//     ray's previous record, the entries) as k_trace8 writes it.
#include <math_constants.h>

#include "gt_device.cuh"
#include "gt_internal.cuh"
#include "gt_trace_common.cuh"
#include "gt_warp.cuh"

namespace gt {

constexpr int kPairCap = 64;  // (proxy, ray) pairs: < 32 queued + the rays of one leaf
// pairs that passed the sphere filter go to the face tests in batches once
// kPacketSurvivors wait (28: 0.3 % faster than 24, 20 slower)
constexpr int kPacketSurvivors = 28;
constexpr int kSurvCap = 64;  // pairs that passed the sphere filter (< kPacketSurvivors + 32)

template <int KB>
struct PacketScratch {
  unsigned long long hk[KB][32];  // 4-ary heap of ray r in column r: hit keys, max at row 0
  uint2 stk[kWarpStack];  // node stack: (node, bits of its entry distance)
  uint32_t lj[8];  // leaf children of the visited node that some ray hit,
  uint32_t lm[8];  // with the mask of those rays
  uint32_t pj[kPairCap];
  uint8_t pr[kPairCap];
  uint32_t svj[kSurvCap];
  uint8_t svr[kSurvCap];
  float hq[kMaxHitsPerProxy][32];  // hits of each lane's pair, column per lane
  uint32_t hp[32];                 // the particle of each lane's pair
  uint8_t hc[32];                  // and its hit count
  float dx[32], dy[32], dz[32];    // ray directions
  float tlo[32], thi[32];          // ray intervals; thi = far bound
  uint8_t hn[32];                  // heap sizes
  float4 nbuf[16];                 // the node being visited
  RayStats stats;
};
// 12.7 KB for 32-entry heaps (16 one-warp blocks an SM: each of the SM's four
// schedulers holds 16K registers, four warps of up to 128 registers a thread)

// float -> uint map that preserves order (for warp min/max reductions)
__device__ __forceinline__ uint32_t ord_f(float x) {
  const uint32_t u = __float_as_uint(x);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unord_f(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Key of hit (t, p): ordered like (t, p) in the k-buffer (t first, then the
// particle index).  -0 is folded into +0 so that equal t compare equal.
__device__ __forceinline__ unsigned long long hit_key(float t, uint32_t p) {
  return ((unsigned long long)ord_f(t + 0.0f) << 32) | p;
}
__device__ __forceinline__ float key_t(unsigned long long k) { return unord_f((uint32_t)(k >> 32)); }
__device__ __forceinline__ uint32_t key_p(unsigned long long k) { return (uint32_t)k; }

// The k-buffer of ray r is a 4-ary max-heap in column r (children of row i:
// rows 4i+1 .. 4i+4): 32 entries are 3 levels deep instead of 5, and the
// four children of a row are loaded together, so a sift waits on 3 rounds
// of shared-memory latency instead of 5.

// Sift key x down from row i of heap column r holding n entries; returns
// the key that ends in row i (x, or the largest child that moved up).
template <int KB>
__device__ __forceinline__ unsigned long long heap_sift(PacketScratch<KB>& W, uint32_t r, uint32_t i, uint32_t n,
                                                        unsigned long long x) {
  const uint32_t i0 = i;
  unsigned long long top = x;
  while (true) {
    const uint32_t c = 4 * i + 1;
    if (c >= n) break;
    // the last child is clamped to the last entry (a repeated child changes
    // nothing: ties keep the first)
    const uint32_t c1 = min(c + 1, n - 1), c2 = min(c + 2, n - 1), c3 = min(c + 3, n - 1);
    const unsigned long long k0 = W.hk[c][r], k1 = W.hk[c1][r], k2 = W.hk[c2][r], k3 = W.hk[c3][r];
    const bool s01 = k0 < k1, s23 = k2 < k3;
    const unsigned long long m01 = s01 ? k1 : k0, m23 = s23 ? k3 : k2;
    const uint32_t i01 = s01 ? c1 : c, i23 = s23 ? c3 : c2;
    const bool s = m01 < m23;
    const unsigned long long ck = s ? m23 : m01;
    if (!(x < ck)) break;
    W.hk[i][r] = ck;
    if (i == i0) top = ck;
    i = s ? i23 : i01;
  }
  W.hk[i][r] = x;
  return top;
}

// Offers the hits of the lanes in `peers` (all of them hits of ray r, hc[q]
// keys of particle hp[q] in column q of hq) to the k-buffer of ray r
// (capacity cap), lane by lane and each lane's last hit first: a hit is kept
// when the buffer is not full or it is below the buffer's largest entry.
// The heap size and root stay in registers over the run; the ray's far bound
// (the root of a full buffer) is written once at the end.
template <int KB>
__device__ __forceinline__ void heap_offer_run(PacketScratch<KB>& W, uint32_t r, uint32_t cap, uint32_t peers) {
  uint32_t n = W.hn[r];
  unsigned long long root = n == cap ? W.hk[0][r] : 0ull;
  while (peers) {
    const int q = __ffs(peers) - 1;
    peers &= peers - 1;
    const uint32_t pq = W.hp[q];
    for (int h = (int)W.hc[q] - 1; h >= 0; --h) {
      const unsigned long long x = hit_key(W.hq[h][q], pq);
      if (n < cap) {
        uint32_t i = n;
        while (i > 0) {
          const uint32_t par = (i - 1) >> 2;
          const unsigned long long pk = W.hk[par][r];
          if (!(pk < x)) break;
          W.hk[i][r] = pk;
          i = par;
        }
        W.hk[i][r] = x;
        if (++n == cap) root = W.hk[0][r];
      } else if (x < root) {
        root = heap_sift(W, r, 0, n, x);
      }
    }
  }
  W.hn[r] = (uint8_t)n;
  if (n == cap) W.thi[r] = key_t(root);
}

// Sorts heap column r (n entries) ascending.
template <int KB>
__device__ __forceinline__ void heap_sort(PacketScratch<KB>& W, uint32_t r, uint32_t n) {
  for (uint32_t end = n; end > 1; --end) {
    const unsigned long long x = W.hk[end - 1][r];
    W.hk[end - 1][r] = W.hk[0][r];
    heap_sift(W, r, 0, end - 1, x);
  }
}

__device__ __forceinline__ float warp_max_f(float x) { return unord_f(__reduce_max_sync(kFull, ord_f(x))); }

// Box test of the whole packet.  All rays of a tile start at the camera, so
// over the live rays the slab distances (x - o) i of an axis are linear in
// the inverse direction i and take their extremes at the smallest and largest
// i of the packet (when i has one sign; an axis whose directions change sign
// culls nothing).  The interval [near, far] so found contains every live
// ray's own padded slab interval: the padding pp is 1.25 times the largest
// per-ray padding, whose extra quarter (>= 1e-6 (|o| + scene size) |i|) is
// far above the few-ulp difference between (x - o) i rounded here and the
// per-ray x i - o i.  So the packet test passes whenever some ray's box test
// passes; it costs one lane per child instead of every lane per child.
struct PacketBox {
  float ox, oy, oz;
  float ax0, ax1, ay0, ay1, az0, az1;  // smallest, largest inverse direction per axis
  float ppx, ppy, ppz;                 // slab padding per axis
  float tlo;                           // smallest t_curr of the live rays
  bool straddle;                       // some axis's directions change sign
};

__device__ __forceinline__ float warp_min_f(float x) { return unord_f(__reduce_min_sync(kFull, ord_f(x))); }

__device__ __forceinline__ PacketBox make_packet_box(V3 o, const BoxRay& br, bool live, float tlo, float scene_mag) {
  PacketBox P;
  P.ox = o.x;
  P.oy = o.y;
  P.oz = o.z;
  const float inf = CUDART_INF_F;
  P.ax0 = warp_min_f(live ? br.ix : inf);
  P.ax1 = warp_max_f(live ? br.ix : -inf);
  P.ay0 = warp_min_f(live ? br.iy : inf);
  P.ay1 = warp_max_f(live ? br.iy : -inf);
  P.az0 = warp_min_f(live ? br.iz : inf);
  P.az1 = warp_max_f(live ? br.iz : -inf);
  P.tlo = warp_min_f(live ? tlo : inf);
  // the per-ray padding (make_boxray) with the same origin for every ray
  const float m = fmaxf(fmaxf(fabsf(o.x), fabsf(o.y)), fabsf(o.z));
  const float pad = 1.25f * (4e-6f * (m + scene_mag) + 1e-7f);
  P.ppx = pad * fmaxf(fabsf(P.ax0), fabsf(P.ax1));
  P.ppy = pad * fmaxf(fabsf(P.ay0), fabsf(P.ay1));
  P.ppz = pad * fmaxf(fabsf(P.az0), fabsf(P.az1));
  P.straddle = (P.ax0 < 0.f && P.ax1 > 0.f) || (P.ay0 < 0.f && P.ay1 > 0.f) || (P.az0 < 0.f && P.az1 > 0.f);
  return P;
}

__device__ __forceinline__ void packet_slab(float lo, float hi, float o, float i0, float i1, float pp, float& n,
                                            float& f) {
  const float dlo = lo - o, dhi = hi - o;
  if (i0 > 0.f) {
    n = fminf(dlo * i0, dlo * i1);
    f = fmaxf(dhi * i0, dhi * i1);
  } else if (i1 < 0.f) {
    n = fminf(dhi * i0, dhi * i1);
    f = fmaxf(dlo * i0, dlo * i1);
  } else {
    n = -CUDART_INF_F;
    f = CUDART_INF_F;
  }
  n = n - pp;
  f = f + pp;
}

// The per-ray padded box test of the tracers (child box a, b against ray br
// with interval [tlo, thi]); returns the entry distance through tn.
__device__ __forceinline__ bool ray_box(const float4 a, const float4 b, const BoxRay& br, float tlo, float thi,
                                        float& tn) {
  const float x0 = __fmaf_rn(a.x, br.ix, -br.ox), x1 = __fmaf_rn(a.w, br.ix, -br.ox);
  const float y0 = __fmaf_rn(a.y, br.iy, -br.oy), y1 = __fmaf_rn(b.x, br.iy, -br.oy);
  const float z0 = __fmaf_rn(a.z, br.iz, -br.oz), z1 = __fmaf_rn(b.y, br.iz, -br.oz);
  tn = fmaxf(fmaxf(fminf(x0, x1) - br.px, fminf(y0, y1) - br.py), fmaxf(fminf(z0, z1) - br.pz, tlo));
  const float tf =
      fminf(fminf(fmaxf(x0, x1) + br.px, fmaxf(y0, y1) + br.py), fminf(fmaxf(z0, z1) + br.pz, thi));
  return tn <= tf;
}

// One traversal of the packet: every live lane's ray collects the cap
// smallest front-face hits with t in (its t_curr, t_max) into its heap.
// Lanes that are not live take no part (far bound -inf).
template <int KB>
__device__ __forceinline__ void packet_traverse(const SceneDev& S, const FaceTable& F, PacketScratch<KB>& W, V3 o,
                                                const BoxRay& br, bool live, float tlo, float t_max, uint32_t cap,
                                                uint32_t& status, uint32_t lane) {
  const uint32_t lt_mask = (1u << lane) - 1u;
  float thi = live ? t_max : -CUDART_INF_F;
  W.tlo[lane] = tlo;
  W.thi[lane] = thi;
  W.hn[lane] = 0;
  if (S.n_kept == 0) return;
  float thi_max = warp_max_f(thi);
  const PacketBox P = make_packet_box(o, br, live, tlo, S.scene_mag);
  RayStats& st = W.stats;
  int sp = 1, nq = 0, ns = 0;
  if (lane == 0) {
    W.stk[0] = make_uint2(0u, __float_as_uint(-CUDART_INF_F));
  }
  __syncwarp();
  uint32_t iters = 0;
  const uint32_t max_iters = min(4u * S.n_kept + 64u, F.lim_steps);
  // lanes 0..15 prefetch the 16 float4 of the node the next pop most likely
  // takes (the top of the stack), so that its load overlaps the leaf work
  uint32_t pf_node = 0;
  float4 pf = make_float4(0.f, 0.f, 0.f, 0.f);
  if (lane < 16) pf = __ldg(S.nodes8 + lane);
  while (true) {
    if (++iters > max_iters) {
      status |= kStatusVisitCap;
      return;
    }
    // pop the top node whose entry distance is within some ray's far bound
    uint32_t node = kInvalid;
    while (sp > 0) {
      --sp;
      const uint2 e = W.stk[sp];
      if (__uint_as_float(e.y) <= thi_max) {
        node = e.x;
        break;
      }
    }
    int nl = 0;  // leaf children of this visit waiting to become pairs
    if (node != kInvalid) {
      if (lane < 16) {
        if (node != pf_node) pf = __ldg(S.nodes8 + 16 * (size_t)node + lane);
        W.nbuf[lane] = pf;
      }
      __syncwarp();
      // lanes 0..7: the packet test of one child each
      bool phit = false, pleaf = false;
      float ptn = CUDART_INF_F;
      uint32_t pref = kInvalid;
      if (P.straddle) {
        // a packet whose directions cross an axis plane gets no bound from
        // that axis (rays nearly parallel to it): every ray tests every
        // child, and a child's key is the smallest entry distance of the
        // rays that hit it
#pragma unroll 1
        for (int c = 0; c < 8; ++c) {
          const float4 a = W.nbuf[2 * c], b = W.nbuf[2 * c + 1];
          const uint32_t ref = __float_as_uint(b.z);
          float tn;
          const bool hit = ref != kInvalid && ray_box(a, b, br, tlo, thi, tn);
          const uint32_t m = __ballot_sync(kFull, hit);
          if (m == 0) continue;
          if (ref & kLeafBit) {
            if (lane == 0) {
              W.lj[nl] = ref & ~kLeafBit;
              W.lm[nl] = m;
            }
            ++nl;
          } else {
            const uint32_t key = __reduce_min_sync(kFull, hit ? ord_f(tn) : 0xFFFFFFFFu);
            if ((int)lane == c) {
              phit = true;
              ptn = unord_f(key);
              pref = ref;
            }
          }
        }
      } else if (lane < 8) {
        const float4 a = W.nbuf[2 * lane], b = W.nbuf[2 * lane + 1];
        pref = __float_as_uint(b.z);
        float nx, fx, ny, fy, nz, fz;
        packet_slab(a.x, a.w, P.ox, P.ax0, P.ax1, P.ppx, nx, fx);
        packet_slab(a.y, b.x, P.oy, P.ay0, P.ay1, P.ppy, ny, fy);
        packet_slab(a.z, b.y, P.oz, P.az0, P.az1, P.ppz, nz, fz);
        ptn = fmaxf(fmaxf(nx, ny), fmaxf(nz, P.tlo));
        const float ptf = fminf(fminf(fx, fy), fminf(fz, thi_max));
        phit = pref != kInvalid && ptn <= ptf;  // empty slots (packed at the end) never hit
        pleaf = (pref & kLeafBit) != 0;
      }
      // leaf children the packet may hit: each ray's own test gives its mask
      uint32_t lmask = __ballot_sync(kFull, phit && pleaf);
      while (lmask) {
        const int c = __ffs(lmask) - 1;
        lmask &= lmask - 1;
        const float4 a = W.nbuf[2 * c], b = W.nbuf[2 * c + 1];
        float tn;
        const bool hit = ray_box(a, b, br, tlo, thi, tn);
        const uint32_t m = __ballot_sync(kFull, hit);
        if (m) {
          if (lane == 0) {
            W.lj[nl] = __float_as_uint(b.z) & ~kLeafBit;
            W.lm[nl] = m;
          }
          ++nl;
        }
      }
      // inner children the packet may hit, keyed by the packet's entry distance
      const uint32_t imask = __ballot_sync(kFull, phit && !pleaf);
      const int ni = __popc(imask);
      uint32_t top = 0;  // the child that goes on top of the stack (nearest)
      if (ni > 0) {
        if (sp + ni > (int)F.lim_stack) {
          status |= kStatusStackOverflow;
          return;
        }
        if (ni == 1) {
          if ((imask >> lane) & 1u) W.stk[sp] = make_uint2(pref, __float_as_uint(ptn));
          top = __shfl_sync(kFull, pref, __ffs(imask) - 1);
        } else {
          // gathered into lanes 0..ni-1 through the free stack slots above
          // sp, sorted, and pushed farthest first
          float mykey = CUDART_INF_F;
          uint32_t myref = 0;
          if ((imask >> lane) & 1u) {
            const int q = sp + __popc(imask & lt_mask);
            W.stk[q] = make_uint2(pref, __float_as_uint(ptn));
          }
          __syncwarp();
          if ((int)lane < ni) {
            const uint2 e = W.stk[sp + (int)lane];
            mykey = __uint_as_float(e.y);
            myref = e.x;
          }
          __syncwarp();
          warp_sort_prefix(mykey, myref, lane, ni);
          if ((int)lane < ni) W.stk[sp + ni - 1 - (int)lane] = make_uint2(myref, __float_as_uint(mykey));
          top = __shfl_sync(kFull, myref, 0);
        }
        sp += ni;
      }
      if (lane == 0) st.node_visits += 1;
      __syncwarp();
      if (sp > 0) {
        pf_node = ni > 0 ? top : W.stk[sp - 1].x;
        if (lane < 16) pf = __ldg(S.nodes8 + 16 * (size_t)pf_node + lane);
      }
    }
    // leaf work: face tests once kPacketSurvivors pairs passed the sphere filter;
    // the visit's hit leaves become (proxy, ray) pairs while fewer than 32
    // pairs wait; the sphere filter once 32 pairs wait; everything when no
    // node is left
    int li = 0;
    while (true) {
      const bool drain = sp == 0 && li == nl;
      if (ns >= kPacketSurvivors || (drain && nq == 0 && ns > 0)) {
        const int nb = ns < 32 ? ns : 32;
        const bool have = (int)lane < nb;
        uint32_t j = 0, r = 0;
        if (have) {
          j = W.svj[ns - nb + (int)lane];
          r = W.svr[ns - nb + (int)lane];
        }
        ns -= nb;
        int nh = 0;
        if (have) {
          const V3 d = mk(W.dx[r], W.dy[r], W.dz[r]);
          const float tb = fminf(next_up(W.thi[r]), t_max);
          auto on_hit = [&](float t, int) {
            if (nh < kMaxHitsPerProxy) W.hq[nh][lane] = t;
            ++nh;
          };
          proxy_test<true, decltype(on_hit)&, false>(F, S.w2o, j, o, d, W.tlo[r], tb, on_hit);
          if (nh > kMaxHitsPerProxy) {
            status |= kStatusHitOverflow;
            nh = kMaxHitsPerProxy;
          }
        }
        const uint32_t found = __reduce_add_sync(kFull, (uint32_t)nh);
        if (lane == 0) st.anyhits += found;
        if (found) {
          // the lowest lane of the lanes whose pairs target one ray inserts
          // all their hits (lane by lane, each lane's last hit first)
          const uint32_t peers = __match_any_sync(kFull, nh ? r : 64u + lane);
          W.hp[lane] = nh ? __ldg(S.leaf_pidx + j) : 0u;
          W.hc[lane] = (uint8_t)nh;
          __syncwarp();
          if (nh && (int)lane == __ffs(peers) - 1) heap_offer_run(W, r, cap, peers);
          __syncwarp();
          thi = W.thi[lane];
          thi_max = warp_max_f(thi);
        }
        continue;
      }
      if (nq < 32 && li < nl) {
        const uint32_t m = W.lm[li];
        if ((m >> lane) & 1u) {
          const int q = nq + __popc(m & lt_mask);
          W.pj[q] = W.lj[li];
          W.pr[q] = (uint8_t)lane;
        }
        nq += __popc(m);
        ++li;
        __syncwarp();
        continue;
      }
      if (nq >= 32 || (drain && nq > 0)) {
        const int nb = nq < 32 ? nq : 32;
        uint32_t j = 0, r = 0;
        const bool have = (int)lane < nb;
        if (have) {
          j = W.pj[nq - nb + (int)lane];
          r = W.pr[nq - nb + (int)lane];
        }
        nq -= nb;
        if (lane == 0) st.proxy_tests += (unsigned)nb;
        const bool surv = have && proxy_sphere(F, S.w2o, j, o, mk(W.dx[r], W.dy[r], W.dz[r]));
        const uint32_t sm = __ballot_sync(kFull, surv);
        if (surv) {
          const int q = ns + __popc(sm & lt_mask);
          W.svj[q] = j;
          W.svr[q] = (uint8_t)r;
        }
        ns += __popc(sm);
        __syncwarp();
        continue;
      }
      break;
    }
    if (sp == 0 && nq == 0 && ns == 0) break;
  }
}

__device__ __forceinline__ bool ray_more(const RayUniforms& u, float T, float t_curr, uint32_t step) {
  return u.T_min < T && t_curr < u.t_max && u.early_stop != step;
}

// Persistent kernel: each warp takes one 8x4 tile at a time from a global
// counter (tiles of all views back to back) and traces its 32 rays.
// CKPT: write the round checkpoint the adjoint replays (gt_backward), with
// the layout and slot numbering of k_trace8's.
template <int KB, bool CKPT>
__global__ void __launch_bounds__(32) k_trace_packet(const ViewDev* __restrict__ views, uint32_t n_views,
                                                     uint32_t total_tiles, DevCounters* ctr,
                                                     const __grid_constant__ FaceTable F, const Handoff hand,
                                                     uint32_t hand_after, const Ckpt ck) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PacketScratch<KB>& W = *reinterpret_cast<PacketScratch<KB>*>(smem_raw);
  const uint32_t lane = threadIdx.x & 31;
  if (lane == 0) W.stats = RayStats{0, 0, 0, 0, 0, 0};
  __syncwarp();
  uint32_t status = 0, rays = 0;
  uint32_t n_rounds = 0, n_entries = 0, n_contrib = 0;
  while (true) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(&ctr->work, 1u);
    tile = __shfl_sync(kFull, tile, 0);
    if (tile >= total_tiles) break;
    const uint32_t vi = n_views == 1 ? 0u : find_view(views, n_views, tile);
    const ViewDev& V = views[vi];
    uint32_t px, py;
    tile_pixel(V.tiles_x, tile - V.tile_begin, lane, px, py);
    const bool valid = px < V.w && py < V.h;
    if (__ballot_sync(kFull, valid) == 0) continue;
    V3 o, d;
    ray_gen(V.u, V.w, V.h, valid ? px : 0u, valid ? py : 0u, o, d);
    const BoxRay br = make_boxray(o, d, V.s.scene_mag);
    W.dx[lane] = d.x;
    W.dy[lane] = d.y;
    W.dz[lane] = d.z;
    const float t_max = V.u.t_max;
    const uint32_t k = V.u.k;
    const uint32_t cap = V.pkbuf < (uint32_t)KB ? V.pkbuf : (uint32_t)KB;
    float L0 = 0.f, L1 = 0.f, L2 = 0.f, T = 1.f, t_curr = V.u.t_min;
    uint32_t step = 0;
    bool live = valid && ray_more(V.u, T, t_curr, step);
    bool handed = false;
    uint32_t n_trav = 0;
    uint32_t ck_head = kInvalid;
    uint32_t ck_fill = ck.kc;  // entries in the open record (checkpoint mode; kc: none open)
    while (__any_sync(kFull, live)) {
      // Once every tile is taken, the launch's end waits on the packets still
      // tracing: a packet then hands its rays over after its current
      // traversal, and the warp-per-ray kernel spreads them over all SMs
      // (1080p 39.5 -> 38.8 ms, 960x540 14.2 -> 12.5 ms).
      bool tiles_done = false;
      if (hand.rays && n_trav >= 1u && n_trav < hand_after) {
        uint32_t taken = 0;
        if (lane == 0) taken = *reinterpret_cast<volatile const uint32_t*>(&ctr->work);
        tiles_done = __shfl_sync(kFull, taken, 0) >= total_tiles;
      }
      if (hand.rays && (n_trav == hand_after || tiles_done)) {
        // hand the rays that still need hits to the warp-per-ray kernel
        const uint32_t hm = __ballot_sync(kFull, live);
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&ctr->handoff, (uint32_t)__popc(hm));
        base = __shfl_sync(kFull, base, 0);
        const uint32_t idx = base + (uint32_t)__popc(hm & ((1u << lane) - 1u));
        if (live && idx < hand.cap) {
          hand.rays[idx] = HandoffRay{32u * tile + lane, step, t_curr, T, L0, L1, L2, ck_head, ck_fill};
          live = false;
          handed = true;
        }
        if (!__any_sync(kFull, live)) break;  // (the buffer may be full: the rest go on here)
        n_trav = hand_after;  // no second hand-over of the rays that did not fit
      }
      ++n_trav;
      packet_traverse<KB>(V.s, F, W, o, br, live, t_curr, t_max, cap, status, lane);
      __syncwarp();
      if (__reduce_or_sync(kFull, status) & (kStatusStackOverflow | kStatusVisitCap | kStatusHitOverflow)) break;
      // the rounds each live ray's buffer serves, warp-synchronously (one
      // record allocation a round for the whole warp when checkpointing)
      uint32_t cnt = 0, head = 0;
      bool complete = false, rounds_on = live;
      if (live) {
        cnt = W.hn[lane];
        complete = cnt < cap;  // every hit beyond t_curr is in the buffer
        heap_sort(W, lane, cnt);
      }
      while (true) {
        bool act = false;
        uint32_t n = 0;
        float new_t = t_max;
        if (rounds_on) {
          if (!ray_more(V.u, T, t_curr, step)) {
            rounds_on = false;
          } else {
            while (head < cnt && !(key_t(W.hk[head][lane]) > t_curr)) ++head;
            const uint32_t avail = cnt - head;
            if (!complete && avail < k) {
              rounds_on = false;  // the next round reaches past the buffer
            } else {
              n = avail < k ? avail : k;
              new_t = n == k ? key_t(W.hk[head + k - 1][lane]) + 1e-4f : t_max;
              act = true;
            }
          }
        }
        const uint32_t am = __ballot_sync(kFull, act);
        if (am == 0) break;
        if (CKPT && ck.kc == 0) {
          // replay mode: one record a round
          uint32_t base = 0;
          if (lane == 0) base = atomicAdd(ck.pool_next, (uint32_t)__popc(am));
          base = __shfl_sync(kFull, base, 0);
          const uint32_t rec = base + (uint32_t)__popc(am & ((1u << lane) - 1u));
          if (act && rec < ck.pool_cap) {  // past the pool the host sizes it up and runs again
            uint32_t* r = ck.pool + (size_t)rec * (kCkptHeader + ck.kc);
            r[0] = __float_as_uint(t_curr);
            r[1] = __float_as_uint(T);
            r[2] = ck_head;
            r[3] = n;
            ck_head = rec;
          }
        }
        if (CKPT && ck.kc) {
          // checkpoint mode: the same accumulation with the rays' entries in
          // step, so that records open with one allocation for the warp
          const uint32_t nmax = __reduce_max_sync(kFull, act ? n : 0u);
          if (act) {
            ++step;
            ++n_rounds;
            n_entries += n;
          }
          for (uint32_t e = 0; e < nmax; ++e) {
            bool contrib = false;
            uint32_t ep = 0;
            float alpha = 0.f, x0 = 0.f, x1 = 0.f, x2 = 0.f;
            if (act && e < n) {
              ep = key_p(W.hk[head + e][lane]);
              const Shade sd = load_shade(V.s.shade, ep);
              alpha = response(sd, o, d) * sd.opacity;
              if (V.u.alpha_min < alpha) {
                contrib = true;
                if (V.rgb) {
                  const float4 q = __ldg(V.rgb + ep);
                  x0 = q.x;
                  x1 = q.y;
                  x2 = q.z;
                } else {
                  entry_colour(V.s.sh, ep, sd.mu, o, V.u.deg, x0, x1, x2);
                }
              }
            }
            const bool open = contrib && ck_fill >= ck.kc;
            const uint32_t om = __ballot_sync(kFull, open);
            if (om) {
              const int leader = __ffs(om) - 1;
              uint32_t base = 0;
              if ((int)lane == leader) base = atomicAdd(ck.pool_next, (uint32_t)__popc(om));
              base = __shfl_sync(kFull, base, leader);
              if (open) {
                const uint32_t rec = base + (uint32_t)__popc(om & ((1u << lane) - 1u));
                if (rec < ck.pool_cap) {  // past the pool the host sizes it up and runs again
                  uint32_t* r = ck.pool + (size_t)rec * (kCkptHeader + ck.kc);
                  r[0] = __float_as_uint(t_curr);
                  r[1] = __float_as_uint(T);
                  r[2] = ck_head;
                }
                ck_head = rec;
                ck_fill = 0;
              }
            }
            if (contrib) {
              if (ck_head < ck.pool_cap) {
                uint32_t* r = ck.pool + (size_t)ck_head * (kCkptHeader + ck.kc);
                r[kCkptHeader + ck_fill] = ep;
                r[3] = ck_fill + 1;
              }
              ++ck_fill;
              const float ta = T * alpha;
              L0 = L0 + ta * x0;
              L1 = L1 + ta * x1;
              L2 = L2 + ta * x2;
              T = T * (1.0f - alpha);
              ++n_contrib;
            }
          }
        } else if (act) {
          ++step;
          ++n_rounds;
          n_entries += n;
          // front-to-back accumulation in entry order (src/GS_shader.ts:250-269);
          // the next entry's shading record is loaded while this one is shaded
          // (not in the checkpointing kernel, whose registers it would spill)
          uint32_t nep = 0;
          Shade nsd{};
          if (!CKPT && n) {
            nep = key_p(W.hk[head][lane]);
            nsd = load_shade(V.s.shade, nep);
          }
          for (uint32_t e = 0; e < n; ++e) {
            uint32_t ep;
            Shade sd;
            if (CKPT) {
              ep = key_p(W.hk[head + e][lane]);
              sd = load_shade(V.s.shade, ep);
            } else {
              ep = nep;
              sd = nsd;
              if (e + 1 < n) {
                nep = key_p(W.hk[head + e + 1][lane]);
                nsd = load_shade(V.s.shade, nep);
              }
            }
            const float alpha = response(sd, o, d) * sd.opacity;
            if (V.u.alpha_min < alpha) {
              float x0, x1, x2;
              if (V.rgb) {
                const float4 q = __ldg(V.rgb + ep);
                x0 = q.x;
                x1 = q.y;
                x2 = q.z;
              } else {
                entry_colour(V.s.sh, ep, sd.mu, o, V.u.deg, x0, x1, x2);
              }
              const float ta = T * alpha;
              L0 = L0 + ta * x0;
              L1 = L1 + ta * x1;
              L2 = L2 + ta * x2;
              T = T * (1.0f - alpha);
              ++n_contrib;
            }
          }
        }
        if (act) {
          head += n;
          t_curr = new_t;
          if (step >= F.lim_rounds && ray_more(V.u, T, t_curr, step)) {
            status |= kStatusRoundCap;
            t_curr = t_max;
          }
        }
      }
      if (live) {
        live = ray_more(V.u, T, t_curr, step);
      }
      __syncwarp();
    }
    if (CKPT && valid && !handed) ck.head[32u * tile + lane] = ck_head < ck.pool_cap ? ck_head : kInvalid;
    if (valid && !handed) {
      const float4 r = make_float4(L0, L1, L2, 1.0f);
      float4* dst = V.out + (size_t)py * V.w + px;
      *dst = V.u.aa ? aa_blend(*dst, r, V.u.frames) : r;
      ++rays;
    }
  }
  const uint32_t s_rays = __reduce_add_sync(kFull, rays);
  const uint32_t s_rounds = __reduce_add_sync(kFull, n_rounds);
  const uint32_t s_entries = __reduce_add_sync(kFull, n_entries);
  const uint32_t s_contrib = __reduce_add_sync(kFull, n_contrib);
  if (lane == 0) {
    W.stats.rounds += s_rounds;
    W.stats.entries += s_entries;
    W.stats.contributing += s_contrib;
  }
  __syncwarp();
  flush_stats(ctr, W.stats, lane == 0 ? s_rays : 0u, status);
}

template <int KB, bool CKPT>
static Err launch_packet_kb(const ViewDev* d_views, uint32_t n_views, uint32_t total_tiles, DevCounters* counters,
                            const FaceTable& faces, int num_sms, cudaStream_t stream, uint64_t* launches,
                            const Handoff& hand, uint32_t hand_after, const Ckpt& ck) {
  const size_t smem = sizeof(PacketScratch<KB>);
  GT_CUDA_TRY(
      cudaFuncSetAttribute(k_trace_packet<KB, CKPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  GT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_packet<KB, CKPT>, 32, smem));
  uint32_t grid = (uint32_t)num_sms * (uint32_t)std::max(1, per_sm);
  if (grid > total_tiles) grid = std::max(1u, total_tiles);
  k_trace_packet<KB, CKPT><<<grid, 32, smem, stream>>>(d_views, n_views, total_tiles, counters, faces, hand,
                                                       hand_after, ck);
  ++*launches;
  GT_CUDA_TRY(cudaGetLastError());
  return Err{};
}

template <int KB>
static Err launch_packet_k(const ViewDev* d_views, uint32_t n_views, uint32_t total_tiles, DevCounters* counters,
                           const FaceTable& faces, int num_sms, cudaStream_t stream, uint64_t* launches,
                           const Handoff& hand, uint32_t hand_after, const Ckpt* ckpt) {
  if (ckpt)
    return launch_packet_kb<KB, true>(d_views, n_views, total_tiles, counters, faces, num_sms, stream, launches,
                                      hand, hand_after, *ckpt);
  return launch_packet_kb<KB, false>(d_views, n_views, total_tiles, counters, faces, num_sms, stream, launches,
                                     hand, hand_after, Ckpt{});
}

Err launch_trace_packet(const ViewDev* views, const ViewDev* d_views, uint32_t n_views, uint32_t total_tiles,
                        DevCounters* counters, const FaceTable& faces, int num_sms, cudaStream_t stream,
                        uint64_t* launches, const Handoff& hand, uint32_t hand_after, const Ckpt* ckpt) {
  uint32_t kmax = 1;
  for (uint32_t i = 0; i < n_views; ++i) kmax = std::max(kmax, views[i].pkbuf);
  if (kmax <= 24)
    return launch_packet_k<24>(d_views, n_views, total_tiles, counters, faces, num_sms, stream, launches, hand,
                               hand_after, ckpt);
  if (kmax <= 32)
    return launch_packet_k<32>(d_views, n_views, total_tiles, counters, faces, num_sms, stream, launches, hand,
                               hand_after, ckpt);
  if (kmax <= 48)
    return launch_packet_k<48>(d_views, n_views, total_tiles, counters, faces, num_sms, stream, launches, hand,
                               hand_after, ckpt);
  return launch_packet_k<64>(d_views, n_views, total_tiles, counters, faces, num_sms, stream, launches, hand,
                             hand_after, ckpt);
}

}  // namespace gt
