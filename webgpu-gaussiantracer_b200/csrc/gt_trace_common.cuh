// gt_trace_common.cuh — pieces shared by the trace kernels: per-ray
// statistics, the box-test ray, the exact ray/proxy test and work helpers.
#pragma once

#include <math_constants.h>

#include "gt_device.cuh"
#include "gt_internal.cuh"

namespace gt {

constexpr int kTileW = 8, kTileH = 4;
constexpr uint32_t kTileBlock = 16;  // tiles per side of a tile block

// Pixel of position s (0..31) in tile lt of a view.  Tiles go in blocks of
// 16 x 16 (128 x 64 pixels), blocks row-major, tiles in Morton order inside a
// block, so that the tiles in flight at any time cover a compact patch of
// the image (1 % faster than row-major tiles on the 1M-Gaussian view).  The
// view's tile grid is padded to whole blocks; pixels past the image edge are
// skipped.
__device__ __forceinline__ void tile_pixel(uint32_t tiles_x, uint32_t lt, uint32_t s, uint32_t& px, uint32_t& py) {
  const uint32_t blk = lt >> 8, in = lt & 255u;
  const uint32_t bpr = tiles_x / kTileBlock;  // blocks per row
  const uint32_t bx = blk % bpr, by = blk / bpr;
  uint32_t mx = in & 0x55u, my = (in >> 1) & 0x55u;  // de-interleave the 8-bit Morton code
  mx = (mx | (mx >> 1)) & 0x33u;
  mx = (mx | (mx >> 2)) & 0x0Fu;
  my = (my | (my >> 1)) & 0x33u;
  my = (my | (my >> 2)) & 0x0Fu;
  px = (bx * kTileBlock + mx) * kTileW + (s % kTileW);
  py = (by * kTileBlock + my) * kTileH + (s / kTileW);
}

// Work counters of one warp, kept in its shared scratch (not in registers)
// and updated by lane 0 with warp totals.
struct RayStats {
  unsigned long long rounds, entries, contributing, proxy_tests, node_visits, anyhits;
};

// Box-test state of a ray: inverse direction, origin times inverse direction
// and, per axis, a padding of the slab planes that covers the rounding of
// the object-space triangle test (hit points lie within ~1e-6 relative of
// |origin| + scene size of the true surface).
struct BoxRay {
  float ix, iy, iz, ox, oy, oz, px, py, pz;
};

__device__ __forceinline__ float safe_inv(float d) {
  float a = fabsf(d) < 1e-30f ? copysignf(1e-30f, d) : d;
  return __frcp_rn(a);
}

__device__ __forceinline__ BoxRay make_boxray(V3 o, V3 d, float scene_mag) {
  BoxRay b;
  b.ix = safe_inv(d.x);
  b.iy = safe_inv(d.y);
  b.iz = safe_inv(d.z);
  b.ox = o.x * b.ix;
  b.oy = o.y * b.iy;
  b.oz = o.z * b.iz;
  float m = fmaxf(fmaxf(fabsf(o.x), fabsf(o.y)), fabsf(o.z));
  float pad = 4e-6f * (m + scene_mag) + 1e-7f;
  b.px = pad * fabsf(b.ix);
  b.py = pad * fabsf(b.iy);
  b.pz = pad * fabsf(b.iz);
  return b;
}

// Ray/proxy test.  Calls on_hit(t, face) for every face hit by the reference
// triangle test with t in (tlo, thi) that is front-facing (CULL) or any
// (!CULL).  Four exact filters run before that test; each skips only work
// whose outcome is already known:
//   * bounding sphere: every triangle lies inside the circumsphere, and the
//     triangle test cannot report a point farther than its rounding error
//     (covered by the 1e-3 + 1e-5 |o_obj| margin) from its triangle;
//   * facing: dot(n, d_obj) and the reference's world-space facing product
//     both approximate n^T W2O d within tau = 1e-5 * nmax * sum(|W2O||d|), so
//     a face whose dot(n, d_obj) exceeds tau is back-facing.  Faces come in
//     antipodal pairs with n_b == -n_a bit for bit, so dot(n_b, d) ==
//     -dot(n_a, d) exactly and one dot product serves both;
//   * t range: the triangle test's t times dn lies within
//     E = 10 u nmax (|p0|_1 + |o|_1) of num = n.p0 - n.o (u = 2^-24), so a
//     face with num >= tlo*dn + M or num <= thi*dn - M (dn < 0) has its t
//     outside (tlo, thi); M = 3e-5 nmax (|o|_1 + 2) + 1e-6 (|tlo|+|thi|)|dn|
//     is ~50x that error;
//   * candidate faces (CULL): of the front faces, only those whose plane
//     crossing lies within the triangle test's rounding reach of the latest
//     crossing can pass it (the proxy is convex; see the bound below), so
//     the triangle test runs on about 1.6 faces a proxy instead of 6.7.
// The bounding-sphere filter of proxy_test on its own: false only when the
// ray certainly misses proxy j.
__device__ __forceinline__ bool proxy_sphere(const FaceTable& F, const float4* w2o, uint32_t j, V3 o, V3 d) {
  Affine W = load_affine(w2o + 3 * (size_t)j);
  V3 oo = xpoint(W, o), od = xdir(W, d);
  float l1o = fabsf(oo.x) + fabsf(oo.y) + fabsf(oo.z);
  float dd = __fmaf_rn(od.x, od.x, __fmaf_rn(od.y, od.y, od.z * od.z));
  float ox = __fmaf_rn(oo.x, od.x, __fmaf_rn(oo.y, od.y, oo.z * od.z));
  float tc = -__fdividef(ox, dd);
  float cx = __fmaf_rn(tc, od.x, oo.x), cy = __fmaf_rn(tc, od.y, oo.y), cz = __fmaf_rn(tc, od.z, oo.z);
  float r2 = __fmaf_rn(cx, cx, __fmaf_rn(cy, cy, cz * cz));
  float rp = __fmaf_rn(1e-5f, l1o, F.r_circ + 1e-3f);
  return (r2 <= rp * rp) || !(dd == dd && r2 == r2);
}

template <bool CULL, class OnHit, bool SPHERE = true>
__device__ __forceinline__ void proxy_test(const FaceTable& F, const float4* w2o, uint32_t j, V3 o, V3 d, float tlo,
                                           float thi, OnHit&& on_hit) {
  Affine W = load_affine(w2o + 3 * (size_t)j);
  V3 oo = xpoint(W, o), od = xdir(W, d);
  float l1o = fabsf(oo.x) + fabsf(oo.y) + fabsf(oo.z);
  if (SPHERE) {
    float dd = __fmaf_rn(od.x, od.x, __fmaf_rn(od.y, od.y, od.z * od.z));
    float ox = __fmaf_rn(oo.x, od.x, __fmaf_rn(oo.y, od.y, oo.z * od.z));
    float tc = -__fdividef(ox, dd);
    float cx = __fmaf_rn(tc, od.x, oo.x), cy = __fmaf_rn(tc, od.y, oo.y), cz = __fmaf_rn(tc, od.z, oo.z);
    float r2 = __fmaf_rn(cx, cx, __fmaf_rn(cy, cy, cz * cz));
    float rp = __fmaf_rn(1e-5f, l1o, F.r_circ + 1e-3f);
    if (!(r2 <= rp * rp)) {
      if (dd == dd && r2 == r2) return;  // NaN falls through to the exact test
    }
  }
  if (!CULL) {
#pragma unroll 1
    for (int f = 0; f < 20; ++f) {
      float dn = vdot(mk(F.n[f][0], F.n[f][1], F.n[f][2]), od);
      float t;
      if (tri_test(F, f, oo, tlo, od, thi, dn, t)) on_hit(t, f);
    }
    return;
  }
  const float* m = W.m;
  float s = fabsf(d.x) * (fabsf(m[0]) + fabsf(m[1]) + fabsf(m[2])) +
            fabsf(d.y) * (fabsf(m[3]) + fabsf(m[4]) + fabsf(m[5])) +
            fabsf(d.z) * (fabsf(m[6]) + fabsf(m[7]) + fabsf(m[8]));
  const float tau = 1e-5f * F.nmax * s;
  const float mbase = 3e-5f * F.nmax * (l1o + 2.0f);
  const float trange = 1e-6f * (fabsf(tlo) + fminf(fabsf(thi), 1e30f));
  // Candidate faces.  For front faces e, f (dn < -tau) with plane crossings
  // t_e >= t_f, the ray at t_f lies outside plane e by (t_e - t_f)|dn_e|/|n|
  // while triangle f lies inside it (the proxy is convex), so the crossing
  // X_f is at least that far from triangle f.  The reference's triangle test
  // accepts points only within its rounding of the triangle, about
  // 10 u |od| |p0 - oo| / |dn_f| in barycentric units (u = 2^-24).  Hence a
  // face can pass only if G = num_e dn_f - num_f dn_e = (t_e - t_f) dn_e dn_f
  // stays below a few tens of u |od|_1 (|oo|_1 + 2); faces above 128 u times
  // that are skipped (a CPU check of 4e7 adversarial rays, edges, vertices
  // and grazing faces, found the first misses below 8).  One pass keeps the
  // face with the largest crossing so far and every face within the bound of
  // the face that was largest when it was seen, a superset of the faces the
  // final largest allows; grazing pairs keep both faces.
  const float gbound = 7.62939453125e-6f * (fabsf(od.x) + fabsf(od.y) + fabsf(od.z)) * (l1o + 2.0f);
  uint32_t cand = 0;
  int best = -1;
  float bnum = 0.0f, bdn = 0.0f;
#pragma unroll
  for (int pair = 0; pair < 10; ++pair) {
    const int fa = F.pa[pair];
    const V3 na = mk(F.pn[pair][0], F.pn[pair][1], F.pn[pair][2]);
    const float dna = vdot(na, od);
    if (fabsf(dna) > tau) {
      // exactly one face of the pair can face the ray
      // the pair's values sit at fixed offsets of the table (the loop is
      // unrolled): no indexed loads, and the pairs' independent products
      // can overlap
      const int fb = F.pb[pair];
      const float ca = F.pca[pair], cb = F.pcb[pair];
      const int f = dna < 0.0f ? fa : fb;
      const float dn = dna < 0.0f ? dna : -dna;
      const float no = __fmaf_rn(na.x, oo.x, __fmaf_rn(na.y, oo.y, na.z * oo.z));
      const float num = (dna < 0.0f ? ca : cb) - (dna < 0.0f ? no : -no);
      if (best < 0) {
        best = f;
        bnum = num;
        bdn = dn;
        cand |= 1u << f;
      } else {
        const float G = bnum * dn - num * bdn;
        if (G < 0.0f) {  // f crosses its plane later: the new largest
          if (-G > gbound) cand &= ~(1u << best);
          best = f;
          bnum = num;
          bdn = dn;
          cand |= 1u << f;
        } else if (G <= gbound) {
          cand |= 1u << f;
        }
      }
    } else {
      // grazing pair: both faces go to the exact test
      cand |= (1u << fa) | (1u << F.pb[pair]);
    }
  }
  // the exact tests of the candidates: t-range prefilter (faces whose facing
  // is certain), then the reference's triangle test and facing rule.  The
  // candidates of non-grazing pairs have dn < -tau: the reference's facing
  // product (within 12 u nmax s of dn, tau = 1e-5 nmax s) is then negative,
  // so only the grazing pairs' faces need it computed.
#pragma unroll 1
  while (cand) {
    const int f = __ffs(cand) - 1;
    cand &= cand - 1;
    const V3 nf = mk(F.n[f][0], F.n[f][1], F.n[f][2]);
    const float dn = vdot(nf, od);
    const bool sure = fabsf(dn) > tau;
    if (sure) {
      // the t-range test: t times dn lies within E = 10 u nmax (|p0|_1 +
      // |o|_1) of num = n.p0 - n.o, so a face with num >= tlo*dn + M or
      // num <= thi*dn - M (dn < 0) has its t outside (tlo, thi)
      const float no = __fmaf_rn(nf.x, oo.x, __fmaf_rn(nf.y, oo.y, nf.z * oo.z));
      const float num = F.c[f] - no;
      const float mg = __fmaf_rn(trange, fabsf(dn), mbase);
      if (num >= __fmaf_rn(tlo, dn, mg) || num <= __fmaf_rn(thi, dn, -mg)) continue;
    }
    float t;
    if (tri_test(F, f, oo, tlo, od, thi, dn, t) &&
        (sure ? dn < 0.0f : front_facing(F, f, load_affine(w2o + 3 * (size_t)j), d)))
      on_hit(t, f);
  }
}

// next float above x: the far bound of the triangle test that still admits
// a tie with the k-th hit
__device__ __forceinline__ float next_up(float x) { return nextafterf(x, CUDART_INF_F); }

// Adds a warp's counters to the launch totals.  `rays` is counted by lane 0;
// `st` is the warp's shared counter block.
__device__ __forceinline__ void flush_stats(DevCounters* ctr, const RayStats& st, uint32_t rays, uint32_t status) {
  uint32_t s = __reduce_or_sync(0xFFFFFFFFu, status);
  __syncwarp();
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&ctr->rays, (unsigned long long)rays);
    atomicAdd(&ctr->rounds, st.rounds);
    atomicAdd(&ctr->entries, st.entries);
    atomicAdd(&ctr->contributing, st.contributing);
    atomicAdd(&ctr->proxy_tests, st.proxy_tests);
    atomicAdd(&ctr->node_visits, st.node_visits);
    atomicAdd(&ctr->anyhits, st.anyhits);
    if (s) atomicOr(&ctr->status, s);
  }
}

__device__ __forceinline__ uint32_t find_view(const ViewDev* views, uint32_t n_views, uint32_t tile) {
  uint32_t lo = 0, hi = n_views - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (views[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}

}  // namespace gt
