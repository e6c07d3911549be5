// gt_trace.cu — forward tracer: one persistent kernel for any number of views.
//
// Replaces the reference's per-pixel mega compute shader (raygen + tracePath
// rounds, src/GS_shader.ts:192-309; traversal, webrtx/src/glsl/trace.glsl:42-245;
// any-hit k-buffer, src/GS_shader.ts:323-367).
//
// Design:
//   * Persistent warps.  A warp takes a tile of 32 pixels (8x4) from a global
//     atomic counter, traces it, and takes the next; tiles of all views of a
//     batch share one counter, so uneven views balance themselves.
//   * One ray per lane.  Each round collects the k closest front-face proxy
//     hits beyond t_curr into a sorted register k-buffer (fully unrolled,
//     KMAX slots; the k active slots sit at the end, the others hold -inf and
//     never move), then composites them in order.
//   * Traversal of the binary LBVH with a per-lane stack in local memory,
//     nearer child first, popped entries skipped once the k-th hit is closer.
//     The far bound of every box test is the current k-th hit, so a round
//     touches only the front of the ray.
//   * A proxy is tested in object space: the ray goes through the leaf's
//     world-to-object map, a conservative bounding-sphere test drops most
//     candidates, and the reference's triangle test then runs on the faces
//     that can be front-facing.
//
// Round semantics (equal to the reference's): the set of a round is the k
// smallest front-face hits with t in (t_curr, t_max), ordered by (t, particle
// index); the reference reaches the same set through its commit rule, which
// never discards one of the k closest hits.  Ties in t are ordered by particle
// index (the reference orders them by arrival).
#include <math_constants.h>

#include "gt_device.cuh"
#include "gt_internal.cuh"

namespace gt {

constexpr int kTileW = 8, kTileH = 4;

struct RayStats {
  uint32_t rounds, entries, contributing, proxy_tests, node_visits, anyhits;
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

// Slab test of the two children of a node against [tlo, thi].
__device__ __forceinline__ void node_test(const float4& f0, const float4& f1, const float4& f2, const BoxRay& r,
                                          float tlo, float thi, float& n0, float& n1, bool& h0, bool& h1) {
  float ax = __fmaf_rn(f0.x, r.ix, -r.ox), bx = __fmaf_rn(f0.y, r.ix, -r.ox);
  float ay = __fmaf_rn(f0.z, r.iy, -r.oy), by = __fmaf_rn(f0.w, r.iy, -r.oy);
  float az = __fmaf_rn(f2.x, r.iz, -r.oz), bz = __fmaf_rn(f2.y, r.iz, -r.oz);
  n0 = fmaxf(fmaxf(fminf(ax, bx) - r.px, fminf(ay, by) - r.py), fmaxf(fminf(az, bz) - r.pz, tlo));
  float x0 = fminf(fminf(fmaxf(ax, bx) + r.px, fmaxf(ay, by) + r.py), fminf(fmaxf(az, bz) + r.pz, thi));
  h0 = n0 <= x0;
  float cx = __fmaf_rn(f1.x, r.ix, -r.ox), dx = __fmaf_rn(f1.y, r.ix, -r.ox);
  float cy = __fmaf_rn(f1.z, r.iy, -r.oy), dy = __fmaf_rn(f1.w, r.iy, -r.oy);
  float cz = __fmaf_rn(f2.z, r.iz, -r.oz), dz = __fmaf_rn(f2.w, r.iz, -r.oz);
  n1 = fmaxf(fmaxf(fminf(cx, dx) - r.px, fminf(cy, dy) - r.py), fmaxf(fminf(cz, dz) - r.pz, tlo));
  float x1 = fminf(fminf(fmaxf(cx, dx) + r.px, fmaxf(cy, dy) + r.py), fminf(fmaxf(cz, dz) + r.pz, thi));
  h1 = n1 <= x1;
}

// Ray/proxy test.  Calls on_hit(t, face) for every face hit by the reference
// triangle test with t in (tlo, thi) that is front-facing (CULL) or any
// (!CULL).  Three exact filters run before that test; each skips only work
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
//     is ~50x that error.
template <bool CULL, class OnHit>
__device__ __forceinline__ void proxy_test(const FaceTable& F, const float4* w2o, uint32_t j, V3 o, V3 d, float tlo,
                                           float thi, OnHit&& on_hit) {
  Affine W = load_affine(w2o + 3 * (size_t)j);
  V3 oo = xpoint(W, o), od = xdir(W, d);
  float l1o = fabsf(oo.x) + fabsf(oo.y) + fabsf(oo.z);
  {
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
  // rolled on purpose: one copy of the triangle test and of the caller's
  // k-buffer insertion keeps the kernel small enough for the instruction cache
#pragma unroll 1
  for (int pair = 0; pair < 10; ++pair) {
    const int fa = F.pa[pair];
    const V3 na = mk(F.n[fa][0], F.n[fa][1], F.n[fa][2]);
    const float dna = vdot(na, od);
    if (fabsf(dna) > tau) {
      // exactly one face of the pair can face the ray
      const int f = dna < 0.0f ? fa : F.pb[pair];
      const float dn = dna < 0.0f ? dna : -dna;
      const float no = __fmaf_rn(na.x, oo.x, __fmaf_rn(na.y, oo.y, na.z * oo.z));
      const float num = F.c[f] - (dna < 0.0f ? no : -no);
      const float mg = __fmaf_rn(trange, fabsf(dn), mbase);
      if (num >= __fmaf_rn(tlo, dn, mg) || num <= __fmaf_rn(thi, dn, -mg)) continue;
      float t;
      if (tri_test(F, f, oo, tlo, od, thi, dn, t) && front_facing(F, f, W, d)) on_hit(t, f);
    } else {
      // grazing pair: both faces go to the exact test
#pragma unroll 1
      for (int c = 0; c < 2; ++c) {
        const int f = c ? F.pb[pair] : fa;
        const float dn = c ? -dna : dna;
        float t;
        if (tri_test(F, f, oo, tlo, od, thi, dn, t) && front_facing(F, f, W, d)) on_hit(t, f);
      }
    }
  }
}

// Generic stack traversal.  thi() gives the current far bound; leaf(j, thi)
// tests proxy j.  Returns false if a bound was exceeded (status set).
template <class ThiFn, class LeafFn>
__device__ __forceinline__ void traverse(const SceneDev& S, const BoxRay& br, float tlo, ThiFn&& thi, LeafFn&& leaf,
                                         RayStats& st, uint32_t& status) {
  if (S.n_kept == 0) return;
  uint32_t stack_node[kStackSize];
  float stack_t[kStackSize];
  int sp = 0;
  uint32_t cur = S.root;
  uint32_t visits = 0;
  // a tree walk pops every internal node at most once
  const uint32_t max_visits = S.n_kept + 64u;
  while (true) {
    if (cur & kLeafBit) {
      ++st.proxy_tests;
      leaf(cur & ~kLeafBit, thi());
    } else {
      ++st.node_visits;
      if (++visits > max_visits) {
        status |= kStatusVisitCap;
        return;
      }
      const float4* nd = S.nodes + 4 * (size_t)cur;
      float4 f0 = __ldg(nd), f1 = __ldg(nd + 1), f2 = __ldg(nd + 2), f3 = __ldg(nd + 3);
      float n0, n1;
      bool h0, h1;
      node_test(f0, f1, f2, br, tlo, thi(), n0, n1, h0, h1);
      uint32_t c0 = __float_as_uint(f3.x), c1 = __float_as_uint(f3.y);
      if (h0 && h1) {
        bool swap = n1 < n0;
        uint32_t nearc = swap ? c1 : c0, farc = swap ? c0 : c1;
        float fart = swap ? n0 : n1;
        if (sp >= kStackSize) {
          status |= kStatusStackOverflow;
          return;
        }
        stack_node[sp] = farc;
        stack_t[sp] = fart;
        ++sp;
        cur = nearc;
        continue;
      } else if (h0) {
        cur = c0;
        continue;
      } else if (h1) {
        cur = c1;
        continue;
      }
    }
    // pop the next entry that is still in range
    bool found = false;
    while (sp > 0) {
      --sp;
      if (stack_t[sp] <= thi()) {
        cur = stack_node[sp];
        found = true;
        break;
      }
    }
    if (!found) return;
  }
}

// (t, p) < (bt, bp) in the round order
__device__ __forceinline__ bool hit_less(float t, uint32_t p, float bt, uint32_t bp) {
  return t < bt || (t == bt && p < bp);
}

template <int KMAX>
__device__ __forceinline__ void kinsert(float (&bt)[KMAX], uint32_t (&bp)[KMAX], float t, uint32_t p) {
#pragma unroll
  for (int i = 0; i < KMAX; ++i) {
    bool lt = hit_less(t, p, bt[i], bp[i]);
    float t2 = lt ? bt[i] : t;
    uint32_t p2 = lt ? bp[i] : p;
    bt[i] = lt ? t : bt[i];
    bp[i] = lt ? p : bp[i];
    t = t2;
    p = p2;
  }
}

// next float above x: the far bound of the triangle test that still admits
// a tie with the k-th hit
__device__ __forceinline__ float next_up(float x) { return nextafterf(x, CUDART_INF_F); }

// One round: the k closest front-face hits with t in (t_lo, t_max).
template <int KMAX>
__device__ __forceinline__ void collect_round(const SceneDev& S, const FaceTable& F, V3 o, V3 d, const BoxRay& br,
                                              float t_lo, float t_max, float (&bt)[KMAX], uint32_t (&bp)[KMAX],
                                              RayStats& st, uint32_t& status) {
  auto thi = [&]() { return bt[KMAX - 1]; };
  auto leaf = [&](uint32_t j, float far) {
    float tb = fminf(next_up(far), t_max);
    proxy_test<true>(F, S.w2o, j, o, d, t_lo, tb, [&](float t, int) {
      ++st.anyhits;
      uint32_t p = __ldg(S.leaf_pidx + j);
      if (hit_less(t, p, bt[KMAX - 1], bp[KMAX - 1])) kinsert<KMAX>(bt, bp, t, p);
    });
  };
  traverse(S, br, t_lo, thi, leaf, st, status);
}

struct NoRecord {
  __device__ __forceinline__ void entry(uint32_t, uint32_t, float, float) {}
};

struct HitRecord {
  uint32_t* pidx;
  float* t;
  float* alpha;
  uint32_t max_entries;
  __device__ __forceinline__ void entry(uint32_t n, uint32_t p, float tt, float a) {
    if (n < max_entries) {
      pidx[n] = p;
      t[n] = tt;
      alpha[n] = a;
    }
  }
};

// Per-lane state of one primary ray between rounds.
struct RayState {
  V3 o, d;
  BoxRay br;
  float L0, L1, L2, T, t_curr;
  uint32_t step, n_entries;
};

__device__ __forceinline__ void ray_init(const ViewDev& V, uint32_t px, uint32_t py, RayState& R) {
  ray_gen(V.u, V.w, V.h, px, py, R.o, R.d);
  R.br = make_boxray(R.o, R.d, V.s.scene_mag);
  R.L0 = R.L1 = R.L2 = 0.0f;
  R.T = 1.0f;
  R.t_curr = V.u.t_min;
  R.step = 0;
  R.n_entries = 0;
}

// The loop condition of tracePath (src/GS_shader.ts:231-234): another round
// starts while T_min < T and t_curr < t_max, unless earlyStop == step.
__device__ __forceinline__ bool ray_more(const ViewDev& V, const RayState& R) {
  return V.u.T_min < R.T && R.t_curr < V.u.t_max && V.u.early_stop != R.step;
}

// One round of tracePath (src/GS_shader.ts:235-269): collect the k closest
// front-face hits beyond t_curr, advance t_curr, composite the entries.
template <int KMAX, class Rec>
__device__ __forceinline__ void ray_round(const ViewDev& V, const FaceTable& F, RayState& R, RayStats& st,
                                          uint32_t& status, Rec& rec) {
  const float t_max = V.u.t_max;
  const int first = KMAX - (int)V.u.k;
  ++R.step;
  float bt[KMAX];
  uint32_t bp[KMAX];
#pragma unroll
  for (int i = 0; i < KMAX; ++i) {
    bt[i] = i < first ? -CUDART_INF_F : t_max;
    bp[i] = i < first ? 0u : kInvalid;
  }
  collect_round<KMAX>(V.s, F, R.o, R.d, R.br, R.t_curr, t_max, bt, bp, st, status);
  ++st.rounds;
  R.t_curr = bt[KMAX - 1] + 1e-4f;
#pragma unroll
  for (int i = 0; i < KMAX; ++i) {
    if (i < first) continue;
    if (bp[i] == kInvalid) {
      R.t_curr = t_max;
      break;
    }
    uint32_t p = bp[i];
    Shade sd = load_shade(V.s.shade, p);
    float alpha = response(sd, R.o, R.d) * sd.opacity;
    rec.entry(R.n_entries, p, bt[i], alpha);
    ++R.n_entries;
    ++st.entries;
    if (V.u.alpha_min < alpha) {
      ++st.contributing;
      V3 dir = vnorm(vsub(sd.mu, R.o));
      float c[3];
      sh_radiance(V.s.sh, p, dir, V.u.deg, c);
      float ta = R.T * alpha;
      R.L0 = R.L0 + ta * (c[0] > 0.0f ? c[0] : 0.0f);
      R.L1 = R.L1 + ta * (c[1] > 0.0f ? c[1] : 0.0f);
      R.L2 = R.L2 + ta * (c[2] > 0.0f ? c[2] : 0.0f);
      R.T = R.T * (1.0f - alpha);
    }
  }
  if (R.step >= kMaxRounds && ray_more(V, R)) {
    status |= kStatusRoundCap;
    R.t_curr = t_max;
  }
}

// tracePath (src/GS_shader.ts:192-273) for one pixel, all rounds.
template <int KMAX, class Rec>
__device__ __forceinline__ float4 trace_pixel(const ViewDev& V, const FaceTable& F, uint32_t px, uint32_t py,
                                              RayStats& st, uint32_t& status, Rec& rec, uint32_t* n_entries_out) {
  RayState R;
  ray_init(V, px, py, R);
  while (ray_more(V, R)) ray_round<KMAX>(V, F, R, st, status, rec);
  if (n_entries_out) *n_entries_out = R.n_entries;
  return make_float4(R.L0, R.L1, R.L2, 1.0f);
}

// Debug views (src/GS_shader.ts:201-228, 289-296, 312-321).
//   mode 1: closest proxy hit of any facing, coloured by max(0, SH(ray dir));
//   mode 2: number of front-face proxy hits in (t_min, t_max), bucketed.
__device__ __forceinline__ float4 trace_debug(const ViewDev& V, const FaceTable& F, uint32_t px, uint32_t py,
                                              RayStats& st, uint32_t& status, uint32_t* count_out) {
  V3 o, d;
  ray_gen(V.u, V.w, V.h, px, py, o, d);
  BoxRay br = make_boxray(o, d, V.s.scene_mag);
  const float t_max = V.u.t_max;
  if (V.u.debug == 1) {
    float bt = t_max;
    uint32_t bp = kInvalid;
    auto thi = [&]() { return bt; };
    auto leaf = [&](uint32_t j, float far) {
      float tb = bp == kInvalid ? t_max : fminf(next_up(far), t_max);
      proxy_test<false>(F, V.s.w2o, j, o, d, V.u.t_min, tb, [&](float t, int) {
        ++st.anyhits;
        uint32_t p = __ldg(V.s.leaf_pidx + j);
        if (hit_less(t, p, bt, bp)) {
          bt = t;
          bp = p;
        }
      });
    };
    traverse(V.s, br, V.u.t_min, thi, leaf, st, status);
    if (count_out) *count_out = bp == kInvalid ? 0u : 1u;
    if (bp == kInvalid) return make_float4(0.f, 0.f, 0.f, 1.f);
    float c[3];
    sh_radiance(V.s.sh, bp, d, V.u.deg, c);
    return make_float4(c[0] > 0.f ? c[0] : 0.f, c[1] > 0.f ? c[1] : 0.f, c[2] > 0.f ? c[2] : 0.f, 1.f);
  }
  uint32_t count = 0;
  auto thi = [&]() { return t_max; };
  auto leaf = [&](uint32_t j, float) {
    proxy_test<true>(F, V.s.w2o, j, o, d, V.u.t_min, t_max, [&](float, int) { ++count; });
  };
  traverse(V.s, br, V.u.t_min, thi, leaf, st, status);
  st.anyhits += count;
  if (count_out) *count_out = count;
  float r = 0.f, g = 0.f, b = 0.f;
  if (count == 0) {
  } else if (count < 20) { r = 0.5f; g = 0.5f; }
  else if (count < 40) { r = 0.5f; b = 0.5f; }
  else if (count < 60) { g = 0.5f; b = 0.5f; }
  else if (count < 80) { r = 0.5f; }
  else if (count < 100) { g = 0.5f; }
  else if (count < 150) { b = 0.5f; }
  else { r = 0.5f; g = 0.5f; b = 0.5f; }
  return make_float4(r, g, b, 1.f);
}

__device__ __forceinline__ void flush_stats(DevCounters* ctr, RayStats& st, uint32_t rays, uint32_t status) {
  unsigned long long v[7] = {rays, st.rounds, st.entries, st.contributing, st.proxy_tests, st.node_visits, st.anyhits};
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    unsigned long long x = v[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, off);
    v[i] = x;
  }
  uint32_t s = __reduce_or_sync(0xFFFFFFFFu, status);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&ctr->rays, v[0]);
    atomicAdd(&ctr->rounds, v[1]);
    atomicAdd(&ctr->entries, v[2]);
    atomicAdd(&ctr->contributing, v[3]);
    atomicAdd(&ctr->proxy_tests, v[4]);
    atomicAdd(&ctr->node_visits, v[5]);
    atomicAdd(&ctr->anyhits, v[6]);
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

// Persistent trace kernel over all pixels of all views.  Work items are
// pixel slots: slot = 32 * tile + lane-in-tile, tiles of 8x4 pixels in
// row-major order per view, views back to back.  A lane whose ray is done
// takes the next slot at once (warp-aggregated atomic), so rays of very
// different length do not hold whole warps idle.
template <int KMAX>
__global__ void __launch_bounds__(128) k_trace(const ViewDev* __restrict__ views, uint32_t n_views,
                                               uint32_t total_tiles, DevCounters* ctr,
                                               const __grid_constant__ FaceTable F) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint32_t total_slots = total_tiles * 32u;
  RayStats st = {0, 0, 0, 0, 0, 0};
  uint32_t status = 0, rays = 0;
  NoRecord rec;
  bool active = false, exhausted = false;
  uint32_t vi = 0, px = 0, py = 0;
  RayState R;
  while (true) {
    bool want = !active && !exhausted;
    uint32_t need = __ballot_sync(0xFFFFFFFFu, want);
    while (need) {
      int leader = __ffs(need) - 1;
      uint32_t base = 0;
      if ((int)lane == leader) base = atomicAdd(&ctr->work, (uint32_t)__popc(need));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      if (want) {
        uint32_t slot = base + __popc(need & lt_mask);
        if (slot >= total_slots || slot < base) {
          exhausted = true;
          want = false;
        } else {
          uint32_t tile = slot >> 5, s = slot & 31u;
          vi = n_views == 1 ? 0u : find_view(views, n_views, tile);
          const ViewDev& V = views[vi];
          uint32_t lt = tile - V.tile_begin;
          px = (lt % V.tiles_x) * kTileW + (s % kTileW);
          py = (lt / V.tiles_x) * kTileH + (s / kTileW);
          if (px < V.w && py < V.h) {
            want = false;
            if (V.u.debug == 0) {
              ray_init(V, px, py, R);
              active = ray_more(V, R);
              if (!active) {  // no round at all: black pixel
                V.out[(size_t)py * V.w + px] = make_float4(0.f, 0.f, 0.f, 1.f);
                ++rays;
              }
            } else {
              V.out[(size_t)py * V.w + px] = trace_debug(V, F, px, py, st, status, nullptr);
              ++rays;
            }
          }
        }
      }
      need = __ballot_sync(0xFFFFFFFFu, want);
    }
    if (!__any_sync(0xFFFFFFFFu, active)) break;
    if (active) {
      const ViewDev& V = views[vi];
      ray_round<KMAX>(V, F, R, st, status, rec);
      if (!ray_more(V, R)) {
        V.out[(size_t)py * V.w + px] = make_float4(R.L0, R.L1, R.L2, 1.0f);
        ++rays;
        active = false;
      }
    }
  }
  flush_stats(ctr, st, rays, status);
}

// Hit-list recording for listed pixels (parity and inspection).
template <int KMAX>
__global__ void __launch_bounds__(128) k_trace_hits(const ViewDev V, const uint32_t* pixels, uint32_t n_pix,
                                                    uint32_t max_entries, uint32_t* out_pidx, float* out_t,
                                                    float* out_alpha, uint32_t* out_count, uint32_t* out_rounds,
                                                    float4* out_rgba, DevCounters* ctr,
                                                    const __grid_constant__ FaceTable F) {
  uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  RayStats st = {0, 0, 0, 0, 0, 0};
  uint32_t status = 0, rays = 0;
  if (q < n_pix) {
    uint32_t pix = pixels[q];
    if (pix < V.w * V.h) {
      HitRecord rec{out_pidx + (size_t)q * max_entries, out_t + (size_t)q * max_entries,
                    out_alpha + (size_t)q * max_entries, max_entries};
      uint32_t n = 0;
      float4 r = V.u.debug == 0 ? trace_pixel<KMAX>(V, F, pix % V.w, pix / V.w, st, status, rec, &n)
                                : trace_debug(V, F, pix % V.w, pix / V.w, st, status, &n);
      out_count[q] = n;
      out_rounds[q] = st.rounds;
      if (out_rgba) out_rgba[q] = r;
      rays = 1;
    }
  }
  flush_stats(ctr, st, rays, status);
}

uint32_t kmax_for(uint32_t k) { return k <= 8 ? 8u : (k <= 16 ? 16u : 32u); }

Err launch_trace(const ViewDev* views, uint32_t n_views, uint32_t total_tiles, DevCounters* counters,
                 const FaceTable& faces, const LaunchShape& shape, int num_sms, cudaStream_t stream, uint64_t* launches,
                 ViewDev* d_views) {
  uint32_t kmax = 8;
  for (uint32_t v = 0; v < n_views; ++v) kmax = kmax_for(std::max(kmax, views[v].u.k));
  GT_CUDA_TRY(cudaMemcpyAsync(d_views, views, sizeof(ViewDev) * n_views, cudaMemcpyHostToDevice, stream));
  uint32_t warps_needed = total_tiles;
  uint32_t block = 128;
  uint32_t grid = (uint32_t)num_sms * std::max(1u, shape.blocks_per_sm);
  uint32_t max_grid = (warps_needed + (block / 32) - 1) / (block / 32);
  if (grid > max_grid) grid = std::max(1u, max_grid);
  if (kmax == 8)
    k_trace<8><<<grid, block, 0, stream>>>(d_views, n_views, total_tiles, counters, faces);
  else if (kmax == 16)
    k_trace<16><<<grid, block, 0, stream>>>(d_views, n_views, total_tiles, counters, faces);
  else
    k_trace<32><<<grid, block, 0, stream>>>(d_views, n_views, total_tiles, counters, faces);
  ++*launches;
  GT_CUDA_TRY(cudaGetLastError());
  return Err{};
}

Err launch_trace_hits(const ViewDev& view, const uint32_t* pixels, uint32_t n_pix, uint32_t max_entries,
                      uint32_t* out_pidx, float* out_t, float* out_alpha, uint32_t* out_count, uint32_t* out_rounds,
                      float4* out_rgba, DevCounters* counters, const FaceTable& faces, cudaStream_t stream,
                      uint64_t* launches) {
  uint32_t kmax = kmax_for(view.u.k);
  uint32_t grid = (n_pix + 127) / 128;
  if (grid == 0) return Err{};
  if (kmax == 8)
    k_trace_hits<8><<<grid, 128, 0, stream>>>(view, pixels, n_pix, max_entries, out_pidx, out_t, out_alpha, out_count,
                                              out_rounds, out_rgba, counters, faces);
  else if (kmax == 16)
    k_trace_hits<16><<<grid, 128, 0, stream>>>(view, pixels, n_pix, max_entries, out_pidx, out_t, out_alpha,
                                               out_count, out_rounds, out_rgba, counters, faces);
  else
    k_trace_hits<32><<<grid, 128, 0, stream>>>(view, pixels, n_pix, max_entries, out_pidx, out_t, out_alpha,
                                               out_count, out_rounds, out_rgba, counters, faces);
  ++*launches;
  GT_CUDA_TRY(cudaGetLastError());
  return Err{};
}

}  // namespace gt
