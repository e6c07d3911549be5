// gt_build.cu — GPU scene build: proxies, LBVH, shading records.
//
// Replaces the reference's host-side acceleration-structure build
// (gaussianSceneToBvh, src/main.ts:30-111; Tlas.build,
// webrtx/src/wasm_bvh_builder.ts:260-377; build_blas/build_tlas,
// webrtx/bvh/src/lib.rs:254-347, 512-603) with a linear BVH built on the GPU:
//
//   1. keep flags (opacity > alpha_min) and an exclusive scan  -> kept list
//   2. per kept particle: proxy matrix M = T R diag(s*scale), world AABB of
//      the 12 transformed icosahedron vertices, box centre, scene bounds
//   3. 30-bit Morton codes of the box centres
//   4. LSD radix sort of (code, kept slot), 4 passes of 8 bits, hand-written
//      (per-tile histograms, one scan, stable warp-ranked scatter)
//   5. Karras (2012) hierarchy over the sorted codes, ties broken by index
//   6. bottom-up refit with one atomic arrival counter per internal node
//   7. leaf records in leaf order (world-to-object map, particle index) and
//      shading records in particle order (mean, opacity, precision matrix, SH)
//
// Node layout (4 x float4 per internal node; children's boxes in the parent):
//   f0 = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   f1 = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   f2 = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   f3 = (child0, child1, 0, 0) as uint bits; kLeafBit | j marks leaf j.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gt_device.cuh"
#include "gt_internal.cuh"

namespace gt {

// ---------------------------------------------------------------- faces
// Icosahedron with inradius 1 (src/main.ts:12-25).
static const int kIcoIdx[60] = {0, 11, 5,  0, 5,  1,  0,  1,  7,  0,  7,  10, 0, 10, 11,
                                1, 5,  9,  5, 11, 4,  11, 10, 2,  10, 7,  6,  7, 1,  8,
                                3, 9,  4,  3, 4,  2,  3,  2,  6,  3,  6,  8,  3, 8,  9,
                                4, 9,  5,  2, 4,  11, 6,  2,  10, 8,  6,  7,  9, 8,  1};

static void ico_vertices(float v[36]) {
  double rr = (3.0 + sqrt(5.0)) / (2.0 * sqrt(3.0));
  double ss = 1.0 / rr;
  double tt = (1.0 + sqrt(5.0)) / (2.0 * rr);
  double t[36] = {-ss, tt, 0, ss,  tt, 0,  -ss, -tt, 0,   ss,  -tt, 0,   0,   -ss, tt,  0, ss,  tt,
                  0,   -ss, -tt, 0, ss, -tt, tt,  0,   -ss, tt,  0,   ss,  -tt, 0,   -ss, -tt, 0, ss};
  for (int i = 0; i < 36; ++i) v[i] = (float)t[i];
}

void make_face_table(FaceTable* F) {
  // Host code is compiled with -ffp-contract=off: each expression below is
  // rounded exactly as the device and the oracle round it.
  float v[36];
  ico_vertices(v);
  float nmax = 0.0f;
  for (int f = 0; f < 20; ++f) {
    const float* p0 = v + 3 * kIcoIdx[3 * f];
    const float* p1 = v + 3 * kIcoIdx[3 * f + 1];
    const float* p2 = v + 3 * kIcoIdx[3 * f + 2];
    float e0[3], e1[3];
    for (int a = 0; a < 3; ++a) {
      e0[a] = p1[a] - p0[a];
      e1[a] = p0[a] - p2[a];
      F->p0[f][a] = p0[a];
      F->e0[f][a] = e0[a];
      F->e1[f][a] = e1[a];
    }
    // n = cross(e1, e0)
    F->n[f][0] = e1[1] * e0[2] - e1[2] * e0[1];
    F->n[f][1] = e1[2] * e0[0] - e1[0] * e0[2];
    F->n[f][2] = e1[0] * e0[1] - e1[1] * e0[0];
    for (int a = 0; a < 3; ++a) nmax = fmaxf(nmax, fabsf(F->n[f][a]));
  }
  F->nmax = nmax;
  float r = 0.0f;
  for (int i = 0; i < 12; ++i)
    r = fmaxf(r, sqrtf(v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]));
  F->r_circ = r;
  float em = 0.0f;
  for (int f = 0; f < 20; ++f) {
    em = fmaxf(em, fabsf(F->e0[f][0]) + fabsf(F->e0[f][1]) + fabsf(F->e0[f][2]));
    em = fmaxf(em, fabsf(F->e1[f][0]) + fabsf(F->e1[f][1]) + fabsf(F->e1[f][2]));
  }
  F->emax = em;
  for (int f = 0; f < 20; ++f)
    F->c[f] = F->n[f][0] * F->p0[f][0] + F->n[f][1] * F->p0[f][1] + F->n[f][2] * F->p0[f][2];
  // antipodal pairs: the face whose vertices are the negated vertices of f
  int q = 0;
  bool used[20] = {false};
  for (int f = 0; f < 20 && q < 10; ++f) {
    if (used[f]) continue;
    for (int g = f + 1; g < 20; ++g) {
      int match = 0;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          const float* va = v + 3 * kIcoIdx[3 * f + a];
          const float* vb = v + 3 * kIcoIdx[3 * g + b];
          if (va[0] == -vb[0] && va[1] == -vb[1] && va[2] == -vb[2]) ++match;
        }
      bool neg = F->n[g][0] == -F->n[f][0] && F->n[g][1] == -F->n[f][1] && F->n[g][2] == -F->n[f][2];
      if (match == 3 && neg) {
        F->pa[q] = f;
        F->pb[q] = g;
        used[f] = used[g] = true;
        ++q;
        break;
      }
    }
  }
  F->npairs = q;
  for (int r = 0; r < q; ++r) {
    for (int a = 0; a < 3; ++a) F->pn[r][a] = F->n[F->pa[r]][a];
    F->pca[r] = F->c[F->pa[r]];
    F->pcb[r] = F->c[F->pb[r]];
  }
  F->lim_steps = 0xFFFFFFFFu;
  F->lim_stack = kWarpStack;
  F->lim_rounds = kMaxRounds;
}
static_assert(sizeof(kIcoIdx) == 60 * sizeof(int), "table size");

struct IcoVerts {
  float v[36];
};

// ---------------------------------------------------------------- proxies
// src/main.ts:79-94: s = sqrt(2 ln(o / alpha_min)); M = T(mu) R diag(s*scale)
// with R = wgpu-matrix mat3.fromQuat([x, y, z, w]) evaluated in double and
// rounded to binary32 (Float32Array), s*scale rounded to binary32, and each
// column entry the binary32 product of the two.
// The activated values the proxy is built from: opacity, scale xyz and
// rotation wxyz.  The reference builds its proxies from the JS numbers of
// gaussianData (double); when the caller supplies them (act64, 8 doubles per
// particle in that order) they are used, else the packed binary32 values.
struct Act64 {
  double o, s[3], q[4];
};
__device__ __forceinline__ Act64 activation(const float* rec, const double* act64, uint64_t i) {
  Act64 a;
  if (act64) {
    const double* p = act64 + 8 * i;
    a.o = p[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) a.s[c] = p[1 + c];
#pragma unroll
    for (int c = 0; c < 4; ++c) a.q[c] = p[4 + c];
  } else {
    a.o = rec[12];
#pragma unroll
    for (int c = 0; c < 3; ++c) a.s[c] = rec[4 + c];
#pragma unroll
    for (int c = 0; c < 4; ++c) a.q[c] = rec[8 + c];
  }
  return a;
}

__device__ __forceinline__ void proxy_o2w(const float* rec, const Act64& A, double alpha_min, float M[12]) {
  double o = A.o;
  double s = __dsqrt_rn(__dmul_rn(2.0, det_log(__ddiv_rn(o, alpha_min))));
  double w = A.q[0], x = A.q[1], y = A.q[2], z = A.q[3];
  double x2 = x + x, y2 = y + y, z2 = z + z;
  double xx = x * x2, yx = y * x2, yy = y * y2;
  double zx = z * x2, zy = z * y2, zz = z * z2;
  double wx = w * x2, wy = w * y2, wz = w * z2;
  double R[9] = {1.0 - yy - zz, yx + wz, zx - wy, yx - wz, 1.0 - xx - zz, zy + wx, zx + wy, zy - wx, 1.0 - xx - yy};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float Sc = __double2float_rn(__dmul_rn(s, A.s[c]));
#pragma unroll
    for (int r = 0; r < 3; ++r) M[3 * c + r] = __double2float_rn(R[3 * c + r]) * Sc;
  }
  M[9] = rec[0];
  M[10] = rec[1];
  M[11] = rec[2];
}

// Affine inverse (replaces glam Affine3A::inverse, webrtx/bvh/src/lib.rs:501-505):
// adjugate from cross products of the columns a, b, c; det = dot(c, cross(a, b)).
__device__ __forceinline__ void affine_inverse(const float M[12], float W[12]) {
  V3 a = mk(M[0], M[1], M[2]), b = mk(M[3], M[4], M[5]), c = mk(M[6], M[7], M[8]);
  V3 p = mk(M[9], M[10], M[11]);
  V3 t0 = vcross(b, c), t1 = vcross(c, a), t2 = vcross(a, b);
  float det = vdot(c, t2);
  float inv = __fdiv_rn(1.0f, det);
  W[0] = t0.x * inv; W[1] = t1.x * inv; W[2] = t2.x * inv;
  W[3] = t0.y * inv; W[4] = t1.y * inv; W[5] = t2.y * inv;
  W[6] = t0.z * inv; W[7] = t1.z * inv; W[8] = t2.z * inv;
  W[9] = -((W[0] * p.x + W[3] * p.y) + W[6] * p.z);
  W[10] = -((W[1] * p.x + W[4] * p.y) + W[7] * p.z);
  W[11] = -((W[2] * p.x + W[5] * p.y) + W[8] * p.z);
}

__device__ __forceinline__ const float* record(const uint8_t* packed, uint64_t i, uint32_t stride) {
  return reinterpret_cast<const float*>(packed + i * (uint64_t)stride);
}

__global__ void k_keep_flags(const uint8_t* packed, uint64_t n, uint32_t stride, double alpha_min,
                             const double* act64, uint32_t* flags) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double o = act64 ? act64[8 * i] : (double)record(packed, i, stride)[12];
  flags[i] = (o > alpha_min) ? 1u : 0u;
}

// float min/max through order-preserving integer maps (for atomics)
__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__global__ void k_proxy_boxes(const uint8_t* packed, uint64_t n, uint32_t stride, double alpha_min,
                              const double* act64, const uint32_t* flags, const uint32_t* slots, const IcoVerts iv, float* box,
                              uint32_t* kept_pidx, uint32_t* bounds_ord) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  float cmin[3] = {CUDART_INF_F, CUDART_INF_F, CUDART_INF_F}, cmax[3] = {-CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F};
  float bmag = 0.0f;
  if (i < n && flags[i]) {
    const float* rec = record(packed, i, stride);
    float M[12];
    proxy_o2w(rec, activation(rec, act64, i), alpha_min, M);
    Affine A;
#pragma unroll
    for (int q = 0; q < 12; ++q) A.m[q] = M[q];
    float lo[3] = {CUDART_INF_F, CUDART_INF_F, CUDART_INF_F}, hi[3] = {-CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F};
#pragma unroll
    for (int v = 0; v < 12; ++v) {
      V3 w = xpoint(A, mk(iv.v[3 * v], iv.v[3 * v + 1], iv.v[3 * v + 2]));
      lo[0] = fminf(lo[0], w.x); lo[1] = fminf(lo[1], w.y); lo[2] = fminf(lo[2], w.z);
      hi[0] = fmaxf(hi[0], w.x); hi[1] = fmaxf(hi[1], w.y); hi[2] = fmaxf(hi[2], w.z);
    }
    float ext = fmaxf(fmaxf(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
    float mag = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) mag = fmaxf(mag, fmaxf(fabsf(lo[a]), fabsf(hi[a])));
    // conservative padding for the rounding of the vertex transform
    float pad = __fmaf_rn(1e-5f, ext, 2e-6f * (mag + 1.0f));
    uint32_t s = slots[i];
    float* b = box + 6 * (size_t)s;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      b[a] = lo[a] - pad;
      b[3 + a] = hi[a] + pad;
      float c = 0.5f * (b[a] + b[3 + a]);
      cmin[a] = c;
      cmax[a] = c;
      bmag = fmaxf(bmag, fmaxf(fabsf(b[a]), fabsf(b[3 + a])));
    }
    kept_pidx[s] = (uint32_t)i;
  }
  // warp-reduce the centre bounds, then one atomic per warp
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      cmin[a] = fminf(cmin[a], __shfl_xor_sync(0xFFFFFFFFu, cmin[a], off));
      cmax[a] = fmaxf(cmax[a], __shfl_xor_sync(0xFFFFFFFFu, cmax[a], off));
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) bmag = fmaxf(bmag, __shfl_xor_sync(0xFFFFFFFFu, bmag, off));
  if ((threadIdx.x & 31) == 0 && cmin[0] <= cmax[0]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      atomicMin(&bounds_ord[a], f2ord(cmin[a]));
      atomicMax(&bounds_ord[3 + a], f2ord(cmax[a]));
    }
    atomicMax(&bounds_ord[6], f2ord(bmag));
  }
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__global__ void k_morton(const float* box, uint32_t m, const uint32_t* bounds_ord, uint32_t* keys,
                         uint32_t* vals) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  uint32_t code = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float lo = ord2f(bounds_ord[a]), hi = ord2f(bounds_ord[3 + a]);
    float c = 0.5f * (box[6 * (size_t)j + a] + box[6 * (size_t)j + 3 + a]);
    float e = hi - lo;
    float u = e > 0.0f ? (c - lo) / e : 0.0f;
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    uint32_t q = (uint32_t)(u * 1023.0f);
    code |= spread10(q) << (2 - a);
  }
  keys[j] = code;
  vals[j] = j;
}

// ------------------------------------------------------------------ scan
constexpr int kScanBlock = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_sums[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
    uint32_t s = lane < nw ? warp_sums[lane] : 0u;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, off);
      if (lane >= off) s += y;
    }
    warp_sums[lane] = s;
  }
  __syncthreads();
  uint32_t base = warp ? warp_sums[warp - 1] : 0u;
  if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

__global__ void k_scan_tiles(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* tile_sums) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (base + i < n) ? in[base + i] : 0u;
    sum += v[i];
  }
  uint32_t total;
  uint32_t pre = block_exclusive_scan(sum, &total);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = pre;
    pre += v[i];
  }
  if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(uint32_t* out, uint64_t n, const uint32_t* tile_offsets) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t add = tile_offsets[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) out[base + i] += add;
}

// Exclusive scan of n uint32 values (in may equal out).  Temporaries are
// stream-ordered allocations.
Err scan_exclusive(const uint32_t* in, uint32_t* out, uint64_t n, cudaStream_t st, uint64_t* launches) {
  if (n == 0) return Err{};
  uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    k_scan_tiles<<<1, kScanBlock, 0, st>>>(in, out, n, nullptr);
    ++*launches;
    GT_CUDA_TRY(cudaGetLastError());
    return Err{};
  }
  uint32_t* sums = nullptr;
  GT_CUDA_TRY(cudaMallocAsync(&sums, tiles * sizeof(uint32_t), st));
  k_scan_tiles<<<(unsigned)tiles, kScanBlock, 0, st>>>(in, out, n, sums);
  ++*launches;
  Err e = scan_exclusive(sums, sums, tiles, st, launches);
  if (e.code == GT_OK) {
    k_scan_add<<<(unsigned)tiles, kScanBlock, 0, st>>>(out, n, sums);
    ++*launches;
  }
  cudaFreeAsync(sums, st);
  if (e.code != GT_OK) return e;
  GT_CUDA_TRY(cudaGetLastError());
  return Err{};
}

// ------------------------------------------------------------ radix sort
constexpr int kRsBlock = 256;
constexpr int kRsItems = 8;
constexpr int kRsTile = kRsBlock * kRsItems;

__global__ void k_rs_hist(const uint32_t* keys, uint32_t n, int shift, uint32_t* hist, uint32_t n_tiles) {
  __shared__ uint32_t cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  uint32_t base = blockIdx.x * kRsTile;
#pragma unroll
  for (int r = 0; r < kRsItems; ++r) {
    uint32_t i = base + r * kRsBlock + threadIdx.x;
    if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * n_tiles + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter: items of a tile are ranked in index order, warp by warp.
__global__ void k_rs_scatter(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, uint32_t n,
                             int shift, const uint32_t* offsets, uint32_t n_tiles) {
  __shared__ uint32_t running[256];
  __shared__ uint32_t whist[kRsBlock / 32][257];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  running[threadIdx.x] = offsets[threadIdx.x * n_tiles + blockIdx.x];
  uint32_t base = blockIdx.x * kRsTile;
  const uint32_t lt_mask = (1u << lane) - 1u;
  for (int r = 0; r < kRsItems; ++r) {
    for (int q = threadIdx.x; q < (kRsBlock / 32) * 257; q += kRsBlock) (&whist[0][0])[q] = 0;
    __syncthreads();
    uint32_t i = base + r * kRsBlock + threadIdx.x;
    uint32_t key = 0, val = 0, digit = 256;
    if (i < n) {
      key = kin[i];
      val = vin[i];
      digit = (key >> shift) & 255u;
    }
    uint32_t peers = __match_any_sync(0xFFFFFFFFu, digit);
    uint32_t rank = __popc(peers & lt_mask);
    if (rank == 0 && digit < 256) whist[warp][digit] = __popc(peers);
    __syncthreads();
    {
      uint32_t d = threadIdx.x;  // kRsBlock == 256 digits
      uint32_t acc = running[d];
#pragma unroll
      for (int w = 0; w < kRsBlock / 32; ++w) {
        uint32_t c = whist[w][d];
        whist[w][d] = acc;
        acc += c;
      }
      running[d] = acc;
    }
    __syncthreads();
    if (digit < 256) {
      uint32_t pos = whist[warp][digit] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
  }
}

static Err radix_sort(uint32_t* keys, uint32_t* vals, uint32_t n, cudaStream_t st, uint64_t* launches) {
  if (n <= 1) return Err{};
  uint32_t n_tiles = (n + kRsTile - 1) / kRsTile;
  uint32_t *k2 = nullptr, *v2 = nullptr, *hist = nullptr;
  GT_CUDA_TRY(cudaMallocAsync(&k2, (size_t)n * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&v2, (size_t)n * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&hist, (size_t)256 * n_tiles * 4, st));
  uint32_t *ka = keys, *va = vals, *kb = k2, *vb = v2;
  Err e;
  for (int shift = 0; shift < 32; shift += 8) {
    k_rs_hist<<<n_tiles, kRsBlock, 0, st>>>(ka, n, shift, hist, n_tiles);
    ++*launches;
    e = scan_exclusive(hist, hist, (uint64_t)256 * n_tiles, st, launches);
    if (e.code != GT_OK) break;
    k_rs_scatter<<<n_tiles, kRsBlock, 0, st>>>(ka, va, kb, vb, n, shift, hist, n_tiles);
    ++*launches;
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  // four passes: the sorted data is back in keys/vals
  cudaFreeAsync(k2, st);
  cudaFreeAsync(v2, st);
  cudaFreeAsync(hist, st);
  if (e.code != GT_OK) return e;
  GT_CUDA_TRY(cudaGetLastError());
  return Err{};
}

// -------------------------------------------------------------- hierarchy
__device__ __forceinline__ int kdelta(const uint32_t* k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint32_t a = k[i], b = k[j];
  if (a == b) return 32 + __clz((uint32_t)i ^ (uint32_t)j);
  return __clz(a ^ b);
}

// Karras 2012, "Maximizing parallelism in the construction of BVHs, octrees
// and k-d trees": internal node i covers a key range found by one exponential
// and two binary searches on the longest common prefix.
__global__ void k_karras(const uint32_t* keys, int n, float4* nodes, uint32_t* parent_int, uint32_t* parent_leaf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = kdelta(keys, n, i, i - d);
  int lmax = 2;
  while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  int j = i + l * d;
  int dnode = kdelta(keys, n, i, j);
  int s = 0, t = l;
  do {
    t = (t + 1) / 2;
    if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  int gamma = i + s * d + min(d, 0);
  int lo = min(i, j), hi = max(i, j);
  uint32_t c0 = (lo == gamma) ? (kLeafBit | (uint32_t)gamma) : (uint32_t)gamma;
  uint32_t c1 = (hi == gamma + 1) ? (kLeafBit | (uint32_t)(gamma + 1)) : (uint32_t)(gamma + 1);
  nodes[4 * (size_t)i + 3] = make_float4(__uint_as_float(c0), __uint_as_float(c1), 0.f, 0.f);
  if (c0 & kLeafBit) parent_leaf[gamma] = (uint32_t)i; else parent_int[gamma] = (uint32_t)i;
  if (c1 & kLeafBit) parent_leaf[gamma + 1] = (uint32_t)i; else parent_int[gamma + 1] = (uint32_t)i;
  if (i == 0) parent_int[0] = kInvalid;
}

// Leaf records in leaf order: world-to-object map, particle index, box.
__global__ void k_leaves(const uint8_t* packed, uint32_t stride, double alpha_min, const double* act64,
                         const uint32_t* sorted_slots, uint32_t m, const uint32_t* kept_pidx, const float* box_by_slot, float4* w2o,
                         uint32_t* leaf_pidx, float* leaf_box) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  uint32_t slot = sorted_slots[j];
  uint32_t p = kept_pidx[slot];
  float M[12], W[12];
  const float* rec = record(packed, p, stride);
  proxy_o2w(rec, activation(rec, act64, p), alpha_min, M);
  affine_inverse(M, W);
  w2o[3 * (size_t)j] = make_float4(W[0], W[1], W[2], W[3]);
  w2o[3 * (size_t)j + 1] = make_float4(W[4], W[5], W[6], W[7]);
  w2o[3 * (size_t)j + 2] = make_float4(W[8], W[9], W[10], W[11]);
  leaf_pidx[j] = p;
#pragma unroll
  for (int a = 0; a < 6; ++a) leaf_box[6 * (size_t)j + a] = box_by_slot[6 * (size_t)slot + a];
}

__device__ __forceinline__ void child_box(uint32_t ref, const float* leaf_box, const float* ibox, float b[6]) {
  const float* src = (ref & kLeafBit) ? leaf_box + 6 * (size_t)(ref & ~kLeafBit) : ibox + 6 * (size_t)ref;
#pragma unroll
  for (int a = 0; a < 6; ++a) b[a] = __ldcg(src + a);
}

// Bottom-up refit: the second child to arrive at a node writes its boxes.
__global__ void k_refit(uint32_t m, const float* leaf_box, float* ibox, float4* nodes, const uint32_t* parent_int,
                        const uint32_t* parent_leaf, uint32_t* arrive) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  uint32_t node = parent_leaf[j];
  uint32_t guard = 0;
  while (node != kInvalid && guard++ < 4096u) {
    __threadfence();
    if (atomicAdd(&arrive[node], 1u) == 0u) return;
    float4 f3 = __ldcg(nodes + 4 * (size_t)node + 3);
    uint32_t c0 = __float_as_uint(f3.x), c1 = __float_as_uint(f3.y);
    float b0[6], b1[6];
    child_box(c0, leaf_box, ibox, b0);
    child_box(c1, leaf_box, ibox, b1);
    nodes[4 * (size_t)node + 0] = make_float4(b0[0], b0[3], b0[1], b0[4]);
    nodes[4 * (size_t)node + 1] = make_float4(b1[0], b1[3], b1[1], b1[4]);
    nodes[4 * (size_t)node + 2] = make_float4(b0[2], b0[5], b1[2], b1[5]);
    float* ib = ibox + 6 * (size_t)node;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      ib[a] = fminf(b0[a], b1[a]);
      ib[3 + a] = fmaxf(b0[3 + a], b1[3 + a]);
    }
    node = parent_int[node];
  }
}

// Tree check before any traversal: every child reference in range and every
// node reached by exactly one parent (the root by none).
__global__ void k_check_children(uint32_t m, const float4* nodes, uint32_t* refcount, uint32_t* bad) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i + 1 >= m) return;
  float4 f3 = nodes[4 * (size_t)i + 3];
  uint32_t c[2] = {__float_as_uint(f3.x), __float_as_uint(f3.y)};
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    uint32_t r = c[q];
    if (r & kLeafBit) {
      uint32_t j = r & ~kLeafBit;
      if (j >= m) atomicOr(bad, 1u); else atomicAdd(&refcount[(m - 1) + j], 1u);
    } else {
      if (r >= m - 1 || r == 0) atomicOr(bad, 2u); else atomicAdd(&refcount[r], 1u);
    }
  }
}
__global__ void k_check_counts(uint32_t total, const uint32_t* refcount, uint32_t* bad) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  uint32_t expect = i == 0 ? 0u : 1u;
  if (refcount[i] != expect) atomicOr(bad, 4u);
}

__global__ void k_depth(uint32_t m, const uint32_t* parent_int, const uint32_t* parent_leaf, uint32_t* depth) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  uint32_t d = 0, node = parent_leaf[j];
  while (node != kInvalid && d < 100000u) {
    ++d;
    node = parent_int[node];
  }
  atomicMax(depth, d);
}

// Shading records in particle order: (mu, opacity), precision matrix A of
// computeResponse (6 unique entries), and the 48 SH floats made tight.
__global__ void k_shade(const uint8_t* packed, uint64_t n, uint32_t stride, uint32_t n_sh, const uint32_t* flags,
                        float4* shade, float4* sh, float4* params) {
  uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (p >= n || !flags[p]) return;
  const float* rec = record(packed, p, stride);
  float q[4] = {rec[8], rec[9], rec[10], rec[11]};
  float sc[3] = {rec[4], rec[5], rec[6]};
  float A[3][3];
  precision_matrix(q, sc, A);
  shade[3 * p] = make_float4(rec[0], rec[1], rec[2], rec[12]);
  params[2 * p] = make_float4(sc[0], sc[1], sc[2], 0.f);
  params[2 * p + 1] = make_float4(q[0], q[1], q[2], q[3]);
  shade[3 * p + 1] = make_float4(A[0][0], A[1][0], A[2][0], A[1][1]);
  shade[3 * p + 2] = make_float4(A[2][1], A[2][2], 0.f, 0.f);
  float v[48];
#pragma unroll
  for (int k = 0; k < 16; ++k)
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) v[3 * k + ch] = (uint32_t)k < n_sh ? rec[16 + 4 * k + ch] : 0.0f;
#pragma unroll
  for (int i = 0; i < 12; ++i) sh[12 * p + i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
}

// ------------------------------------------------------------- BVH8 collapse
// Greedy collapse of the binary hierarchy into 8-wide nodes: a node starts
// with the two children of a binary node and repeatedly opens its internal
// entry of largest surface area until it holds 8 entries or only leaves.
// Each binary internal node ends up inside exactly one 8-wide node, and
// every 8-wide node opens at least one binary node, so there are fewer
// 8-wide nodes than binary internal nodes.
//
// 8-wide node layout: 8 child records of 32 bytes (2 float4):
//   f0 = (lo.x, lo.y, lo.z, hi.x), f1 = (hi.y, hi.z, ref, 0)
// ref = kLeafBit | j for leaf j, an 8-wide node index, or kInvalid (empty
// slot, with an empty box).
struct Entry8 {
  float b[6];
  uint32_t ref;  // binary reference: kLeafBit | j or internal index
};

__device__ __forceinline__ void binary_children(const float4* bn, uint32_t i, Entry8& c0, Entry8& c1) {
  float4 f0 = bn[4 * (size_t)i], f1 = bn[4 * (size_t)i + 1], f2 = bn[4 * (size_t)i + 2], f3 = bn[4 * (size_t)i + 3];
  c0.b[0] = f0.x; c0.b[3] = f0.y; c0.b[1] = f0.z; c0.b[4] = f0.w; c0.b[2] = f2.x; c0.b[5] = f2.y;
  c1.b[0] = f1.x; c1.b[3] = f1.y; c1.b[1] = f1.z; c1.b[4] = f1.w; c1.b[2] = f2.z; c1.b[5] = f2.w;
  c0.ref = __float_as_uint(f3.x);
  c1.ref = __float_as_uint(f3.y);
}

__device__ __forceinline__ float half_area(const float b[6]) {
  float x = b[3] - b[0], y = b[4] - b[1], z = b[5] - b[2];
  return x * y + y * z + z * x;
}

__global__ void k_collapse8(const float4* bn, const uint32_t* front_bin, const uint32_t* front_n8, uint32_t n_front,
                            float4* nodes8, uint32_t* next_bin, uint32_t* next_n8, uint32_t* counters,
                            uint32_t max_nodes8) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_front) return;
  uint32_t bi = front_bin[i], n8 = front_n8[i];
  Entry8 e[8];
  binary_children(bn, bi, e[0], e[1]);
  int cnt = 2;
  while (cnt < 8) {
    int best = -1;
    float ba = -1.0f;
    for (int q = 0; q < cnt; ++q) {
      if (e[q].ref & kLeafBit) continue;
      float a = half_area(e[q].b);
      if (a > ba) {
        ba = a;
        best = q;
      }
    }
    if (best < 0) break;
    Entry8 c0, c1;
    binary_children(bn, e[best].ref, c0, c1);
    e[best] = c0;
    e[cnt++] = c1;
  }
  float4* out = nodes8 + 16 * (size_t)n8;
  for (int q = 0; q < 8; ++q) {
    if (q < cnt) {
      uint32_t ref = e[q].ref;
      if (!(ref & kLeafBit)) {
        uint32_t child8 = atomicAdd(&counters[0], 1u);
        if (child8 >= max_nodes8) {
          atomicOr(&counters[2], 1u);
          child8 = 0;
        } else {
          uint32_t slot = atomicAdd(&counters[1], 1u);
          next_bin[slot] = ref;
          next_n8[slot] = child8;
        }
        ref = child8;
      }
      out[2 * q] = make_float4(e[q].b[0], e[q].b[1], e[q].b[2], e[q].b[3]);
      out[2 * q + 1] = make_float4(e[q].b[4], e[q].b[5], __uint_as_float(ref), 0.f);
    } else {
      out[2 * q] = make_float4(1e30f, 1e30f, 1e30f, -1e30f);
      out[2 * q + 1] = make_float4(-1e30f, -1e30f, __uint_as_float(kInvalid), 0.f);
    }
  }
}

// Collapses the binary hierarchy (m leaves) into `*out8` (exactly sized).
static Err collapse_bvh8(const float4* bn, const float* leaf_box, uint32_t m, cudaStream_t st, float4** out8,
                         uint32_t* n_nodes8, uint64_t* launches) {
  uint32_t cap = std::max<uint32_t>(m > 1 ? m - 1 : 1, 1);
  float4* tmp = nullptr;
  uint32_t *fb = nullptr, *fn = nullptr, *nb = nullptr, *nn = nullptr, *ctr = nullptr;
  GT_CUDA_TRY(cudaMallocAsync(&tmp, (size_t)cap * 16 * sizeof(float4), st));
  GT_CUDA_TRY(cudaMallocAsync(&fb, (size_t)cap * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&fn, (size_t)cap * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&nb, (size_t)cap * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&nn, (size_t)cap * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&ctr, 4 * 4, st));
  uint32_t total = 1;
  if (m == 1) {
    float lb[6];
    GT_CUDA_TRY(cudaMemcpyAsync(lb, leaf_box, sizeof lb, cudaMemcpyDeviceToHost, st));
    GT_CUDA_TRY(cudaStreamSynchronize(st));
    auto bits = [](uint32_t u) {
      float f;
      memcpy(&f, &u, 4);
      return f;
    };
    float4 host[16];
    host[0] = make_float4(lb[0], lb[1], lb[2], lb[3]);
    host[1] = make_float4(lb[4], lb[5], bits(kLeafBit | 0u), 0.f);
    for (int q = 1; q < 8; ++q) {
      host[2 * q] = make_float4(1e30f, 1e30f, 1e30f, -1e30f);
      host[2 * q + 1] = make_float4(-1e30f, -1e30f, bits(kInvalid), 0.f);
    }
    GT_CUDA_TRY(cudaMemcpyAsync(tmp, host, sizeof host, cudaMemcpyHostToDevice, st));
  } else {
    uint32_t init[4] = {1u, 0u, 0u, 0u};
    uint32_t zero = 0u;
    GT_CUDA_TRY(cudaMemcpyAsync(ctr, init, sizeof init, cudaMemcpyHostToDevice, st));
    GT_CUDA_TRY(cudaMemcpyAsync(fb, &zero, 4, cudaMemcpyHostToDevice, st));
    GT_CUDA_TRY(cudaMemcpyAsync(fn, &zero, 4, cudaMemcpyHostToDevice, st));
    uint32_t n_front = 1;
    for (int level = 0; n_front > 0 && level < 1000; ++level) {
      GT_CUDA_TRY(cudaMemsetAsync(ctr + 1, 0, 4, st));
      k_collapse8<<<(n_front + 127) / 128, 128, 0, st>>>(bn, fb, fn, n_front, tmp, nb, nn, ctr, cap);
      ++*launches;
      GT_CUDA_TRY(cudaGetLastError());
      uint32_t c[4];
      GT_CUDA_TRY(cudaMemcpyAsync(c, ctr, sizeof c, cudaMemcpyDeviceToHost, st));
      GT_CUDA_TRY(cudaStreamSynchronize(st));
      if (c[2]) return Err{GT_ERR_CUDA, "internal error: 8-wide collapse exceeded its node bound"};
      total = c[0];
      n_front = c[1];
      std::swap(fb, nb);
      std::swap(fn, nn);
    }
  }
  GT_CUDA_TRY(cudaMallocAsync(out8, (size_t)total * 16 * sizeof(float4), st));
  GT_CUDA_TRY(cudaMemcpyAsync(*out8, tmp, (size_t)total * 16 * sizeof(float4), cudaMemcpyDeviceToDevice, st));
  cudaFreeAsync(tmp, st);
  cudaFreeAsync(fb, st);
  cudaFreeAsync(fn, st);
  cudaFreeAsync(nb, st);
  cudaFreeAsync(nn, st);
  cudaFreeAsync(ctr, st);
  *n_nodes8 = total;
  return Err{};
}

// -------------------------------------------------------------- driver
// The scene's buffers come from the device's stream-ordered pool (which the
// context keeps from releasing), so a scene built after another was freed
// reuses its memory instead of mapping new pages.
void free_scene(SceneBuffers* b, cudaStream_t st) {
  for (void* p : {(void*)b->nodes, (void*)b->nodes8, (void*)b->w2o, (void*)b->leaf_pidx, (void*)b->shade,
                  (void*)b->sh, (void*)b->params})
    if (p) cudaFreeAsync(p, st);
  *b = SceneBuffers{};
}

static inline unsigned grid_for(uint64_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

Err build_scene(const void* packed_dev, uint64_t n, uint32_t stride, double alpha_min, cudaStream_t st,
                SceneBuffers* out, uint64_t* launches, bool fast_build, const double* act64) {
  SceneBuffers b;
  b.n_sh = std::min<uint32_t>(16u, (stride - 64u) / 16u);
  const uint8_t* packed = static_cast<const uint8_t*>(packed_dev);
  if (n == 0) {
    *out = b;
    return Err{};
  }
  if (n >= (1ull << 31)) return Err{GT_ERR_INVALID_ARG, "scene larger than 2^31 particles"};
  // shading records (every particle slot; only kept ones are written/read)
  GT_CUDA_TRY(cudaMallocAsync(&b.shade, n * 3 * sizeof(float4), st));
  GT_CUDA_TRY(cudaMallocAsync(&b.sh, n * 12 * sizeof(float4), st));
  GT_CUDA_TRY(cudaMallocAsync(&b.params, n * 2 * sizeof(float4), st));
  b.bytes += n * 17 * sizeof(float4);
  uint32_t *flags = nullptr, *slots = nullptr, *bounds = nullptr;
  GT_CUDA_TRY(cudaMallocAsync(&flags, n * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&slots, n * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&bounds, 8 * 4, st));
  const unsigned B = 256;
  k_keep_flags<<<grid_for(n, B), B, 0, st>>>(packed, n, stride, alpha_min, act64, flags);
  ++*launches;
  GT_CUDA_TRY(cudaGetLastError());
  Err e = scan_exclusive(flags, slots, n, st, launches);
  if (e.code != GT_OK) return e;
  uint32_t last_flag = 0, last_slot = 0;
  GT_CUDA_TRY(cudaMemcpyAsync(&last_flag, flags + (n - 1), 4, cudaMemcpyDeviceToHost, st));
  GT_CUDA_TRY(cudaMemcpyAsync(&last_slot, slots + (n - 1), 4, cudaMemcpyDeviceToHost, st));
  GT_CUDA_TRY(cudaStreamSynchronize(st));
  uint32_t m = last_slot + last_flag;
  b.n_kept = m;
  k_shade<<<grid_for(n, 128), 128, 0, st>>>(packed, n, stride, b.n_sh, flags, b.shade, b.sh, b.params);
  ++*launches;
  if (m == 0) {
    cudaFreeAsync(flags, st);
    cudaFreeAsync(slots, st);
    cudaFreeAsync(bounds, st);
    GT_CUDA_TRY(cudaStreamSynchronize(st));
    *out = b;
    return Err{};
  }
  float* box = nullptr;
  uint32_t *kept_pidx = nullptr, *keys = nullptr, *vals = nullptr;
  GT_CUDA_TRY(cudaMallocAsync(&box, (size_t)m * 6 * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&kept_pidx, (size_t)m * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&keys, (size_t)m * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&vals, (size_t)m * 4, st));
  {
    uint32_t init[8] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u, 0u, 0u};
    GT_CUDA_TRY(cudaMemcpyAsync(bounds, init, sizeof init, cudaMemcpyHostToDevice, st));
  }
  IcoVerts iv;
  ico_vertices(iv.v);
  k_proxy_boxes<<<grid_for(n, B), B, 0, st>>>(packed, n, stride, alpha_min, act64, flags, slots, iv, box, kept_pidx,
                                              bounds);
  ++*launches;
  k_morton<<<grid_for(m, B), B, 0, st>>>(box, m, bounds, keys, vals);
  ++*launches;
  GT_CUDA_TRY(cudaGetLastError());
  e = radix_sort(keys, vals, m, st, launches);
  if (e.code != GT_OK) return e;
  // scene records
  uint32_t n_int = m > 1 ? m - 1 : 0;
  GT_CUDA_TRY(cudaMallocAsync(&b.w2o, (size_t)m * 3 * sizeof(float4), st));
  GT_CUDA_TRY(cudaMallocAsync(&b.leaf_pidx, (size_t)m * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&b.nodes, (size_t)std::max<uint32_t>(n_int, 1) * 4 * sizeof(float4), st));
  b.bytes += (uint64_t)m * (3 * sizeof(float4) + 4) + (uint64_t)std::max<uint32_t>(n_int, 1) * 4 * sizeof(float4);
  float *leaf_box = nullptr, *ibox = nullptr;
  uint32_t *parent_int = nullptr, *parent_leaf = nullptr, *arrive = nullptr, *depth = nullptr;
  GT_CUDA_TRY(cudaMallocAsync(&leaf_box, (size_t)m * 6 * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&ibox, (size_t)std::max<uint32_t>(n_int, 1) * 6 * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&parent_int, (size_t)std::max<uint32_t>(n_int, 1) * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&parent_leaf, (size_t)m * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&arrive, (size_t)std::max<uint32_t>(n_int, 1) * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&depth, 4, st));
  GT_CUDA_TRY(cudaMemsetAsync(arrive, 0, (size_t)std::max<uint32_t>(n_int, 1) * 4, st));
  GT_CUDA_TRY(cudaMemsetAsync(depth, 0, 4, st));
  k_leaves<<<grid_for(m, B), B, 0, st>>>(packed, stride, alpha_min, act64, vals, m, kept_pidx, box, b.w2o, b.leaf_pidx,
                                          leaf_box);
  ++*launches;
  if (m > 1) {
    if (fast_build) {
      k_karras<<<grid_for(n_int, B), B, 0, st>>>(keys, (int)m, b.nodes, parent_int, parent_leaf);
      k_refit<<<grid_for(m, B), B, 0, st>>>(m, leaf_box, ibox, b.nodes, parent_int, parent_leaf, arrive);
      *launches += 2;
    } else {
      Err pe = build_ploc(leaf_box, m, st, b.nodes, ibox, parent_int, parent_leaf, launches);
      if (pe.code != GT_OK) return pe;
    }
    k_depth<<<grid_for(m, B), B, 0, st>>>(m, parent_int, parent_leaf, depth);
    *launches += 1;
    // structural check: refcount over [internal 0..m-2 | leaves 0..m-1]
    uint32_t* refc = nullptr;
    GT_CUDA_TRY(cudaMallocAsync(&refc, (size_t)(2 * m - 1) * 4, st));
    GT_CUDA_TRY(cudaMemsetAsync(refc, 0, (size_t)(2 * m - 1) * 4, st));
    GT_CUDA_TRY(cudaMemsetAsync(bounds + 7, 0, 4, st));
    k_check_children<<<grid_for(n_int, B), B, 0, st>>>(m, b.nodes, refc, bounds + 7);
    k_check_counts<<<grid_for(2 * m - 1, B), B, 0, st>>>(2 * m - 1, refc, bounds + 7);
    *launches += 2;
    cudaFreeAsync(refc, st);
    b.root = 0;
  } else {
    b.root = kLeafBit | 0u;
  }
  GT_CUDA_TRY(cudaGetLastError());
  {
    Err ce = collapse_bvh8(b.nodes, leaf_box, m, st, &b.nodes8, &b.n_nodes8, launches);
    if (ce.code != GT_OK) return ce;
    b.bytes += (uint64_t)b.n_nodes8 * 16 * sizeof(float4);
    // traversal reads only the 8-wide nodes: the binary hierarchy goes
    cudaFreeAsync(b.nodes, st);
    b.nodes = nullptr;
    b.bytes -= (uint64_t)std::max<uint32_t>(n_int, 1) * 4 * sizeof(float4);
  }
  float rb[6];
  uint32_t bo[8];
  GT_CUDA_TRY(cudaMemcpyAsync(rb, m > 1 ? ibox : leaf_box, sizeof rb, cudaMemcpyDeviceToHost, st));
  GT_CUDA_TRY(cudaMemcpyAsync(&b.depth, depth, 4, cudaMemcpyDeviceToHost, st));
  GT_CUDA_TRY(cudaMemcpyAsync(bo, bounds, sizeof bo, cudaMemcpyDeviceToHost, st));
  GT_CUDA_TRY(cudaStreamSynchronize(st));
  for (int a = 0; a < 6; ++a) b.bounds[a] = rb[a];
  float mag = 0.0f;
  for (int a = 0; a < 6; ++a) mag = std::max(mag, std::fabs(rb[a]));
  b.scene_mag = mag;
  cudaFreeAsync(flags, st);
  cudaFreeAsync(slots, st);
  cudaFreeAsync(bounds, st);
  cudaFreeAsync(box, st);
  cudaFreeAsync(kept_pidx, st);
  cudaFreeAsync(keys, st);
  cudaFreeAsync(vals, st);
  cudaFreeAsync(leaf_box, st);
  cudaFreeAsync(ibox, st);
  cudaFreeAsync(parent_int, st);
  cudaFreeAsync(parent_leaf, st);
  cudaFreeAsync(arrive, st);
  cudaFreeAsync(depth, st);
  GT_CUDA_TRY(cudaStreamSynchronize(st));
  if (bo[7] != 0) {
    free_scene(&b, st);
    return Err{GT_ERR_CUDA, "internal error: the built hierarchy is not a tree"};
  }
  if (b.depth > kMaxDepth) {
    free_scene(&b, st);
    return Err{GT_ERR_UNSUPPORTED, "BVH deeper than the traversal stack allows"};
  }
  *out = b;
  return Err{};
}

}  // namespace gt
