// gt_ploc.cu — binary hierarchy by parallel locally-ordered clustering.
//
// PLOC (Meister and Bittner, "Parallel Locally-Ordered Clustering for
// Bounding Volume Hierarchy Construction", IEEE TVCG 2018): the clusters
// start as the proxies in Morton order; every iteration each cluster finds
// its nearest neighbour among the kPlocRadius clusters on either side (the
// distance is the surface area of the merged box), mutual nearest neighbours
// merge into a new internal node, and the cluster array is compacted in
// order.  The result replaces the Karras hierarchy in front of the 8-wide
// collapse; traversal visits fewer nodes and tests fewer proxies on it
// because merges follow surface area instead of Morton-code prefixes.
//
// Determinism: a tie in area is broken towards the smaller cluster index.
// For a fixed cluster i that is the lexicographic order of the pairs
// (area, min(i, j), max(i, j)), a strict total order, so the globally
// smallest pair is always mutual and every iteration merges at least once.
// Node indices come from prefix sums, so the tree and its layout are the
// same on every run.
#include <math_constants.h>

#include <algorithm>

#include "gt_internal.cuh"

namespace gt {

constexpr int kPlocRadius = 16;
constexpr int kPlocBlock = 256;

// Cluster record: c0 = (lo.x, lo.y, lo.z, hi.x), c1 = (hi.y, hi.z, ref, 0);
// ref = kLeafBit | leaf or an internal node index.
struct PlocCluster {
  float4 c0, c1;
};

__device__ __forceinline__ float merged_half_area(float ax0, float ay0, float az0, float ax1, float ay1, float az1,
                                                  float bx0, float by0, float bz0, float bx1, float by1, float bz1) {
  const float x = fmaxf(ax1, bx1) - fminf(ax0, bx0);
  const float y = fmaxf(ay1, by1) - fminf(ay0, by0);
  const float z = fmaxf(az1, bz1) - fminf(az0, bz0);
  return x * y + y * z + z * x;
}

__global__ void k_ploc_init(const float* leaf_box, uint32_t m, PlocCluster* c) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const float* b = leaf_box + 6 * (size_t)j;
  c[j].c0 = make_float4(b[0], b[1], b[2], b[3]);
  c[j].c1 = make_float4(b[4], b[5], __uint_as_float(kLeafBit | j), 0.f);
}

// Nearest neighbour of every cluster within the window; boxes of the block's
// clusters and both halos are staged in shared memory (structure of arrays).
__global__ void __launch_bounds__(kPlocBlock) k_ploc_nn(const PlocCluster* __restrict__ c, uint32_t n,
                                                        uint32_t* __restrict__ nn) {
  constexpr int kSpan = kPlocBlock + 2 * kPlocRadius;
  __shared__ float sb[6][kSpan];
  const int base = (int)(blockIdx.x * kPlocBlock) - kPlocRadius;
  for (int s = threadIdx.x; s < kSpan; s += kPlocBlock) {
    const int g = base + s;
    if (g >= 0 && g < (int)n) {
      const float4 a = c[g].c0, b = c[g].c1;
      sb[0][s] = a.x;
      sb[1][s] = a.y;
      sb[2][s] = a.z;
      sb[3][s] = a.w;
      sb[4][s] = b.x;
      sb[5][s] = b.y;
    }
  }
  __syncthreads();
  const int i = (int)(blockIdx.x * kPlocBlock + threadIdx.x);
  if (i >= (int)n) return;
  const int si = i - base;
  const float x0 = sb[0][si], y0 = sb[1][si], z0 = sb[2][si], x1 = sb[3][si], y1 = sb[4][si], z1 = sb[5][si];
  float best = CUDART_INF_F;
  int bj = -1;
  const int lo = max(0, i - kPlocRadius), hi = min((int)n - 1, i + kPlocRadius);
  for (int j = lo; j <= hi; ++j) {  // ascending j: a tie keeps the smaller index
    if (j == i) continue;
    const int s = j - base;
    const float a = merged_half_area(x0, y0, z0, x1, y1, z1, sb[0][s], sb[1][s], sb[2][s], sb[3][s], sb[4][s],
                                     sb[5][s]);
    if (a < best || bj < 0) {
      best = a;
      bj = j;
    }
  }
  nn[i] = bj < 0 ? kInvalid : (uint32_t)bj;
}

// valid: the cluster survives the iteration (merged pairs survive at the
// smaller index); merge: it is the smaller index of a mutual pair.
__global__ void k_ploc_flags(const uint32_t* __restrict__ nn, uint32_t n, uint32_t* valid, uint32_t* merge) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = nn[i];
  const bool mutual = j != kInvalid && nn[j] == i;
  valid[i] = (mutual && j < i) ? 0u : 1u;
  merge[i] = (mutual && i < j) ? 1u : 0u;
}

__global__ void k_ploc_write(const PlocCluster* __restrict__ cin, const uint32_t* __restrict__ nn,
                             const uint32_t* __restrict__ valid, const uint32_t* __restrict__ merge,
                             const uint32_t* __restrict__ vpos, const uint32_t* __restrict__ mpos, uint32_t n,
                             uint32_t next_id, PlocCluster* __restrict__ cout, float4* nodes, float* ibox,
                             uint32_t* parent_int, uint32_t* parent_leaf) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !valid[i]) return;
  const uint32_t p = vpos[i];
  if (!merge[i]) {
    cout[p] = cin[i];
    return;
  }
  const uint32_t id = next_id - mpos[i];
  const PlocCluster a = cin[i], b = cin[nn[i]];
  const uint32_t ra = __float_as_uint(a.c1.z), rb = __float_as_uint(b.c1.z);
  // binary node: child boxes as (lo.x, hi.x, lo.y, hi.y) x 2, (lo.z, hi.z) x 2, refs
  nodes[4 * (size_t)id + 0] = make_float4(a.c0.x, a.c0.w, a.c0.y, a.c1.x);
  nodes[4 * (size_t)id + 1] = make_float4(b.c0.x, b.c0.w, b.c0.y, b.c1.x);
  nodes[4 * (size_t)id + 2] = make_float4(a.c0.z, a.c1.y, b.c0.z, b.c1.y);
  nodes[4 * (size_t)id + 3] = make_float4(__uint_as_float(ra), __uint_as_float(rb), 0.f, 0.f);
  const float u[6] = {fminf(a.c0.x, b.c0.x), fminf(a.c0.y, b.c0.y), fminf(a.c0.z, b.c0.z),
                      fmaxf(a.c0.w, b.c0.w), fmaxf(a.c1.x, b.c1.x), fmaxf(a.c1.y, b.c1.y)};
#pragma unroll
  for (int q = 0; q < 6; ++q) ibox[6 * (size_t)id + q] = u[q];
  if (ra & kLeafBit) parent_leaf[ra & ~kLeafBit] = id; else parent_int[ra] = id;
  if (rb & kLeafBit) parent_leaf[rb & ~kLeafBit] = id; else parent_int[rb] = id;
  if (id == 0) parent_int[0] = kInvalid;
  cout[p].c0 = make_float4(u[0], u[1], u[2], u[3]);
  cout[p].c1 = make_float4(u[4], u[5], __uint_as_float(id), 0.f);
}

static inline unsigned ploc_grid(uint64_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

Err build_ploc(const float* leaf_box, uint32_t m, cudaStream_t st, float4* nodes, float* ibox, uint32_t* parent_int,
               uint32_t* parent_leaf, uint64_t* launches) {
  if (m < 2) return Err{};
  PlocCluster *ca = nullptr, *cb = nullptr;
  uint32_t *nn = nullptr, *valid = nullptr, *merge = nullptr, *vpos = nullptr, *mpos = nullptr;
  GT_CUDA_TRY(cudaMallocAsync(&ca, (size_t)m * sizeof(PlocCluster), st));
  GT_CUDA_TRY(cudaMallocAsync(&cb, (size_t)m * sizeof(PlocCluster), st));
  GT_CUDA_TRY(cudaMallocAsync(&nn, (size_t)m * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&valid, (size_t)m * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&merge, (size_t)m * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&vpos, (size_t)m * 4, st));
  GT_CUDA_TRY(cudaMallocAsync(&mpos, (size_t)m * 4, st));
  auto release = [&]() {
    cudaFreeAsync(ca, st);
    cudaFreeAsync(cb, st);
    cudaFreeAsync(nn, st);
    cudaFreeAsync(valid, st);
    cudaFreeAsync(merge, st);
    cudaFreeAsync(vpos, st);
    cudaFreeAsync(mpos, st);
  };
  k_ploc_init<<<ploc_grid(m, 256), 256, 0, st>>>(leaf_box, m, ca);
  ++*launches;
  uint32_t n = m, next_id = m - 2;
  // every iteration merges at least one pair, so m - 1 iterations bound it
  for (uint32_t it = 0; n > 1 && it < m; ++it) {
    k_ploc_nn<<<ploc_grid(n, kPlocBlock), kPlocBlock, 0, st>>>(ca, n, nn);
    k_ploc_flags<<<ploc_grid(n, 256), 256, 0, st>>>(nn, n, valid, merge);
    *launches += 2;
    Err e = scan_exclusive(valid, vpos, n, st, launches);
    if (e.code == GT_OK) e = scan_exclusive(merge, mpos, n, st, launches);
    if (e.code != GT_OK) {
      release();
      return e;
    }
    uint32_t tail[4];
    GT_CUDA_TRY(cudaMemcpyAsync(&tail[0], valid + (n - 1), 4, cudaMemcpyDeviceToHost, st));
    GT_CUDA_TRY(cudaMemcpyAsync(&tail[1], vpos + (n - 1), 4, cudaMemcpyDeviceToHost, st));
    GT_CUDA_TRY(cudaMemcpyAsync(&tail[2], merge + (n - 1), 4, cudaMemcpyDeviceToHost, st));
    GT_CUDA_TRY(cudaMemcpyAsync(&tail[3], mpos + (n - 1), 4, cudaMemcpyDeviceToHost, st));
    GT_CUDA_TRY(cudaStreamSynchronize(st));
    const uint32_t n_next = tail[0] + tail[1], merges = tail[2] + tail[3];
    if (merges == 0 || merges > next_id + 1 || n_next != n - merges) {
      release();
      return Err{GT_ERR_CUDA, "internal error: clustering made no progress"};
    }
    k_ploc_write<<<ploc_grid(n, 256), 256, 0, st>>>(ca, nn, valid, merge, vpos, mpos, n, next_id, cb, nodes, ibox,
                                                    parent_int, parent_leaf);
    ++*launches;
    GT_CUDA_TRY(cudaGetLastError());
    std::swap(ca, cb);
    n = n_next;
    next_id -= merges;  // wraps past zero after the root: n is then 1
  }
  release();
  if (n != 1) return Err{GT_ERR_CUDA, "internal error: clustering did not finish"};
  return Err{};
}

}  // namespace gt
