// gt_internal.cuh — shared declarations of the CUDA tracer library.
//
// Numerics contract.  The tracer follows one fixed IEEE-754 binary32
// operation order (the one the CPU oracle states in C): every product and
// sum is rounded separately (the library is compiled with -fmad=false and
// uses __f*_rn intrinsics where it matters), division and square root are
// correctly rounded, and exp is the deterministic Cody-Waite routine below.
// Hit t values, alphas and radiance are therefore bit-identical to the
// oracle's float build on the same inputs.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/gtrace.h"

namespace gt {

// ------------------------------------------------------------------ limits
constexpr uint32_t kMaxDepth = 120;        // deepest BVH the build accepts
constexpr uint32_t kInvalid = 0xFFFFFFFFu; // empty k-buffer slot (uint(-1))
constexpr uint32_t kLeafBit = 0x80000000u; // child reference: leaf flag
constexpr uint32_t kMaxRounds = 1u << 22;          // round cap per ray
constexpr int kWarpStack = 256;                    // traversal stack entries per warp

// device status word bits
constexpr uint32_t kStatusStackOverflow = 1u;
constexpr uint32_t kStatusVisitCap = 2u;
constexpr uint32_t kStatusRoundCap = 4u;
constexpr uint32_t kStatusCheckpointFull = 8u;
constexpr uint32_t kStatusHitOverflow = 16u;  // more hits on one proxy than a vertex allows

// Unit icosahedron face constants (src/main.ts:12-25): p0, e0 = p1 - p0,
// e1 = p0 - p2, n = cross(e1, e0), all in binary32 from the rounded
// vertices (webrtx/src/glsl/intersect.glsl:73-92 uses exactly these).
struct FaceTable {
  float p0[20][3];
  float e0[20][3];
  float e1[20][3];
  float n[20][3];
  float nmax;      // max |n| component over all faces
  float r_circ;    // circumradius of the vertex set
  float emax;      // max L1 norm of the edge vectors e0, e1
  float c[20];     // plane offsets n . p0 (pre-check only)
  int pa[10], pb[10];  // antipodal face pairs: n[pb[q]] == -n[pa[q]] bit for bit
  float pn[10][3];     // n[pa[q]], pair-major: the unrolled candidate pass reads them
  float pca[10], pcb[10];  // c[pa[q]], c[pb[q]]   at fixed parameter offsets
  int npairs;          // 10 (checked when the context is created)
  // Device loop limits of the trace kernels (this table is a kernel
  // parameter, so they cost no registers).  gt_set_limits lowers them to
  // exercise the failure path: a traversal past lim_steps steps, a stack
  // past lim_stack entries or a ray past lim_rounds rounds stops and sets a
  // status bit that the host turns into an error.
  uint32_t lim_steps;   // traversal steps per traversal (after 4 n_kept + 64)
  uint32_t lim_stack;   // stack entries per warp (<= kWarpStack)
  uint32_t lim_rounds;  // rounds per ray
};
void make_face_table(FaceTable* ft);

// Counters and status shared by the kernels of one call.
struct DevCounters {
  unsigned long long rays, rounds, entries, contributing, proxy_tests, node_visits, anyhits;
  unsigned long long ckpt_rounds;
  unsigned int status;
  unsigned int work;  // work-stealing tile counter
  unsigned int work2;    // the same for the second kernel of a launch
  unsigned int handoff;  // rays the tile-packet kernel handed to the warp-per-ray kernel
};

// Scene as the kernels see it.  Records of kept proxies are in BVH leaf
// order j; shading records are indexed by particle index p.
struct SceneDev {
  const float4* nodes8;     // 16 float4 per 8-wide node (see gt_build.cu)
  const float4* w2o;        // 3 float4 per leaf: world-to-object 4x3 column-major
  const uint32_t* leaf_pidx;// particle index of leaf j
  const float4* shade;      // 3 float4 per particle: (mu, opacity), (a00,a01,a02,a11), (a12,a22,-,-)
  const float4* sh;         // 12 float4 per particle: 16 RGB coefficients, tight
  const float4* params;     // 2 float4 per particle: (scale, 0), rotation (w, x, y, z)
  uint32_t root;            // root reference (kLeafBit | j for a one-proxy scene)
  uint32_t n_kept;
  uint32_t n_sh;            // coefficients present (16 for degree-3 data)
  float scene_mag;          // max |coordinate| of the proxy boxes (padding scale)
};

// Uniform block fields the kernels use (a copy of gt_uniforms, widened).
struct RayUniforms {
  float tw[16];
  float asp[2];
  float t_min, t_max, T_min, alpha_min;
  uint32_t k, deg, early_stop, debug;
  uint32_t frames;  // accumulated_frames
  uint32_t aa;      // 1: jittered pixel sample, blended into the previous image
};

inline RayUniforms to_ray_uniforms(const gt_uniforms& u) {
  RayUniforms r;
  for (int i = 0; i < 16; ++i) r.tw[i] = u.to_world[i];
  r.asp[0] = u.camera_aspect[0];
  r.asp[1] = u.camera_aspect[1];
  r.t_min = u.t_min;
  r.t_max = u.t_max;
  r.T_min = u.T_min;
  r.alpha_min = u.alpha_min;
  r.k = u.k;
  r.deg = u.sh_degree_max;
  r.early_stop = u.early_stop;
  r.debug = u.debug_mode;
  r.frames = u.accumulated_frames;
  r.aa = 0;
  return r;
}

// One view of a launch: image, output and work-tile range.
struct ViewDev {
  RayUniforms u;
  SceneDev s;
  float4* out;          // w*h pixels
  uint32_t w, h;
  uint32_t tiles_x;     // tiles per row
  uint32_t tile_begin;  // first global tile index of this view
  uint32_t n_tiles;
  uint32_t kbuf;        // k-buffer entries (k..128): a traversal keeps the kbuf closest hits
  uint32_t pkbuf;       // the tile-packet kernel's k-buffer entries per ray (k..64)
  uint32_t leaf_batch;  // queued leaves that trigger a batch of proxy tests (8..32)
  const float4* dL;     // backward: dL/drgba (w*h)
  float4* grad;         // backward: the scene's per-particle sums of the response terms (4 float4 a particle)
  float4* grad_sh;      // backward: this view's per-particle sums of the colour weights (1 float4 a particle)
  uint64_t n_particles;
  // this view's colour of every particle, max(0, SH(normalize(mu - camera)))
  // per channel (k_view_colours, before the trace launch), or null: the
  // trace kernels evaluate the SH per composited entry
  float4* rgb;
};

// Launch shape of the persistent trace kernel.
constexpr uint32_t kMaxKbuf = 128;  // up to four buffer entries per lane

struct LaunchShape {
  uint32_t block_threads = 128;
  uint32_t blocks_per_sm = 8;
  uint32_t tile_w = 8, tile_h = 4;  // pixel tile of the work order (tile_w*tile_h == 32)
  uint32_t kbuf = 64;               // k-buffer entries (raised to k when k is larger; <= kMaxKbuf)
  uint32_t leaf_batch = 32;         // leaf queue size that triggers proxy tests
  // Plain renders (debugMode 0, no checkpoint) run one warp per 8x4 tile of
  // rays (gt_packet.cu) when packet is 1, one warp per ray when it is 0, and
  // by default (2) the tile packets when the launch has at least
  // kPacketTilesPerSm tiles per SM.  The packet kernel's k-buffer has
  // packet_kbuf entries per ray (raised to k; <= kMaxPacketKbuf).
  uint32_t packet = 2;
  uint32_t packet_kbuf = 32;
  // A packet that has traced handoff_after times hands its rays that still
  // need hits to the warp-per-ray kernel (0: never), when the launch has a
  // handoff buffer.
  uint32_t handoff_after = 3;
};
constexpr uint32_t kMaxPacketKbuf = 64;
// A tile packet is a coarse work item: a few tiles whose rays have many
// hits take several times the mean, so with few tiles per resident warp (16
// warps an SM) their tail outweighs the packets' gain even with the handoff
// (1M-Gaussian view, ms as packets / a ray per warp, with the early handoff
// once every tile is taken: 480x270 (35 tiles an SM) 14.9 / 5.2; 640x360
// (52) 7.6 / 8.8; 800x450 (97) 9.7 / 13.7; 960x540 (109) 12.5 / 19.3).
constexpr uint32_t kPacketTilesPerSm = 48;

// ----------------------------------------------------------- host helpers
// Work slots of a w x h view: 32 per 8 x 4 tile of its tile grid, padded to
// whole blocks of 16 x 16 tiles (see tile_pixel).  A launch takes at most
// kMaxSlots of them (its 32-bit work counter counts past the total).
inline uint64_t view_slots(uint32_t w, uint32_t h) {
  const uint64_t tx = (((uint64_t)w + 7) / 8 + 15) / 16 * 16;
  const uint64_t ty = (((uint64_t)h + 3) / 4 + 15) / 16 * 16;
  return tx * ty * 32;
}
constexpr uint64_t kMaxSlots = 1ull << 31;

struct Err {
  gt_status code = GT_OK;
  std::string msg;
};

#define GT_CUDA_TRY(expr)                                                         \
  do {                                                                            \
    cudaError_t e_ = (expr);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      (void)cudaGetLastError(); /* clear it: the caller reports it once */        \
      return ::gt::Err{e_ == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA, \
                       std::string(#expr) + ": " + cudaGetErrorString(e_)};        \
    }                                                                             \
  } while (0)

// Scene build (gt_build.cu).
struct SceneBuffers {
  float4* nodes = nullptr;   // binary hierarchy: only during the build
  float4* nodes8 = nullptr;  // 8-wide nodes: 8 child records of 2 float4
  uint32_t n_nodes8 = 0;
  float4* w2o = nullptr;
  uint32_t* leaf_pidx = nullptr;
  float4* shade = nullptr;
  float4* sh = nullptr;
  float4* params = nullptr;  // per particle: (scale, 0), (w, x, y, z)
  uint32_t root = 0;
  uint64_t n_kept = 0;
  uint32_t depth = 0;
  uint32_t n_sh = 0;
  float bounds[6] = {0, 0, 0, 0, 0, 0};
  float scene_mag = 0;
  uint64_t bytes = 0;
};
// fast_build: Karras LBVH (a few ms for 1M proxies); otherwise PLOC
// clustering (slower to build, faster to trace).  act64 (device, optional):
// the activated values in double, 8 per particle (opacity, scale xyz,
// rotation wxyz), from which the proxies are then built, as the reference
// builds them from its JS numbers; shading always uses the packed records.
Err build_scene(const void* packed_dev, uint64_t n, uint32_t stride_bytes, double alpha_min,
                cudaStream_t stream, SceneBuffers* out, uint64_t* launches, bool fast_build = false,
                const double* act64 = nullptr);
// Binary hierarchy over m leaves in Morton order by PLOC (gt_ploc.cu): root 0,
// node format and parent links as the Karras build plus refit produce them.
Err build_ploc(const float* leaf_box, uint32_t m, cudaStream_t st, float4* nodes, float* ibox, uint32_t* parent_int,
               uint32_t* parent_leaf, uint64_t* launches);
// Exclusive prefix sum of n words (gt_build.cu).
Err scan_exclusive(const uint32_t* in, uint32_t* out, uint64_t n, cudaStream_t st, uint64_t* launches);
void free_scene(SceneBuffers* b, cudaStream_t st);

// Checkpoint written by the forward pass of gt_backward, in records from a
// shared pool; the records of a ray are linked from its last to its first,
// the order the adjoint walks them, so memory follows the work actually done.
// Record layout (uint32 words): [0] t_curr when the record opened (float
// bits), [1] T at that point (float bits), [2] previous record of the ray
// (kInvalid for the first), [3] number of entries, [4, 4 + kc) particle
// indices.
//   * checkpoint mode (kc > 0): a record holds the next kc contributing
//     entries of the ray in compositing order (alpha above alpha_min; the
//     others change neither T nor the colour), across round boundaries, and
//     [1] is the transmittance before its first entry.  The forward opens a
//     record when an entry contributes and the ray has none open or a full
//     one (warp-aggregated allocation);
//   * replay mode (kc == 0): one record per round ([0], [1] at the round's
//     start), the adjoint traces the round's entries again.
struct Ckpt {
  uint32_t* head = nullptr;       // [slots] last record of the ray, kInvalid if none
  uint32_t* pool = nullptr;       // [pool_cap][4 + kc]
  uint32_t* pool_next = nullptr;  // allocation counter (counts past pool_cap on overflow)
  uint32_t pool_cap = 0;          // records
  uint32_t kc = 0;                // particle indices stored per record (0: replay mode)
};
// contributing entries a checkpoint record holds (the adjoint's segment width)
constexpr uint32_t kCkptChunk = 16;
constexpr uint32_t kCkptHeader = 4;

// A ray that a tile packet hands over part way: its work slot (32 * tile +
// position in the tile) and its compositing state between two rounds.
struct HandoffRay {
  uint32_t item, step;
  float t_curr, T, L0, L1, L2;
  uint32_t ck_head;  // checkpointing launches: the ray's last record
  uint32_t ck_fill;  // entries in that record (checkpoint mode; kc when none is open)
};
// The handoff buffer of a launch (rays == nullptr: no handoff).
struct Handoff {
  HandoffRay* rays = nullptr;
  uint32_t cap = 0;
};

// Trace launches (gt_trace.cu).  launch_trace writes the shape's k-buffer
// size and leaf batch into the host view table before uploading it.
// Whether launch_trace renders these views with the tile-packet kernel.
bool packet_launch(const ViewDev* views, uint32_t n_views, uint32_t total_tiles, int num_sms,
                   const LaunchShape& shape, bool ckpt);
// Sets each view's k-buffer size and leaf batch for a launch of either kernel.
void apply_shape(ViewDev* views, uint32_t n_views, const LaunchShape& shape);
// Fills the colour table of every view that has one (ViewDev::rgb) from the
// device copy of the view table.
Err launch_view_colours(const ViewDev* views, const ViewDev* d_views, uint32_t n_views, int num_sms,
                        cudaStream_t stream, uint64_t* launches);
Err launch_trace(ViewDev* views, uint32_t n_views, uint32_t total_tiles, DevCounters* counters,
                 const FaceTable& faces, const LaunchShape& shape, int num_sms, cudaStream_t stream,
                 uint64_t* launches, ViewDev* d_views_scratch, const Ckpt* ckpt = nullptr,
                 const Handoff* handoff = nullptr);
Err launch_trace_packet(const ViewDev* views, const ViewDev* d_views, uint32_t n_views, uint32_t total_tiles,
                        DevCounters* counters, const FaceTable& faces, int num_sms, cudaStream_t stream,
                        uint64_t* launches, const Handoff& handoff, uint32_t handoff_after,
                        const Ckpt* ckpt = nullptr);
Err launch_trace_hits(const ViewDev& view, ViewDev* d_views, const uint32_t* pixels, uint32_t n_pix,
                      uint32_t max_entries, uint32_t* out_pidx, float* out_t, float* out_alpha, uint32_t* out_count,
                      uint32_t* out_rounds, float4* out_rgba, DevCounters* counters, const FaceTable& faces,
                      cudaStream_t stream, uint64_t* launches);
uint32_t kmax_for(uint32_t k);

}  // namespace gt
