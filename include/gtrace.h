/*
 * gtrace.h — C ABI of the B200-native Gaussian ray tracer.
 *
 * The reference (DeepGPU/WebGPU-GaussianTracer) renders through the WebRTX
 * emulation of the Vulkan ray-tracing API on WebGPU:
 *
 *   device.createRayTracingAccelerationContainer(tlasDesc)       webrtx/src/patch.ts:211-213
 *   device.hostBuildRayTracingAccelerationContainer(tlas)        webrtx/src/patch.ts:216-219
 *   passEncoder.traceRays(device, sbt, width, height)            webrtx/src/pass_encoder.ts:35-65
 *
 * with the bind group of src/main.ts:497-512 (binding 0 = TLAS, 1 = RGBA-f32
 * pixel buffer, 2 = packed particle buffer, 3 = 112-byte uniform block).
 * This header replaces that call chain with plain C: a scene handle built on
 * the GPU from the same packed particle buffer, and one render call that
 * takes the same uniform block and writes the same pixel buffer.
 *
 * Conventions
 *   - Every entry point returns a gt_status; GT_OK is 0.  No entry point
 *     aborts, traps or throws.  gt_last_error() gives a one-line message for
 *     the last failing call on a context.
 *   - The caller owns every buffer it passes.  The library never keeps a
 *     caller pointer after the call returns.  Context and scene handles are
 *     opaque and owned by the library.
 *   - A pointer is a host pointer unless the matching GT_*_DEVICE flag is set,
 *     in which case it is a device pointer on the context's GPU.
 *   - One context owns one CUDA stream.  Calls on one context must be
 *     serialised by the caller; different contexts are independent.
 *   - Calls are synchronous unless GT_FLAG_ASYNC is given (device buffers
 *     only); an asynchronous call returns once its work is queued.
 */
#ifndef GTRACE_H
#define GTRACE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GT_ABI_VERSION 2u

/* ---------------------------------------------------------------- status */
typedef int32_t gt_status;
enum {
  GT_OK = 0,
  GT_ERR_INVALID_ARG = 1,     /* bad pointer, size, k, stride ...            */
  GT_ERR_OOM = 2,             /* device or host allocation failed            */
  GT_ERR_CUDA = 3,            /* a CUDA runtime call failed                  */
  GT_ERR_DEVICE_TIMEOUT = 4,  /* a device loop hit its iteration limit       */
  GT_ERR_STACK_OVERFLOW = 5,  /* traversal stack overflowed (status word)    */
  GT_ERR_UNSUPPORTED = 6,     /* valid request this build does not support  */
  GT_ERR_NO_DEVICE = 7        /* no CUDA device, or the ordinal is invalid   */
};

/* ----------------------------------------------------------------- flags */
#define GT_FLAG_INPUT_DEVICE   0x1u  /* input buffers are device pointers     */
#define GT_FLAG_OUTPUT_DEVICE  0x2u  /* output buffers are device pointers    */
#define GT_FLAG_ASYNC          0x4u  /* do not wait (device buffers only)     */
#define GT_FLAG_ACCUMULATE     0x8u  /* backward: add into dL_dparams         */
#define GT_FLAG_CHECKPOINT     0x10u /* render: keep the round checkpoint in the context;
                                        backward: reuse it when the views match  */
#define GT_FLAG_FAST_BUILD     0x20u /* scene: Morton-prefix (LBVH) hierarchy instead
                                        of surface-area clustering: builds faster,
                                        traces slower (scenes rebuilt every step) */
#define GT_FLAG_ANTIALIAS      0x40u /* render: progressive anti-aliasing, the
                                        reference's `antialiasing` path
                                        (src/GS_shader.ts:54,281-308, a constant
                                        false there): one jittered sample per pixel,
                                        seeded by (pixel, u.accumulated_frames) and
                                        blended into the previous contents of
                                        out_rgba (replaced when frames == 0) */

/* -------------------------------------------------------- opaque handles */
typedef struct gt_context gt_context;
typedef struct gt_scene gt_scene;

/* ------------------------------------------------------ uniform block
 * Byte-identical to the reference's 112-byte `rtUniforms` block
 * (src/GS_shader.ts:96-108), packed by src/main.ts:516-534. */
typedef struct gt_uniforms {
  float to_world[16];          /*   0  camera matrix, column-major: right, up, back, position */
  float camera_aspect[2];      /*  64  tan(hfov/2), tan(hfov/2) * height / width            */
  float t_min;                 /*  72                                                       */
  float t_max;                 /*  76                                                       */
  float T_min;                 /*  80  transmittance cutoff                                 */
  float alpha_min;             /*  84  compositing threshold                                */
  uint32_t k;                  /*  88  hit_array_size: hits collected per round (1..32)     */
  uint32_t sh_degree_max;      /*  92  0..3                                                 */
  uint32_t accumulated_frames; /*  96  progressive-average frame index                      */
  uint32_t early_stop;         /* 100  stop before round `early_stop`; 0xFFFFFFFF = off      */
  uint32_t debug_mode;         /* 104  0 = render, 1 = proxy view, 2 = any-hit count        */
  uint32_t _pad;               /* 108                                                       */
} gt_uniforms;

/* Per-particle record of the packed buffer: the std430 `GaussianParticle`
 * (src/GS_shader.ts:78-89, packed by src/GS_ply.ts:199-252): position vec3 @0,
 * scale vec3 @16, rotation (w,x,y,z) vec4 @32, opacity f32 @48, sh vec3[16]
 * (array stride 16) @64.  320 bytes for SH degree 3. */
#define GT_PARTICLE_STRIDE 320u
#define GT_PARAMS_PER_PARTICLE 59u   /* 3 pos + 3 scale + 4 rot + 1 opacity + 48 sh */

/* ----------------------------------------------------------- statistics */
typedef struct gt_render_stats {
  float kernel_ms;        /* device time of the trace kernel (CUDA events)        */
  float total_ms;         /* device time of the whole call, copies included       */
  uint64_t rays;          /* primary rays traced                                  */
  uint64_t rounds;        /* traversal rounds, summed over rays                   */
  uint64_t entries;       /* valid hit entries composited (any alpha)             */
  uint64_t contributing;  /* entries with alpha > alpha_min                       */
  uint64_t proxy_tests;   /* ray-proxy tests                                      */
  uint64_t node_visits;   /* BVH nodes popped                                     */
  uint64_t anyhits;       /* front-face proxy hits offered to the k-buffer         */
  uint32_t status_flags;  /* device status word (0 = clean)                       */
  uint32_t handed;        /* rays that reached the tile packets' traversal limit: the
                             warp-per-ray kernel finishes those that fit the handoff
                             buffer (a quarter of the launch's rays), the packets the
                             rest (0 when the warp-per-ray kernel traced the views)   */
} gt_render_stats;

typedef struct gt_scene_info {
  uint64_t n_particles;   /* particles in the packed buffer                       */
  uint64_t n_kept;        /* particles with opacity > alpha_min (proxies)         */
  uint64_t device_bytes;  /* device memory held by the scene                      */
  uint32_t bvh_depth;     /* deepest leaf                                         */
  uint32_t _pad;
  float build_ms;         /* device time of the GPU build                         */
  float bounds[6];        /* world AABB of the proxies: min xyz, max xyz          */
  float upload_ms;        /* host time of the host-to-device copy of the records  */
} gt_scene_info;

/* ============================================================ context */

/* Library version (GT_ABI_VERSION of the built library). */
uint32_t gt_version(void);

/* Creates a context on CUDA device `device`.  Replaces the adapter/device
 * request of src/main.ts:396-427.  Besides its scenes, a context keeps the
 * scratch of its largest call so far: staging images, the hand-off buffer,
 * checkpoints, and the colour tables of plain renders (16 bytes per
 * particle per view of a call, at most 2 GiB; each particle's SH colour as
 * seen from the view's camera, computed once per call before tracing). */
gt_status gt_context_create(int device, gt_context** out);
/* Destroys the context and every scene still alive on it (their handles
 * become invalid). */
gt_status gt_context_destroy(gt_context* ctx);

/* Copies the last error message of `ctx` (NUL-terminated, truncated to
 * `len`).  With ctx == NULL it reports the last context-less error (for
 * example a failed gt_context_create). */
gt_status gt_last_error(const gt_context* ctx, char* buf, size_t len);

/* ============================================================== scene */

/* Builds a scene from the packed particle buffer.
 * Replaces gaussianSceneToBvh (src/main.ts:30-111) together with
 * createRayTracingAccelerationContainer/hostBuildRayTracingAccelerationContainer
 * (webrtx/src/patch.ts:211-219 → webrtx/src/wasm_bvh_builder.ts:260-377 →
 * webrtx/bvh/src/lib.rs:254-347, 512-603) and the shader binding table of
 * src/main.ts:335-393.
 *   packed        n records of `stride_bytes` (>= 320) in the layout above,
 *                 already activated (scale = exp, unit quaternion, sigmoid
 *                 opacity), exactly what PackedGaussians.gaussiansBuffer holds
 *   alpha_min     proxy cut: particle i gets a proxy iff opacity > alpha_min;
 *                 its icosahedron is scaled by sqrt(2 ln(opacity/alpha_min))
 *                 (src/main.ts:79-87).  A double, like the JS number it replaces.
 *   flags         GT_FLAG_INPUT_DEVICE if `packed` is a device pointer,
 *                 GT_FLAG_FAST_BUILD for the Karras LBVH hierarchy
 * The build (proxy transforms, Morton codes, radix sort, binary hierarchy by
 * PLOC clustering or LBVH, 8-wide collapse) runs on the GPU.  Any hierarchy
 * gives the same images: only the traversal cost differs.  n == 0 gives an
 * empty scene that renders black. */
gt_status gt_scene_create(gt_context* ctx, const void* packed, uint64_t n,
                          uint32_t stride_bytes, double alpha_min,
                          uint32_t flags, gt_scene** out);
/* gt_scene_create with the activated values in double precision beside the
 * packed records: `activated` holds 8 doubles per particle, opacity, scale
 * x y z, rotation w x y z, exactly the numbers of gaussianData
 * (src/GS_ply.ts:225-235) that the reference builds its proxies from
 * (src/main.ts:72-94: the opacity cut, s = sqrt(2 ln(o / alpha_min)), the
 * rotation and the scale).  The proxies are then built from them, as the
 * reference's are; shading still reads the packed binary32 records, as the
 * reference's shader does.  NULL gives gt_scene_create.  A host pointer
 * unless GT_FLAG_INPUT_DEVICE (then both buffers are device pointers). */
gt_status gt_scene_create_ex(gt_context* ctx, const void* packed, uint64_t n, uint32_t stride_bytes,
                             double alpha_min, const double* activated, uint32_t flags, gt_scene** out);
gt_status gt_scene_destroy(gt_scene* scene);
gt_status gt_scene_get_info(const gt_scene* scene, gt_scene_info* info);

/* Inspection of the built hierarchy (no counterpart in the reference; the
 * tests check its invariants with it).  Host copies of the 8-wide nodes:
 * n_nodes8 records of 8 children x 2 float4, child c of node i at floats
 * 64 i + 8 c: (lo.x, lo.y, lo.z, hi.x), (hi.y, hi.z, ref, 0) with ref (as
 * uint32 bits) = 0x80000000 | leaf j, a node index, or 0xFFFFFFFF for an
 * empty slot; and the particle index of every leaf j.  The root is node 0,
 * or the leaf reference `root` of a one-proxy scene.  Either buffer may be
 * NULL. */
typedef struct gt_bvh_info {
  uint32_t n_nodes8;
  uint32_t n_leaves;      /* proxies (particles with opacity > alpha_min) */
  uint32_t root;
  uint32_t depth;         /* deepest leaf of the binary hierarchy */
} gt_bvh_info;
gt_status gt_scene_export_bvh(const gt_scene* scene, void* nodes8, uint64_t nodes_bytes, uint32_t* leaf_pidx,
                              uint64_t leaf_count, gt_bvh_info* info);

/* ========================================================= PLY ingest
 * Native replacement of PackedGaussians (src/GS_ply.ts:39-253): the 3DGS
 * PLY header is decoded on the host with the reference loader's rules
 * (decodeHeader :58-111, readRawVertex :113-132: 50-byte header chunks,
 * "element vertex" count, "property <type> <name>" in JavaScript object-key
 * order, float and uchar properties read, others skipped), and the vertex
 * rows are activated (:225-235: scale = exp, quaternion / its norm,
 * opacity = sigmoid, in double) and packed into the 320-byte std430 records
 * (:199-207; 64 + 16 (deg+1)^2 bytes for lower SH degrees) on the GPU.
 * The header must be ASCII.  A missing float/uchar property, an SH degree
 * outside 0..3 or a body shorter than the header says is GT_ERR_INVALID_ARG
 * (the reference packs NaN or throws a RangeError there).  The PLY buffer is
 * always a host buffer. */
typedef struct gt_ply_info {
  uint64_t n_vertices;    /* "element vertex" count                              */
  uint64_t data_offset;   /* byte offset of the vertex data (one past end_header) */
  uint32_t sh_degree;     /* 0..3, from the number of f_rest_* properties         */
  uint32_t record_stride; /* bytes per packed record: 64 + 16 (sh_degree+1)^2     */
  uint32_t row_bytes;     /* bytes per vertex row as the reference reads it       */
  uint32_t n_properties;  /* distinct property names in the header                */
  float ingest_ms;        /* device time of upload + activation/packing           */
  uint32_t _pad;
} gt_ply_info;

/* Decodes the header only (host, no device work).  Errors are reported by
 * gt_last_error(NULL, ...). */
gt_status gt_ply_parse_header(const void* ply, uint64_t len, gt_ply_info* info);
/* Writes PackedGaussians.gaussiansBuffer: n_vertices * record_stride bytes
 * into out_packed (host, or device with GT_FLAG_OUTPUT_DEVICE, 16-byte
 * aligned); out_bytes is its capacity. */
gt_status gt_ply_pack(gt_context* ctx, const void* ply, uint64_t len, void* out_packed,
                      uint64_t out_bytes, uint32_t flags, gt_ply_info* info);
/* loadGaussianSplatting + PackedGaussians + gaussianSceneToBvh in one call:
 * the packed records never leave the device.  flags: GT_FLAG_FAST_BUILD. */
gt_status gt_scene_create_from_ply(gt_context* ctx, const void* ply, uint64_t len, double alpha_min,
                                   uint32_t flags, gt_scene** out, gt_ply_info* info);
/* The same from a file path (read with stdio). */
gt_status gt_scene_create_from_ply_file(gt_context* ctx, const char* path, double alpha_min,
                                        uint32_t flags, gt_scene** out, gt_ply_info* info);

/* ============================================================= render */

/* Renders one view.  Replaces traceRays (webrtx/src/pass_encoder.ts:35-65),
 * i.e. one invocation of the ray-generation shader per pixel
 * (src/GS_shader.ts:275-309) with its tracePath rounds (:192-273), any-hit
 * k-buffer (:323-367) and compositing.
 *   u          the 112-byte uniform block (debug_mode 0, 1 and 2 are supported)
 *   w, h       image size; any value >= 1 (the reference needs multiples of 8)
 *   out_rgba   w*h*4 floats, pixel (x, y) at index 4*(w*y + x); RGB = radiance,
 *              A = 1 (src/GS_shader.ts:300-301).  A host buffer that is
 *              page-locked for this GPU (gt_host_alloc, cudaHostAlloc,
 *              cudaMallocHost, cudaHostRegister) is written by the kernels
 *              directly, tile by tile; any other host buffer receives one copy
 *              after the render
 *   flags      GT_FLAG_OUTPUT_DEVICE, GT_FLAG_ASYNC, GT_FLAG_ANTIALIAS (out_rgba
 *              then also holds the running average of the earlier frames),
 *              GT_FLAG_CHECKPOINT (not with GT_FLAG_ANTIALIAS)
 *   stats      optional (NULL allowed); not filled for asynchronous calls */
gt_status gt_render(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u,
                    uint32_t w, uint32_t h, float* out_rgba, uint32_t flags,
                    gt_render_stats* stats);

/* Parity/inspection variant of gt_render: for the `n_pix` pixel indices
 * (w*y + x) in `pixels` it records the composited hit sequence, in the order
 * entries were composited: particle index, hit t and alpha of each valid
 * k-buffer entry (src/GS_shader.ts:250-269), at most `max_entries` per pixel.
 * out_count[i] is the full number of valid entries of pixel i (it may exceed
 * max_entries; only the first max_entries are stored).  out_rounds[i] is the
 * number of traversal rounds.  out_rgba (4 floats per listed pixel) may be
 * NULL.  All buffers are host buffers. */
gt_status gt_render_hits(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u,
                         uint32_t w, uint32_t h, const uint32_t* pixels, uint32_t n_pix,
                         uint32_t max_entries, uint32_t* out_pidx, float* out_t,
                         float* out_alpha, uint32_t* out_count, uint32_t* out_rounds,
                         float* out_rgba);

/* ============================================================ display
 * The reference's tone-map render pass (src/toneMapper.ts:15-24, a full-screen
 * fragment shader into an 8-bit swap-chain texture) as a headless RGBA8
 * buffer: byte 4i..4i+3 = R, G, B, 255 of pixel i, each channel clamped to
 * [0, 1] and rounded from c * 255 (unorm8).  exposure is 1.66 in the
 * reference.  exp and the 1/2.2 power use this library's deterministic
 * routines, so the bytes are reproducible. */
#define GT_TONEMAP_HDR            0u /* the shader's active line: vec4(hdr, 1)          */
#define GT_TONEMAP_EXPOSURE       1u /* 1 - exp(-exposure hdr)                          */
#define GT_TONEMAP_EXPOSURE_GAMMA 2u /* (1 - exp(-exposure hdr))^(1/2.2), the commented  */
                                     /* gamma line                                       */
/* rgba: n_pixels * 4 floats (host, or device with GT_FLAG_INPUT_DEVICE,
 * 16-byte aligned); out_rgba8: n_pixels * 4 bytes (host, or device with
 * GT_FLAG_OUTPUT_DEVICE, 4-byte aligned).  GT_FLAG_ASYNC needs both on the
 * device. */
gt_status gt_tonemap(gt_context* ctx, const float* rgba, uint64_t n_pixels, uint32_t mode, float exposure,
                     uint8_t* out_rgba8, uint32_t flags);

/* ============================================================ backward
 * No counterpart in the reference (it has no training path, README.md:69). */
typedef struct gt_bwd_opts {
  uint32_t mode;          /* 0 = auto (checkpoint if it fits), 1 = checkpoint, 2 = replay */
  uint32_t max_rounds;    /* in: expected records per ray, sizes the first checkpoint pool
                             (0 = the previous call's count, else 4); the pool grows to
                             the records actually written.  A record holds up to 16
                             contributing entries of a ray (checkpoint mode) or one
                             round (replay mode).  out: records used                  */
  uint64_t mem_budget;    /* bytes the checkpoint may use (0 = 1/2 of free device memory),
                             and the adjoint's per-view colour sums (16 bytes a particle
                             a view; 0 = 1/4 of free memory): views whose sums do not fit
                             together run in successive adjoint launches               */
  uint32_t used_mode;     /* out: 1 = checkpoint, 2 = replay                              */
  uint32_t _pad;
  float fwd_ms;           /* out: device time of the forward (checkpointing) pass         */
  float bwd_ms;           /* out: device time of the adjoint pass                         */
} gt_bwd_opts;

/* Gradient of a loss with respect to every particle parameter, given the
 * gradient with respect to the rendered RGBA image.
 *   dL_drgba     w*h*4 floats (the A channel is ignored: the rendered A is 1)
 *   dL_dparams   59 * n floats, parameter-major (SoA): row p holds parameter p
 *                of every particle.  Rows: 0-2 position, 3-5 scale,
 *                6-9 rotation (w,x,y,z as stored), 10 opacity, 11-58 sh
 *                (coefficient c, channel ch at row 11 + 3*c + ch).  Particles
 *                without a proxy get 0.  Overwritten unless GT_FLAG_ACCUMULATE.
 *   flags        GT_FLAG_INPUT_DEVICE (dL_drgba), GT_FLAG_OUTPUT_DEVICE
 *                (dL_dparams), GT_FLAG_ACCUMULATE, GT_FLAG_CHECKPOINT (skip the
 *                checkpointing forward when the last gt_render/gt_render_batch
 *                call with GT_FLAG_CHECKPOINT rendered exactly these views)
 * Hit sets are held fixed (the proxy geometry is piecewise constant); the
 * response, opacity, SH colour and compositing are differentiated exactly. */
gt_status gt_backward(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u,
                      uint32_t w, uint32_t h, const float* dL_drgba,
                      float* dL_dparams, uint32_t flags, gt_bwd_opts* opts,
                      gt_render_stats* stats);

/* ============================================================= batches
 * No counterpart in the reference.  Many views of several scenes, traced by
 * one persistent kernel launch (captured in a CUDA graph and replayed when
 * the batch shape repeats). */
typedef struct gt_batch_item {
  const gt_scene* scene;
  gt_uniforms u;          /* per-view uniform block (its k is used)            */
  uint32_t w, h;
  float* out_rgba;        /* w*h*4 floats; host unless GT_FLAG_OUTPUT_DEVICE  */
  const float* dL_drgba;  /* backward batches only                              */
} gt_batch_item;

gt_status gt_render_batch(gt_context* ctx, const gt_batch_item* items, uint32_t count,
                          uint32_t flags, gt_render_stats* stats);

/* Renders a batch exactly like gt_render_batch but allocates no memory.
 * For callers that cannot allocate while they render: a frame loop that must
 * never stall on cudaMalloc/cudaFree (both synchronise the whole device), or
 * a process whose GPU memory is owned and capped by another allocator.
 * No counterpart in the reference.
 *   - outputs must be device buffers: GT_FLAG_OUTPUT_DEVICE is required
 *     (host outputs would need a staging allocation); GT_FLAG_ANTIALIAS
 *     blends into them as in gt_render_batch; GT_FLAG_CHECKPOINT is
 *     rejected (the checkpoint records would need an allocation);
 *   - stats (optional) carries the counters and the kernel and call times;
 *   - at most 256 views per call; larger counts are rejected with
 *     GT_ERR_INVALID_ARG;
 *   - the launch's scratch (tile counter, statistics, device view table,
 *     about 60 KB) lives in one fixed array in the library's device image;
 *     every GPU that loads the library holds a copy until the process exits;
 *   - the first call on a device looks up that array's address (do it before
 *     any stream capture);
 *   - all calls on a device share the array and it keeps the last call's
 *     contents: calls whose GPU work overlaps (other contexts or streams on
 *     the same device) race; calls on one context are stream-ordered. */
gt_status gt_render_batch_noalloc(gt_context* ctx, const gt_batch_item* items, uint32_t count,
                                  uint32_t flags, gt_render_stats* stats);

/* Accumulates, per scene, the gradients of all its views in one launch.
 * dL_dparams[s] receives the sum over the items whose scene is scenes[s]. */
gt_status gt_backward_batch(gt_context* ctx, const gt_batch_item* items, uint32_t count,
                            const gt_scene* const* scenes, float* const* dL_dparams,
                            uint32_t n_scenes, uint32_t flags, gt_bwd_opts* opts,
                            gt_render_stats* stats);

/* L2 image loss for the differentiable path: loss = sum over pixels of
 * |rgb - target_rgb|^2 (A ignored), dL_drgba = 2 (rgb - target), A = 0.
 * All three image buffers are device buffers of n_pixels * 4 floats; `loss`
 * (host, optional) receives the sum in double.  No counterpart in the
 * reference. */
gt_status gt_l2_loss(gt_context* ctx, const float* rgba, const float* target, uint64_t n_pixels,
                     float* dL_drgba, double* loss);

/* ============================================================ tuning
 * No counterpart in the reference.  Times the tracer's launch shapes on the
 * given view and caches the fastest per (GPU, scene-size bucket, image-size
 * bucket, k).  gt_render and gt_render_batch use the cached choice.
 * Two kernels render the plain image (debugMode 0), with identical results:
 *   block_threads 32:  a warp traces the 32 rays of an 8x4 tile together;
 *                      kbuf = k-buffer entries per ray (k..64, default 32),
 *                      handoff_after as below (the tuner times 2 to 8
 *                      and 64 for the fastest kbuf); blocks_per_sm and leaf_batch are
 *                      not used (the grid fills the SMs);
 *   block_threads 128: a warp traces one ray; kbuf = k-buffer entries of a
 *                      traversal (k..128, default 64), blocks_per_sm and
 *                      leaf_batch as below.
 * Without a cached shape a launch takes the first kernel when it has at
 * least 48 8x4 tiles per SM (about 0.23 Mpixels on a 148-SM B200) and the
 * second otherwise: tiles are coarse work items, and with few of them per
 * warp the slowest ones decide the time.  With the first kernel, the rays
 * of a tile that still need hits after three traversals (or after the
 * current one, once every tile of the launch is taken) are finished by
 * the second one (a second launch).  The same choice holds for the
 * checkpointing forward of gt_backward; debug modes and hit recording
 * always use the second kernel. */
typedef struct gt_tune_result {
  uint32_t block_threads; /* 32: a warp per 8x4 tile; 128: a warp per ray      */
  uint32_t blocks_per_sm; /* resident blocks per SM of the persistent grid      */
  uint32_t tile_w, tile_h;/* pixel tile a warp takes per work-stealing step     */
  float best_ms;          /* fastest trace time measured                        */
  float default_ms;       /* trace time of the default launch shape             */
  uint32_t kbuf;          /* k-buffer entries (see above; raised to k)          */
  uint32_t leaf_batch;    /* queued leaves that start a batch of proxy tests    */
  uint32_t handoff_after; /* block_threads 32: traversals after which a tile   *
                           * hands its unfinished rays to a warp-per-ray       *
                           * launch (0: the default, 3)                         */
  uint32_t _pad;
} gt_tune_result;

gt_status gt_autotune(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u,
                      uint32_t w, uint32_t h, gt_tune_result* result);
/* Times launch shapes on a whole batch (the items of a gt_render_batch call:
 * views, scenes and k as given; the images go to a scratch buffer of the
 * context, out_rgba is not written) and caches the fastest for batches of
 * that shape (the same view count, tile count and k bucket), which
 * gt_render_batch and the checkpointing forward of a batch then use ahead of
 * the per-view cache.  Tried: the tile packets with k-buffers of k, 24, 32,
 * 48 and 64 entries and hand-offs after 2, 3, 4 and 6 traversals, and a warp
 * per ray at 4 and 8 blocks per SM.  The tile (8 x 4) and the traversal stack
 * (256 entries) are fixed: other tiles measured within 0.3 %, and a smaller
 * stack would turn deep packets into GT_ERR_STACK_OVERFLOW. */
gt_status gt_autotune_batch(gt_context* ctx, const gt_batch_item* items, uint32_t count,
                            gt_tune_result* result);
/* Installs a launch shape for the bucket of (scene, u->k, w x h) without
 * timing anything (for example one found by gt_autotune in an earlier run).
 * block_threads must be 32 or 128 and the tile 8 x 4; blocks_per_sm 1..32,
 * kbuf 1..128 (used up to 64 with block_threads 32) and leaf_batch 1..32.
 * best_ms/default_ms are ignored. */
gt_status gt_set_tune(gt_context* ctx, const gt_scene* scene, const gt_uniforms* u, uint32_t w,
                      uint32_t h, const gt_tune_result* shape);
/* Drops every cached tuning result of the context. */
gt_status gt_autotune_reset(gt_context* ctx);

/* ======================================================== loop limits
 * No counterpart in the reference.  Every device loop of the trace kernels is
 * bounded: traversal steps (4 n + 64 per traversal), stack entries (256 per
 * warp) and rounds per ray (2^22).  A ray that reaches a bound stops, and the
 * call returns GT_ERR_DEVICE_TIMEOUT (steps, rounds) or GT_ERR_STACK_OVERFLOW
 * (stack) with the context still usable.  gt_set_limits lowers the bounds (0
 * restores a default) so that callers and tests can exercise that path
 * without a fault; it drops the context's captured batch graphs. */
gt_status gt_set_limits(gt_context* ctx, uint32_t max_steps, uint32_t stack_entries, uint32_t max_rounds);

/* ====================================================== device helpers
 * For callers without a CUDA binding of their own (the N-API addon, the
 * benchmark): plain device buffers on the context's GPU, and CUDA-event
 * timing on the context's stream. */
gt_status gt_device_alloc(gt_context* ctx, uint64_t bytes, void** out);
gt_status gt_device_free(gt_context* ctx, void* ptr);
/* Page-locked host buffers (fast host<->device copies). */
gt_status gt_host_alloc(gt_context* ctx, uint64_t bytes, void** out);
gt_status gt_host_free(gt_context* ctx, void* ptr);
/* kind: 0 = host to device, 1 = device to host, 2 = device to device. */
gt_status gt_memcpy(gt_context* ctx, void* dst, const void* src, uint64_t bytes, int kind);
gt_status gt_synchronize(gt_context* ctx);
/* Records a CUDA event on the context stream; gt_timer_stop records a second
 * one, waits for it and returns the elapsed device milliseconds. */
gt_status gt_timer_start(gt_context* ctx);
gt_status gt_timer_stop(gt_context* ctx, float* ms);
/* Device durations of the trace-kernel launches made since the previous call
 * (at most `max`, oldest first; each launch is bracketed by CUDA events on
 * the context stream).  Waits for them to finish. */
gt_status gt_kernel_times(gt_context* ctx, float* out_ms, uint32_t max, uint32_t* n);
/* Number of kernel launches the library has made on this context. */
gt_status gt_launch_count(const gt_context* ctx, uint64_t* n);
/* The context's GPU: streaming multiprocessors and the SM clock the driver
 * reports as its maximum (kHz), for issue-rate rooflines.  Either pointer
 * may be NULL. */
gt_status gt_device_attributes(const gt_context* ctx, uint32_t* sm_count, uint32_t* max_sm_khz);

#ifdef __cplusplus
}
#endif
#endif /* GTRACE_H */
