/*
 * gt_oracle.h — CPU oracle of the Gaussian ray tracer.  TEST INFRASTRUCTURE.
 *
 * This library is the parity checker for the CUDA tracer and the timed CPU
 * baseline of the benchmark.  It is never linked into, loaded by or called
 * from the product library.  Only the tests, the smoke check and the
 * benchmark's CPU-baseline leg use it.
 *
 * Parity unpinned: the reference runs only as a browser WebGPU application
 * (TypeScript + WebRTX GLSL transpiled to WGSL, Rust compiled to WASM); none
 * of its code can run in this environment and its repository holds no
 * golden vectors or known-answer tests for the render path.  This oracle
 * restates the reference's algorithm from its source (file:line cited on
 * every function) and is itself pinned by analytic known-answer tests.
 *
 * Each function exists for float (_f32) and double (_f64).  The float build
 * follows one fixed IEEE-754 operation order (no contraction, correctly
 * rounded division and square root, a deterministic exp/log written here)
 * that the CUDA tracer follows too, so the two agree bit for bit; the
 * double build is the FP64 reference render used for error statistics.
 */
#ifndef GT_ORACLE_H
#define GT_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_scene_f32 or_scene_f32;
typedef struct or_scene_f64 or_scene_f64;

/* Hit-list recording of a render (all arrays sized by the caller). */
typedef struct or_hits {
  uint32_t max_entries;  /* capacity per pixel                                     */
  uint32_t* pidx;        /* [n_pix * max_entries] particle index of each entry     */
  float* t;              /* [n_pix * max_entries] hit t                             */
  float* alpha;          /* [n_pix * max_entries] alpha of the entry                */
  uint32_t* count;       /* [n_pix] valid entries (may exceed max_entries)          */
  uint32_t* rounds;      /* [n_pix] traversal rounds                                */
  uint64_t anyhits;      /* out: front-face hits offered to the k-buffer (total)    */
  uint64_t node_visits;  /* out: BVH nodes visited (total)                          */
} or_hits;

/* PLY ingest restatement of PackedGaussians (src/GS_ply.ts:58-253).
 * Returns 0 on success.  With aos == NULL only n/sh_degree/stride are set.
 * act64 (optional, with aos): the activated values in double, 8 per vertex:
 * opacity, scale xyz, rotation wxyz (gaussianData, before the binary32
 * rounding of the packed records). */
int or_ply_to_aos(const uint8_t* bytes, size_t len, uint32_t* n, uint32_t* sh_degree,
                  uint32_t* stride, float* aos, double* act64);

/* Progressive anti-aliasing restatement: renders the full image with the
 * jittered samples of (pixel, uniforms.accumulatedFrames) and blends it into
 * accum (w*h*4), src/GS_shader.ts:275-308 with antialiasing = true. */
int or_render_accum_f32(const or_scene_f32* s, const void* uniforms, uint32_t w, uint32_t h,
                        int threads, float* accum);
/* getNewSeed and rng of src/GS_shader.ts:6-31. */
uint32_t or_new_seed(uint32_t p1, uint32_t p2, uint32_t rounds);
float or_rng(uint32_t* seed);
/* Tone map of src/toneMapper.ts:15-24 into unorm8 RGBA (modes 0..2). */
int or_tonemap(const float* rgba, uint64_t n, uint32_t mode, float exposure, uint8_t* out);

/* Deterministic elementary functions shared by the float oracle and the CUDA
 * tracer's specification (exposed for their unit tests). */
float or_expf(float x);
double or_log(double x);

or_scene_f32* or_scene_create_f32(const float* aos, uint64_t n, uint32_t stride_bytes,
                                  double alpha_min);
or_scene_f64* or_scene_create_f64(const float* aos, uint64_t n, uint32_t stride_bytes,
                                  double alpha_min);
/* As or_scene_create_* with the activated values in double (8 per particle:
 * opacity, scale xyz, rotation wxyz): the opacity cut and the proxies use
 * them, as src/main.ts:72-94 uses the JS numbers; NULL = the packed values. */
or_scene_f32* or_scene_create_ex_f32(const float* aos, uint64_t n, uint32_t stride_bytes,
                                     double alpha_min, const double* act64);
or_scene_f64* or_scene_create_ex_f64(const float* aos, uint64_t n, uint32_t stride_bytes,
                                     double alpha_min, const double* act64);
void or_scene_destroy_f32(or_scene_f32* s);
void or_scene_destroy_f64(or_scene_f64* s);
uint64_t or_scene_kept_f32(const or_scene_f32* s);
uint64_t or_scene_kept_f64(const or_scene_f64* s);
/* Proxy data of kept proxy j: particle index, object-to-world and
 * world-to-object 4x3 column-major matrices (as float). */
int or_scene_proxy_f32(const or_scene_f32* s, uint64_t j, uint32_t* pidx, float* o2w,
                       float* w2o);

/* Renders the listed pixels (pixels == NULL: the full image, n_pix = w*h).
 *   uniforms  the 112-byte block of include/gtrace.h
 *   algo      0 = sort-all-hits checker: every front-face proxy hit in
 *                 (t_min, t_max) is gathered, ordered by (t, particle index),
 *                 and the reference's rounds are replayed on that list;
 *             1 = reference traversal: per round a stackless traversal of a
 *                 two-level BVH with the any-hit k-buffer insertion and
 *                 commit rule (webrtx/src/glsl/trace.glsl:42-245,
 *                 src/GS_shader.ts:323-367)
 *   threads   OpenMP threads (0 = all)
 *   out_rgba  4 floats per listed pixel
 *   hits      optional hit-list recording (NULL allowed)
 * Returns 0 on success. */
int or_render_f32(const or_scene_f32* s, const void* uniforms, uint32_t w, uint32_t h,
                  const uint32_t* pixels, uint32_t n_pix, int algo, int threads,
                  float* out_rgba, or_hits* hits);
int or_render_f64(const or_scene_f64* s, const void* uniforms, uint32_t w, uint32_t h,
                  const uint32_t* pixels, uint32_t n_pix, int algo, int threads,
                  double* out_rgba, or_hits* hits);

/* FP64 adjoint: gradient of sum(dL_drgba * rgba) w.r.t. the 59 parameters of
 * every particle (parameter-major, 59*n), hit sets held fixed.  Uses the
 * algo-0 hit lists of the double render. */
int or_backward_f64(const or_scene_f64* s, const void* uniforms, uint32_t w, uint32_t h,
                    const uint32_t* pixels, uint32_t n_pix, const double* dL_drgba,
                    int threads, double* dL_dparams);

/* FP64 adjoint on given entry lists: for each listed pixel, the composited
 * hit sequence of a render (particle indices, `counts` entries, rows of
 * `max_e`) and optionally which entries passed alpha_min (NULL: decided in
 * double).  Rounds are implicit in the lists. */
int or_backward_lists_f64(const or_scene_f64* s, const void* uniforms, uint32_t w, uint32_t h,
                          const uint32_t* pixels, uint32_t n_pix, const uint32_t* lists,
                          const uint8_t* contrib, const uint32_t* counts, uint32_t max_e,
                          const double* dL_drgba, int threads, double* dL_dparams);

#ifdef __cplusplus
}
#endif
#endif
