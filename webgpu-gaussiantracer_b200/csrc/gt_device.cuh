// gt_device.cuh — device math of the tracer: ray generation, the ray/proxy
// test, the Gaussian response, SH radiance and compositing.
//
// Every function here follows the fixed binary32 operation order of the
// numerics contract (gt_internal.cuh).  The translation units that include
// this header are compiled with -fmad=false, so `a * b + c` is two rounded
// operations, evaluated in the order written; division and square root use
// the correctly rounded intrinsics.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "gt_internal.cuh"

namespace gt {

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 mk(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 vscale(float s, V3 a) { return mk(s * a.x, s * a.y, s * a.z); }
// dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z
__device__ __forceinline__ float vdot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ V3 vcross(V3 a, V3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// normalize(v) = v / sqrt(dot(v, v))
__device__ __forceinline__ V3 vnorm(V3 v) {
  float l = __fsqrt_rn(vdot(v, v));
  return mk(__fdiv_rn(v.x, l), __fdiv_rn(v.y, l), __fdiv_rn(v.z, l));
}

// World-to-object map of a proxy: 4x3 column-major in 3 float4.
struct Affine {
  float m[12];
};
__device__ __forceinline__ Affine load_affine(const float4* p) {
  float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  return Affine{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w}};
}
// M * vec4(p, 1) = ((c0*p.x + c1*p.y) + c2*p.z) + c3
__device__ __forceinline__ V3 xpoint(const Affine& M, V3 p) {
  const float* m = M.m;
  return mk(((m[0] * p.x + m[3] * p.y) + m[6] * p.z) + m[9], ((m[1] * p.x + m[4] * p.y) + m[7] * p.z) + m[10],
            ((m[2] * p.x + m[5] * p.y) + m[8] * p.z) + m[11]);
}
// M * vec4(d, 0) = (c0*d.x + c1*d.y) + c2*d.z
__device__ __forceinline__ V3 xdir(const Affine& M, V3 d) {
  const float* m = M.m;
  return mk((m[0] * d.x + m[3] * d.y) + m[6] * d.z, (m[1] * d.x + m[4] * d.y) + m[7] * d.z,
            (m[2] * d.x + m[5] * d.y) + m[8] * d.z);
}

// Deterministic exp: Cody-Waite reduction with a 16-bit head of ln 2, a
// degree-7 Taylor polynomial of e^r on |r| <= ln2/2 (Horner), scaling by
// 2^n from exponent bits.  Same bits as the oracle's or_expf on any input.
__device__ __forceinline__ float det_expf(float x) {
  if (x != x) return x;
  if (x > 88.0f) return CUDART_INF_F;
  if (x < -87.0f) return 0.0f;
  const float log2e = 1.44269504088896340736f;
  const float ln2_hi = 0.693145751953125f;
  const float ln2_lo = 1.42860682030941723212e-6f;
  float fn = floorf(x * log2e + 0.5f);
  float r = (x - fn * ln2_hi) - fn * ln2_lo;
  float p = 1.98412698412698412698e-4f;
  p = p * r + 1.38888888888888888889e-3f;
  p = p * r + 8.33333333333333333333e-3f;
  p = p * r + 4.16666666666666666667e-2f;
  p = p * r + 1.66666666666666666667e-1f;
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  int n = (int)fn;
  return p * __int_as_float((n + 127) << 23);
}

// Deterministic natural log in double: x = m 2^e, m in [sqrt(1/2), sqrt(2)),
// log m = 2 atanh((m-1)/(m+1)) by its odd power series to degree 23.
__device__ __forceinline__ double det_log(double x) {
  if (x != x) return x;
  if (x <= 0.0) return x == 0.0 ? -CUDART_INF : CUDART_NAN;
  if (isinf(x)) return x;
  int e = 0;
  double m = frexp(x, &e);
  if (m < 0.70710678118654752440) {
    m = __dmul_rn(m, 2.0);
    e = e - 1;
  }
  double f = __ddiv_rn(__dsub_rn(m, 1.0), __dadd_rn(m, 1.0));
  double f2 = __dmul_rn(f, f);
  double s = __ddiv_rn(1.0, 23.0);
  for (int k = 21; k >= 1; k -= 2) s = __dadd_rn(__dmul_rn(s, f2), __ddiv_rn(1.0, (double)k));
  double lm = __dmul_rn(__dmul_rn(2.0, f), s);
  return __dadd_rn(__dmul_rn((double)e, 0.69314718055994530942), lm);
}

// Ray generation (src/GS_shader.ts:275-285).
// Per-pixel seed of the reference's progressive anti-aliasing
// (getNewSeed, src/GS_shader.ts:9-23): 8 rounds of the TEA block cipher
// (Wheeler and Needham 1994) keyed by the reference's four constants.
__device__ __forceinline__ uint32_t aa_seed(uint32_t p1, uint32_t p2) {
  uint32_t s0 = 0, v0 = p1, v1 = p2;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    s0 += 0x9e3779b9u;
    v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
    v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
  }
  return v0;
}

// rng (src/GS_shader.ts:25-29): LCG step, low 24 bits scaled to [0, 1).
__device__ __forceinline__ float aa_rng(uint32_t& seed) {
  seed = 1664525u * seed + 1013904223u;
  return (float)(seed & 0x00FFFFFFu) * (1.0f / 16777216.0f);
}

// Ray generation (src/GS_shader.ts:275-285): camera basis from the columns
// of toWorld; the pixel sample is the centre, or with anti-aliasing the
// jitter (rng(seed), rng(seed)) of seed = getNewSeed(W*y + x, frames, 8).
__device__ __forceinline__ void ray_gen(const RayUniforms& u, uint32_t w, uint32_t h, uint32_t px, uint32_t py,
                                        V3& o, V3& d) {
  V3 cx = mk(-u.tw[0], -u.tw[1], -u.tw[2]);
  V3 cy = mk(u.tw[4], u.tw[5], u.tw[6]);
  V3 cz = mk(-u.tw[8], -u.tw[9], -u.tw[10]);
  o = mk(u.tw[12], u.tw[13], u.tw[14]);
  float jx = 0.5f, jy = 0.5f;
  if (u.aa) {
    uint32_t seed = aa_seed(w * py + px, u.frames);
    jx = aa_rng(seed);
    jy = aa_rng(seed);
  }
  float nx = __fdiv_rn((float)px + jx, (float)w) * 2.0f - 1.0f;
  float ny = __fdiv_rn((float)py + jy, (float)h) * 2.0f - 1.0f;
  float ax = nx * u.asp[0], ay = ny * u.asp[1];
  V3 v = mk((ax * cx.x + ay * cy.x) + cz.x, (ax * cx.y + ay * cy.y) + cz.y, (ax * cx.z + ay * cy.z) + cz.z);
  d = vnorm(v);
}

// Progressive average (src/GS_shader.ts:302-308): frame 0 replaces the
// pixel, frame f > 0 blends mix(old, new, 1 / (f + 1)) = old (1 - a) + new a.
__device__ __forceinline__ float4 aa_blend(float4 old, float4 nw, uint32_t frames) {
  if (frames == 0) return make_float4(nw.x, nw.y, nw.z, 1.0f);
  const float a = __fdiv_rn(1.0f, __uint2float_rn(frames) + 1.0f);
  const float b = 1.0f - a;
  return make_float4(old.x * b + nw.x * a, old.y * b + nw.y * a, old.z * b + nw.z * a, 1.0f);
}

// intersect_triangle_branchless0 (webrtx/src/glsl/intersect.glsl:73-92):
// e2 = (1/dot(n,d)) (p0 - o); t = dot(n, e2) in (tmin, tmax);
// i = cross(d, e2); beta = dot(i, e1) >= 0, gamma = dot(i, e0) >= 0,
// beta + gamma <= 1.  `dn` is dot(n, d), computed by the caller.
__device__ __forceinline__ bool tri_test(const FaceTable& F, int f, V3 o, float tmin, V3 d, float tmax, float dn,
                                         float& t_out) {
  V3 p0 = mk(F.p0[f][0], F.p0[f][1], F.p0[f][2]);
  V3 n = mk(F.n[f][0], F.n[f][1], F.n[f][2]);
  float r = __frcp_rn(dn);
  V3 e2 = vscale(r, vsub(p0, o));
  float t = vdot(n, e2);
  if (t <= tmin || tmax <= t || t != t) return false;
  V3 i = vcross(d, e2);
  float beta = vdot(i, mk(F.e1[f][0], F.e1[f][1], F.e1[f][2]));
  float gamma = vdot(i, mk(F.e0[f][0], F.e0[f][1], F.e0[f][2]));
  t_out = t;
  return beta >= 0.0f && gamma >= 0.0f && beta + gamma <= 1.0f;
}

// Facing (webrtx/src/glsl/trace.glsl:154-164): n_world = n * W2O, front iff
// dot(n_world, d_world) < 0.
__device__ __forceinline__ bool front_facing(const FaceTable& F, int f, const Affine& W, V3 d) {
  V3 n = mk(F.n[f][0], F.n[f][1], F.n[f][2]);
  const float* m = W.m;
  V3 nw = mk(vdot(n, mk(m[0], m[1], m[2])), vdot(n, mk(m[3], m[4], m[5])), vdot(n, mk(m[6], m[7], m[8])));
  return vdot(nw, d) < 0.0f;
}

// Shading record of one particle (see SceneDev::shade).
struct Shade {
  V3 mu;
  float opacity;
  float a00, a01, a02, a11, a12, a22;
};
__device__ __forceinline__ Shade load_shade(const float4* shade, uint32_t p) {
  const float4* s = shade + 3 * (size_t)p;
  float4 a = __ldg(s), b = __ldg(s + 1), c = __ldg(s + 2);
  return Shade{mk(a.x, a.y, a.z), a.w, b.x, b.y, b.z, b.w, c.x, c.y};
}

// Precision matrix A = (invS R)^T (invS R) of computeResponse
// (src/GS_shader.ts:115-130), GLSL column-major: R columns from (r,x,y,z).
// Used by the scene build; the result is symmetric bit for bit.
__device__ __forceinline__ void precision_matrix(const float q[4], const float sc[3], float A[3][3]) {
  float r = q[0], x = q[1], y = q[2], z = q[3];
  float R[3][3];
  R[0][0] = 1.0f - 2.0f * (y * y + z * z);
  R[0][1] = 2.0f * (x * y - r * z);
  R[0][2] = 2.0f * (x * z + r * y);
  R[1][0] = 2.0f * (x * y + r * z);
  R[1][1] = 1.0f - 2.0f * (x * x + z * z);
  R[1][2] = 2.0f * (y * z - r * x);
  R[2][0] = 2.0f * (x * z - r * y);
  R[2][1] = 2.0f * (y * z + r * x);
  R[2][2] = 1.0f - 2.0f * (x * x + y * y);
  float is[3] = {__fdiv_rn(1.0f, sc[0]), __fdiv_rn(1.0f, sc[1]), __fdiv_rn(1.0f, sc[2])};
  float M1[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int rr = 0; rr < 3; ++rr) M1[c][rr] = is[rr] * R[c][rr];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int rr = 0; rr < 3; ++rr) A[c][rr] = (M1[rr][0] * M1[c][0] + M1[rr][1] * M1[c][1]) + M1[rr][2] * M1[c][2];
}

// computeResponse (src/GS_shader.ts:111-136): response at the point of
// maximum density along the ray.  Also returns q = p - mu for the adjoint.
__device__ __forceinline__ float response(const Shade& s, V3 o, V3 d, V3* q_out = nullptr) {
  V3 temp = mk((s.a00 * d.x + s.a01 * d.y) + s.a02 * d.z, (s.a01 * d.x + s.a11 * d.y) + s.a12 * d.z,
               (s.a02 * d.x + s.a12 * d.y) + s.a22 * d.z);
  float tau = __fdiv_rn(vdot(vsub(s.mu, o), temp), vdot(d, temp));
  V3 p = mk(o.x + tau * d.x, o.y + tau * d.y, o.z + tau * d.z);
  V3 pm = vsub(p, s.mu);
  V3 apm = mk((s.a00 * pm.x + s.a01 * pm.y) + s.a02 * pm.z, (s.a01 * pm.x + s.a11 * pm.y) + s.a12 * pm.z,
              (s.a02 * pm.x + s.a12 * pm.y) + s.a22 * pm.z);
  float e = vdot(vsub(s.mu, p), apm);
  if (q_out) *q_out = pm;
  return det_expf(e);
}

// SH constants (src/GS_shader.ts:39-52)
#define GT_SH_C0 0.28209479177387814f
#define GT_SH_C1 0.4886025119029199f
#define GT_SH_C2_0 1.0925484305920792f
#define GT_SH_C2_1 -1.0925484305920792f
#define GT_SH_C2_2 0.31539156525252005f
#define GT_SH_C2_3 -1.0925484305920792f
#define GT_SH_C2_4 0.5462742152960396f
#define GT_SH_C3_0 -0.5900435899266435f
#define GT_SH_C3_1 2.890611442640554f
#define GT_SH_C3_2 -0.4570457994644658f
#define GT_SH_C3_3 0.3731763325901154f
#define GT_SH_C3_4 -0.4570457994644658f
#define GT_SH_C3_5 1.445305721320277f
#define GT_SH_C3_6 -0.5900435899266435f

// shToRadiance (src/GS_shader.ts:138-177) before the max(0, .), for one
// channel; `c` holds the 16 coefficients of that channel.
__device__ __forceinline__ float sh_channel(const float c[16], V3 d, uint32_t deg) {
  float L = 0.5f + GT_SH_C0 * c[0];
  if (deg == 0) return L;
  float x = d.x, y = d.y, z = d.z;
  L = L + GT_SH_C1 * ((-y * c[1] + z * c[2]) - x * c[3]);
  if (deg == 1) return L;
  float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
  float s2 = GT_SH_C2_0 * xy * c[4];
  s2 = s2 + GT_SH_C2_1 * yz * c[5];
  s2 = s2 + GT_SH_C2_2 * ((2.0f * zz - xx) - yy) * c[6];
  s2 = s2 + GT_SH_C2_3 * xz * c[7];
  s2 = s2 + GT_SH_C2_4 * (xx - yy) * c[8];
  L = L + s2;
  if (deg == 2) return L;
  float s3 = GT_SH_C3_0 * y * (3.0f * xx - yy) * c[9];
  s3 = s3 + GT_SH_C3_1 * xy * z * c[10];
  s3 = s3 + GT_SH_C3_2 * y * ((4.0f * zz - xx) - yy) * c[11];
  s3 = s3 + GT_SH_C3_3 * z * ((2.0f * zz - 3.0f * xx) - 3.0f * yy) * c[12];
  s3 = s3 + GT_SH_C3_4 * x * ((4.0f * zz - xx) - yy) * c[13];
  s3 = s3 + GT_SH_C3_5 * z * (xx - yy) * c[14];
  s3 = s3 + GT_SH_C3_6 * x * (xx - 3.0f * yy) * c[15];
  return L + s3;
}

// Loads the 48 SH floats of particle p (12 x 128-bit loads) and evaluates
// the three channels (raw, before the clamp).
__device__ __forceinline__ void sh_radiance(const float4* sh, uint32_t p, V3 d, uint32_t deg, float out[3]) {
  const float4* s = sh + 12 * (size_t)p;
  float v[48];
  int nload = deg == 0 ? 1 : (deg == 1 ? 3 : (deg == 2 ? 7 : 12));
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    float4 q = i < nload ? __ldg(s + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    v[4 * i] = q.x;
    v[4 * i + 1] = q.y;
    v[4 * i + 2] = q.z;
    v[4 * i + 3] = q.w;
  }
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    float c[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) c[k] = v[3 * k + ch];
    out[ch] = sh_channel(c, d, deg);
  }
}

// The colour an entry of particle p adds for a ray from o
// (src/GS_shader.ts:258-264,189): max(0, SH(normalize(mu - o))) per channel
// (NaN and -0 become +0).  It does not depend on the ray's direction, so all
// primary rays of a view (they share o) get the same colour for p.
__device__ __forceinline__ void entry_colour(const float4* sh, uint32_t p, V3 mu, V3 o, uint32_t deg, float& x0,
                                             float& x1, float& x2) {
  const V3 dir = vnorm(vsub(mu, o));
  float c[3];
  sh_radiance(sh, p, dir, deg, c);
  x0 = c[0] > 0.f ? c[0] : 0.f;
  x1 = c[1] > 0.f ? c[1] : 0.f;
  x2 = c[2] > 0.f ? c[2] : 0.f;
}

}  // namespace gt
