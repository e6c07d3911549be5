/*
 * gt_oracle.c — CPU oracle of the Gaussian ray tracer.  TEST INFRASTRUCTURE
 * (parity checker and timed CPU baseline only; never part of the product).
 * Parity unpinned: see gt_oracle.h.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).  The float
 * instantiation depends on -ffp-contract=off: every a*b+c below is two
 * rounded operations, in the order written.
 */
#include "gt_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------
 * Deterministic exp (float).  Cody & Waite argument reduction
 * (W. J. Cody, W. Waite, "Software Manual for the Elementary Functions",
 * 1980): x = n ln2 + r with ln2 split into a 16-bit head and a tail, then a
 * degree-7 Taylor polynomial of e^r on |r| <= ln2/2 in Horner form, then a
 * scale by 2^n built from the exponent bits.  Only +, -, *, floor and bit
 * moves, so any IEEE-754 binary32 machine without contraction returns the
 * same bits.  Error is within 2 ulp of e^x on [-87, 88]; results below
 * e^-87 flush to 0 (alpha values that small never pass alpha_min).
 * ---------------------------------------------------------------------- */
float or_expf(float x) {
  if (x != x) return x;
  if (x > 88.0f) return INFINITY;
  if (x < -87.0f) return 0.0f;
  const float log2e = 1.44269504088896340736f;
  const float ln2_hi = 0.693145751953125f;       /* 16 significant bits */
  const float ln2_lo = 1.42860682030941723212e-6f;
  float fn = floorf(x * log2e + 0.5f);
  float r = (x - fn * ln2_hi) - fn * ln2_lo;
  float p = 1.98412698412698412698e-4f;  /* 1/7! */
  p = p * r + 1.38888888888888888889e-3f; /* 1/6! */
  p = p * r + 8.33333333333333333333e-3f; /* 1/5! */
  p = p * r + 4.16666666666666666667e-2f; /* 1/4! */
  p = p * r + 1.66666666666666666667e-1f; /* 1/3! */
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  int n = (int)fn;
  uint32_t bits = (uint32_t)(n + 127) << 23;
  float scale;
  memcpy(&scale, &bits, sizeof scale);
  return p * scale;
}

/* ------------------------------------------------------------------------
 * Deterministic natural log (double).  x = m 2^e with m in [sqrt(1/2),
 * sqrt(2)), log m = 2 atanh(f), f = (m-1)/(m+1), by its odd power series
 * to f^23 (|f| <= 0.1716, truncation below 1e-19).  Used only for the proxy
 * scale sqrt(2 ln(opacity/alpha_min)) (src/main.ts:84).
 * ---------------------------------------------------------------------- */
double or_log(double x) {
  if (x != x) return x;
  if (x <= 0.0) return x == 0.0 ? -INFINITY : NAN;
  if (isinf(x)) return x;
  int e = 0;
  double m = frexp(x, &e);
  if (m < 0.70710678118654752440) {
    m = m * 2.0;
    e = e - 1;
  }
  double f = (m - 1.0) / (m + 1.0);
  double f2 = f * f;
  double s = 1.0 / 23.0;
  for (int k = 21; k >= 1; k -= 2) s = s * f2 + 1.0 / (double)k;
  double lm = 2.0 * f * s;
  return (double)e * 0.69314718055994530942 + lm;
}

/* ------------------------------------------------------------------------
 * PLY ingest: restatement of PackedGaussians (src/GS_ply.ts:58-253).
 *   header: "element vertex N", "property <type> <name>" (float | uchar),
 *           data starts one byte after "end_header" (:103)
 *   per vertex, in header order: float -> f32 LE, uchar -> byte/255 (:120-128)
 *   activation (in double, :225-235): scale = exp, quaternion / its norm,
 *           opacity = 1/(1+exp(-x))
 *   SH order (:188-196): sh[0] = f_dc_0..2; sh[i+1].rgb = f_rest_{rgb*n+i},
 *           n = #f_rest / 3
 *   std430 packing (src/GS_packing.ts:146-174,233-245): position @0,
 *           scale @16, rotation @32, opacity @48, sh[j] @64+16j;
 *           record size rounded up to 16.
 * ---------------------------------------------------------------------- */
#define OR_MAX_PROPS 256
int or_ply_to_aos(const uint8_t* bytes, size_t len, uint32_t* n_out, uint32_t* deg_out,
                  uint32_t* stride_out, float* aos) {
  const char* end_tag = "end_header";
  size_t hdr_end = 0;
  for (size_t i = 0; i + 10 <= len; ++i) {
    if (memcmp(bytes + i, end_tag, 10) == 0) {
      hdr_end = i + 10 + 1;
      break;
    }
  }
  if (hdr_end == 0 || hdr_end > len) return 1;
  char names[OR_MAX_PROPS][32];
  int is_float[OR_MAX_PROPS];
  int np = 0;
  uint64_t nvert = 0;
  size_t pos = 0;
  while (pos < hdr_end) {
    size_t e = pos;
    while (e < hdr_end && bytes[e] != '\n') ++e;
    char line[256];
    size_t l = e - pos < 255 ? e - pos : 255;
    memcpy(line, bytes + pos, l);
    line[l] = 0;
    /* trim */
    char* p = line;
    while (*p == ' ' || *p == '\t' || *p == '\r') ++p;
    size_t pl = strlen(p);
    while (pl && (p[pl - 1] == ' ' || p[pl - 1] == '\r' || p[pl - 1] == '\t')) p[--pl] = 0;
    if (strncmp(p, "element vertex", 14) == 0) {
      const char* q = p;
      while (*q && (*q < '0' || *q > '9')) ++q;
      nvert = strtoull(q, NULL, 10);
    } else if (strncmp(p, "property", 8) == 0) {
      char a[64], t[64], nm[64];
      if (sscanf(p, "%63s %63s %63s", a, t, nm) == 3) {
        int idx = -1;
        for (int i = 0; i < np; ++i)
          if (strcmp(names[i], nm) == 0) idx = i;
        if (idx < 0) {
          if (np >= OR_MAX_PROPS) return 2;
          idx = np++;
          snprintf(names[idx], sizeof names[idx], "%s", nm);
        }
        is_float[idx] = strcmp(t, "float") == 0 ? 1 : (strcmp(t, "uchar") == 0 ? 0 : -1);
      }
    } else if (strcmp(p, "end_header") == 0) {
      break;
    }
    pos = e + 1;
  }
  int n_rest = 0;
  for (int i = 0; i < np; ++i)
    if (strncmp(names[i], "f_rest_", 7) == 0) ++n_rest;
  int per_color = n_rest / 3;
  double degf = sqrt((double)per_color + 1.0) - 1.0;
  int deg = (int)degf;
  if ((double)deg != degf || deg < 0 || deg > 3) return 3;
  int n_sh = (deg + 1) * (deg + 1);
  /* struct: 64 bytes of header fields + n_sh vec3 at stride 16, size rounded to 16 */
  uint32_t stride = 64u + 16u * (uint32_t)n_sh;
  *n_out = (uint32_t)nvert;
  *deg_out = (uint32_t)deg;
  *stride_out = stride;
  if (!aos) return 0;
  /* bytes per vertex */
  size_t vbytes = 0;
  for (int i = 0; i < np; ++i) vbytes += is_float[i] == 1 ? 4 : (is_float[i] == 0 ? 1 : 0);
  if (hdr_end + vbytes * nvert > len) return 4;
  int ix[14];
  const char* want[14] = {"x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0",
                          "rot_1", "rot_2", "rot_3", "opacity", "f_dc_0", "f_dc_1", "f_dc_2"};
  for (int w = 0; w < 14; ++w) {
    ix[w] = -1;
    for (int i = 0; i < np; ++i)
      if (strcmp(names[i], want[w]) == 0) ix[w] = i;
    if (ix[w] < 0) return 5;
  }
  int rest_ix[45];
  for (int r = 0; r < n_rest && r < 45; ++r) {
    char nm[32];
    snprintf(nm, sizeof nm, "f_rest_%d", r);
    rest_ix[r] = -1;
    for (int i = 0; i < np; ++i)
      if (strcmp(names[i], nm) == 0) rest_ix[r] = i;
    if (rest_ix[r] < 0) return 6;
  }
  double* v = (double*)malloc(sizeof(double) * (size_t)np);
  if (!v) return 7;
  const uint8_t* data = bytes + hdr_end;
  for (uint64_t g = 0; g < nvert; ++g) {
    size_t off = 0;
    for (int i = 0; i < np; ++i) {
      if (is_float[i] == 1) {
        float f;
        memcpy(&f, data + off, 4);
        v[i] = (double)f;
        off += 4;
      } else if (is_float[i] == 0) {
        v[i] = (double)data[off] / 255.0;
        off += 1;
      }
    }
    data += vbytes;
    float* rec = aos + (size_t)g * (stride / 4);
    memset(rec, 0, stride);
    rec[0] = (float)v[ix[0]];
    rec[1] = (float)v[ix[1]];
    rec[2] = (float)v[ix[2]];
    rec[4] = (float)exp(v[ix[3]]);
    rec[5] = (float)exp(v[ix[4]]);
    rec[6] = (float)exp(v[ix[5]]);
    double q0 = v[ix[6]], q1 = v[ix[7]], q2 = v[ix[8]], q3 = v[ix[9]];
    double nrm = sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
    rec[8] = (float)(q0 / nrm);
    rec[9] = (float)(q1 / nrm);
    rec[10] = (float)(q2 / nrm);
    rec[11] = (float)(q3 / nrm);
    rec[12] = (float)(1.0 / (1.0 + exp(-v[ix[10]])));
    for (int c = 0; c < 3; ++c) rec[16 + c] = (float)v[ix[11 + c]];
    for (int i = 0; i < per_color; ++i)
      for (int c = 0; c < 3; ++c) rec[16 + 4 * (i + 1) + c] = (float)v[rest_ix[c * per_color + i]];
  }
  free(v);
  return 0;
}

/* ------------------------------------------------------------------------
 * Unit icosahedron with inradius 1 (src/main.ts:10-25): vertex table in
 * double; the float build rounds each coordinate to binary32 exactly as the
 * reference's Float32Array does.
 * ---------------------------------------------------------------------- */
static const int ico_idx[60] = {0, 11, 5, 0, 5,  1,  0, 1, 7, 0, 7,  10, 0, 10, 11,
                                1, 5,  9, 5, 11, 4,  11, 10, 2, 10, 7, 6, 7, 1, 8,
                                3, 9,  4, 3, 4,  2,  3, 2, 6, 3, 6,  8,  3, 8,  9,
                                4, 9,  5, 2, 4,  11, 6, 2, 10, 8, 6, 7, 9, 8, 1};

static void ico_vertices_d(double v[36]) {
  double rr = (3.0 + sqrt(5.0)) / (2.0 * sqrt(3.0));
  double ss = 1.0 / rr;
  double tt = (1.0 + sqrt(5.0)) / (2.0 * rr);
  double t[36] = {-ss, tt,  0,   ss,  tt, 0,   -ss, -tt, 0,   ss,  -tt, 0,
                  0,   -ss, tt,  0,   ss, tt,  0,   -ss, -tt, 0,   ss,  -tt,
                  tt,  0,   -ss, tt,  0,  ss,  -tt, 0,   -ss, -tt, 0,   ss};
  memcpy(v, t, sizeof t);
}

/* ------------------------------------------------------------------------
 * The REAL-generic part: proxies, BVH, traversal, shading, compositing.
 * ---------------------------------------------------------------------- */
#define REAL float
#define SFX(name) name##_f32
#define OR_IS_F32 1
#include "gt_oracle_impl.inc"
#undef REAL
#undef SFX
#undef OR_IS_F32

#define REAL double
#define SFX(name) name##_f64
#define OR_IS_F32 0
#include "gt_oracle_impl.inc"
#undef REAL
#undef SFX
#undef OR_IS_F32
