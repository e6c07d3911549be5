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
 *   header (decodeHeader, :58-111): 50-byte chunks are read until the text
 *           holds "end_header" (a file ending inside that chunk throws); the
 *           '\n'-split, trimmed lines of those chunks are scanned up to a line
 *           equal to "end_header": "element vertex" -> count (first digit
 *           run, last line wins), "property" -> (type, name) = groups 2, 3 of
 *           the first match of (\w+)\s+(\w+)\s+(\w+); names in JS object-key
 *           order (array-index names ascending first, then insertion order; a
 *           repeated name keeps its place, takes the later type;
 *           "__proto__" adds nothing); data one byte after "end_header" (:103)
 *   per vertex, in key order: float -> f32 LE, uchar -> byte/255, other
 *           types not read and 0 bytes (:120-128)
 *   activation (in double, :225-235): scale = exp, quaternion / its norm,
 *           opacity = 1/(1+exp(-x))
 *   SH order (:188-196): sh[0] = f_dc_0..2; sh[i+1].rgb = f_rest_{rgb*n+i},
 *           n = #f_rest / 3; degree 0..3 (:136-148)
 *   std430 packing (src/GS_packing.ts:146-174,233-245): position @0,
 *           scale @16, rotation @32, opacity @48, sh[j] @64+16j;
 *           record size rounded up to 16.
 * Non-ASCII headers, missing float/uchar properties and short bodies are
 * errors (the reference packs NaN or throws there).
 * ---------------------------------------------------------------------- */
#define OR_MAX_PROPS 1024
#define OR_NAME 64
typedef struct {
  char name[OR_NAME];
  int kind; /* 1 float, 0 uchar, -1 other */
  int is_index;
  unsigned long long index;
  int order; /* insertion order */
} or_prop;

static int or_js_space(int c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }
static int or_js_word(int c) {
  return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_';
}

/* (\w+)\s+(\w+)\s+(\w+): leftmost match; returns 1 and the spans of groups 2, 3 */
static int or_prop_match(const char* s, size_t L, size_t* t0, size_t* t1, size_t* n0, size_t* n1) {
  for (size_t i = 0; i < L; ++i) {
    if (!or_js_word((unsigned char)s[i])) continue;
    size_t a = i;
    while (a < L && or_js_word((unsigned char)s[a])) ++a;
    size_t b = a;
    while (b < L && or_js_space((unsigned char)s[b])) ++b;
    if (b > a && b < L && or_js_word((unsigned char)s[b])) {
      size_t c = b;
      while (c < L && or_js_word((unsigned char)s[c])) ++c;
      size_t d = c;
      while (d < L && or_js_space((unsigned char)s[d])) ++d;
      if (d > c && d < L && or_js_word((unsigned char)s[d])) {
        size_t e = d;
        while (e < L && or_js_word((unsigned char)s[e])) ++e;
        *t0 = b;
        *t1 = c;
        *n0 = d;
        *n1 = e;
        return 1;
      }
    }
    i = a; /* the loop's ++i moves past the non-word character at a */
  }
  return 0;
}

static int or_array_index(const char* nm, unsigned long long* v) {
  size_t l = strlen(nm);
  if (l == 0 || l > 10) return 0;
  for (size_t i = 0; i < l; ++i)
    if (nm[i] < '0' || nm[i] > '9') return 0;
  if (nm[0] == '0' && l > 1) return 0;
  unsigned long long x = strtoull(nm, NULL, 10);
  if (x >= 4294967295ull) return 0;
  *v = x;
  return 1;
}

static int or_prop_cmp(const void* pa, const void* pb) {
  const or_prop* a = (const or_prop*)pa;
  const or_prop* b = (const or_prop*)pb;
  if (a->is_index != b->is_index) return a->is_index ? -1 : 1;
  if (a->is_index) return a->index < b->index ? -1 : (a->index > b->index ? 1 : 0);
  return a->order - b->order;
}

int or_ply_to_aos(const uint8_t* bytes, size_t len, uint32_t* n_out, uint32_t* deg_out,
                  uint32_t* stride_out, float* aos, double* act64) {
  size_t pos = (size_t)-1;
  for (size_t i = 0; i + 10 <= len; ++i)
    if (memcmp(bytes + i, "end_header", 10) == 0) {
      pos = i;
      break;
    }
  if (pos == (size_t)-1) return 1;
  const size_t chunk_end = (pos + 10 + 49) / 50 * 50;
  if (chunk_end > len) return 1;
  for (size_t i = 0; i < pos; ++i)
    if (bytes[i] >= 0x80) return 1;
  const size_t hdr_end = pos + 11;
  or_prop* props = (or_prop*)calloc(OR_MAX_PROPS, sizeof(or_prop));
  if (!props) return 7;
  int np = 0, next_order = 0;
  unsigned long long nvert = 0;
  int nvert_ok = 1;
  size_t ls = 0;
  for (;;) {
    size_t le = ls;
    while (le < chunk_end && bytes[le] != '\n') ++le;
    size_t a = ls, b = le;
    while (a < b && or_js_space(bytes[a])) ++a;
    while (b > a && or_js_space(bytes[b - 1])) --b;
    const char* p = (const char*)bytes + a;
    const size_t pl = b - a;
    if (pl >= 14 && memcmp(p, "element vertex", 14) == 0) {
      size_t d = 0;
      while (d < pl && !(p[d] >= '0' && p[d] <= '9')) ++d;
      if (d < pl) {
        size_t e = d;
        while (e < pl && p[e] >= '0' && p[e] <= '9') ++e;
        while (d + 1 < e && p[d] == '0') ++d; /* leading zeros */
        if (e - d > 12) {
          nvert_ok = 0;
        } else {
          char num[16];
          memcpy(num, p + d, e - d);
          num[e - d] = 0;
          nvert = strtoull(num, NULL, 10);
          nvert_ok = 1;
        }
      }
    } else if (pl >= 8 && memcmp(p, "property", 8) == 0) {
      size_t t0 = 0, t1 = 0, n0 = 0, n1 = 0;
      if (or_prop_match(p, pl, &t0, &t1, &n0, &n1) && n1 - n0 < OR_NAME && !(n1 - n0 == 9 && !memcmp(p + n0, "__proto__", 9))) {
        char nm[OR_NAME];
        memcpy(nm, p + n0, n1 - n0);
        nm[n1 - n0] = 0;
        int kind = (t1 - t0 == 5 && !memcmp(p + t0, "float", 5)) ? 1 : ((t1 - t0 == 5 && !memcmp(p + t0, "uchar", 5)) ? 0 : -1);
        int idx = -1;
        for (int i = 0; i < np; ++i)
          if (strcmp(props[i].name, nm) == 0) idx = i;
        if (idx < 0) {
          if (np >= OR_MAX_PROPS) {
            free(props);
            return 2;
          }
          idx = np++;
          snprintf(props[idx].name, OR_NAME, "%s", nm);
          props[idx].order = next_order++;
          props[idx].is_index = or_array_index(nm, &props[idx].index);
        }
        props[idx].kind = kind;
      } else if (n1 - n0 >= OR_NAME) {
        free(props);
        return 2;
      }
    } else if (pl == 10 && memcmp(p, "end_header", 10) == 0) {
      break;
    }
    if (le >= chunk_end) break;
    ls = le + 1;
  }
  if (!nvert_ok || nvert >= (1ull << 31)) {
    free(props);
    return 2;
  }
  qsort(props, (size_t)np, sizeof(or_prop), or_prop_cmp);
  char names[OR_MAX_PROPS][OR_NAME];
  int is_float[OR_MAX_PROPS];
  for (int i = 0; i < np; ++i) {
    memcpy(names[i], props[i].name, OR_NAME);
    is_float[i] = props[i].kind;
  }
  free(props);
  int n_rest = 0;
  for (int i = 0; i < np; ++i)
    if (strncmp(names[i], "f_rest_", 7) == 0) ++n_rest;
  double per_color_d = (double)n_rest / 3.0;
  double degf = sqrt(per_color_d + 1.0) - 1.0;
  if (!(degf == 0.0 || degf == 1.0 || degf == 2.0 || degf == 3.0)) return 3;
  int deg = (int)degf;
  int per_color = n_rest / 3;
  int n_sh = (deg + 1) * (deg + 1);
  /* struct: 64 bytes of header fields + n_sh vec3 at stride 16, size rounded to 16 */
  uint32_t stride = 64u + 16u * (uint32_t)n_sh;
  /* every required property must be read (float or uchar) */
  int ix[14];
  const char* want[14] = {"x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0",
                          "rot_1", "rot_2", "rot_3", "opacity", "f_dc_0", "f_dc_1", "f_dc_2"};
  for (int w = 0; w < 14; ++w) {
    ix[w] = -1;
    for (int i = 0; i < np; ++i)
      if (strcmp(names[i], want[w]) == 0 && is_float[i] >= 0) ix[w] = i;
    if (ix[w] < 0) return 5;
  }
  int rest_ix[45];
  for (int r = 0; r < 3 * per_color && r < 45; ++r) {
    char nm[32];
    snprintf(nm, sizeof nm, "f_rest_%d", r);
    rest_ix[r] = -1;
    for (int i = 0; i < np; ++i)
      if (strcmp(names[i], nm) == 0 && is_float[i] >= 0) rest_ix[r] = i;
    if (rest_ix[r] < 0) return 6;
  }
  /* bytes per vertex */
  size_t vbytes = 0;
  for (int i = 0; i < np; ++i) vbytes += is_float[i] == 1 ? 4 : (is_float[i] == 0 ? 1 : 0);
  if (nvert > 0 && (len - hdr_end) / vbytes < nvert) return 4;
  *n_out = (uint32_t)nvert;
  *deg_out = (uint32_t)deg;
  *stride_out = stride;
  if (!aos) return 0;
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
    double a8[8];
    a8[0] = 1.0 / (1.0 + exp(-v[ix[10]]));
    for (int c = 0; c < 3; ++c) a8[1 + c] = exp(v[ix[3 + c]]);
    double q0 = v[ix[6]], q1 = v[ix[7]], q2 = v[ix[8]], q3 = v[ix[9]];
    double nrm = sqrt(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
    a8[4] = q0 / nrm;
    a8[5] = q1 / nrm;
    a8[6] = q2 / nrm;
    a8[7] = q3 / nrm;
    if (act64) memcpy(act64 + 8 * g, a8, sizeof a8);
    for (int c = 0; c < 3; ++c) rec[4 + c] = (float)a8[1 + c];
    for (int c = 0; c < 4; ++c) rec[8 + c] = (float)a8[4 + c];
    rec[12] = (float)a8[0];
    for (int c = 0; c < 3; ++c) rec[16 + c] = (float)v[ix[11 + c]];
    for (int i = 0; i < per_color; ++i)
      for (int c = 0; c < 3; ++c) rec[16 + 4 * (i + 1) + c] = (float)v[rest_ix[c * per_color + i]];
  }
  free(v);
  return 0;
}

/* ------------------------------------------------------------------------
 * Anti-aliasing jitter (src/GS_shader.ts:6-31): getNewSeed is numPermutation
 * rounds of the TEA block cipher (Wheeler and Needham 1994) with the
 * reference's constants; rng is an LCG step whose low 24 bits are scaled to
 * [0, 1).
 * ---------------------------------------------------------------------- */
uint32_t or_new_seed(uint32_t p1, uint32_t p2, uint32_t rounds) {
  uint32_t s0 = 0, v0 = p1, v1 = p2;
  for (uint32_t r = 0; r < rounds; ++r) {
    s0 += 0x9e3779b9u;
    v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
    v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
  }
  return v0;
}

float or_rng(uint32_t* seed) {
  *seed = 1664525u * *seed + 1013904223u;
  return (float)(*seed & 0x00FFFFFFu) / (float)0x01000000;
}

/* ------------------------------------------------------------------------
 * Tone map (src/toneMapper.ts:15-24) into unorm8 RGBA: mode 0 shows hdr as
 * the reference's fragment shader does, mode 1 applies 1 - exp(-exposure
 * hdr), mode 2 also the 1/2.2 power (written as exp(log(x) / 2.2) with the
 * deterministic routines above); unorm8 clamps to [0, 1] and rounds c * 255
 * to nearest (ties to even); NaN gives 0.
 * ---------------------------------------------------------------------- */
static uint8_t or_unorm8(float c) {
  if (!(c > 0.0f)) return 0;
  if (c >= 1.0f) return 255;
  return (uint8_t)nearbyintf(c * 255.0f);
}

static float or_tone(float hdr, uint32_t mode, float exposure) {
  if (mode == 0) return hdr;
  float ldr = 1.0f - or_expf(-(exposure * hdr));
  if (mode == 1) return ldr;
  if (!(ldr > 0.0f)) return ldr;
  return or_expf((float)(or_log((double)ldr) / 2.2));
}

int or_tonemap(const float* rgba, uint64_t n, uint32_t mode, float exposure, uint8_t* out) {
  if (mode > 2) return 1;
  for (uint64_t i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) out[4 * i + c] = or_unorm8(or_tone(rgba[4 * i + c], mode, exposure));
    out[4 * i + 3] = 255;
  }
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
