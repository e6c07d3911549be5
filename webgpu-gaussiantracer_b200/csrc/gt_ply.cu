// gt_ply.cu — native 3DGS PLY ingest: header decode on the host, activation
// and std430 packing on the GPU.
//
// Replaces PackedGaussians (src/GS_ply.ts:39-253), which decodes, activates
// and packs every vertex through per-vertex JS objects on the main thread.
//
// Header (host), with the reference loader's rules (decodeHeader,
// src/GS_ply.ts:58-111; readRawVertex, :113-132):
//   * the header is read in 50-byte chunks until the text holds "end_header"
//     (:67-76); a file that ends inside that chunk is an error (the
//     reference's 50-byte Uint8Array view throws there);
//   * the lines of those chunks are split on '\n' and trimmed; a line that
//     starts with "element vertex" gives the vertex count (first run of
//     digits; the last such line wins), one that starts with "property" gives
//     (type, name) from the first match of (\w+)\s+(\w+)\s+(\w+) in it, and a
//     line equal to "end_header" ends the scan (:84-101);
//   * names are kept in JavaScript object-key order (propertyTypes is a plain
//     object): array-index names first in ascending order, then the others in
//     first-insertion order; a repeated name keeps its place and takes the
//     later type; "__proto__" creates no entry;
//   * the body starts one byte past the first "end_header" (:103); each vertex
//     is the properties in key order, float as little-endian f32 (4 bytes),
//     uchar as byte / 255 (1 byte); other types are not read and take no
//     bytes (:120-128);
//   * the SH degree follows from the number of f_rest_* names (:178-184) and
//     must be 0..3 (nShCoeffs throws otherwise, :136-148).
// Where the reference would pack undefined values (a missing property) or
// read past the end of the buffer, these functions return an error instead.
// The header must be ASCII (the reference decodes it as UTF-8 and takes byte
// offsets from the decoded text, which only agree for ASCII).
//
// Body (device): k_ply_pack stages tiles of vertex rows through shared memory
// with coalesced loads, activates them in double precision exactly as the
// reference's JS numbers do (:225-235: scale = exp(raw), quaternion divided
// by the square root of the sum of its squares, opacity = 1 / (1 + exp(-raw))),
// rounds each value to binary32 (DataView.setFloat32), and writes the std430
// GaussianParticle records (:199-207): position @0, scale @16, rotation @32,
// opacity @48, sh[j] @64 + 16 j (sh[0] = f_dc_0..2, sh[i+1] = (f_rest_i,
// f_rest_{n+i}, f_rest_{2n+i}), n = #f_rest / 3, :188-196); record size
// 64 + 16 (deg+1)^2 bytes, padding words zero.  Tiles of records are written
// back with 16-byte coalesced stores.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "gt_handles.h"
#include "gt_internal.cuh"

namespace gt {

// Field descriptors of the packed words: byte offset in the vertex row, with
// bit 31 set for a uchar property.
constexpr uint32_t kPlyUchar = 0x80000000u;
constexpr int kPlyFields = 11 + 48;  // x y z, scale_0..2, rot_0..3, opacity, 16 x rgb
constexpr uint32_t kPlyMaxRow = 32768;

struct PlyLayout {
  uint64_t n = 0;
  uint64_t data_offset = 0;
  uint32_t degree = 0, n_sh = 1, stride = 80, row_bytes = 0, n_props = 0;
  uint32_t field[kPlyFields] = {};
};

struct PlyFields {
  uint32_t field[kPlyFields];
  uint32_t row_bytes, stride, n_sh, rows_per_tile;
};

// ------------------------------------------------------------- host decode
static bool js_space(unsigned char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }
static bool js_word(unsigned char c) {
  return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_';
}

// Canonical array-index string ("0" or no leading zero, value < 2^32 - 1).
static bool array_index(const std::string& s, uint64_t* v) {
  if (s.empty() || s.size() > 10) return false;
  if (s[0] == '0') {
    if (s.size() != 1) return false;
    *v = 0;
    return true;
  }
  uint64_t x = 0;
  for (char c : s) {
    if (c < '0' || c > '9') return false;
    x = x * 10 + (uint64_t)(c - '0');
  }
  if (x >= 4294967295ull) return false;
  *v = x;
  return true;
}

// First match of (\w+)\s+(\w+)\s+(\w+) in `line`: groups 2 and 3.  Word and
// space classes are disjoint, so the first group always runs to the end of
// its word, and the leftmost match starts at the first word followed by
// space, word, space, word.
static bool property_match(const std::string& line, std::string* type, std::string* name) {
  const size_t L = line.size();
  size_t i = 0;
  while (i < L) {
    if (!js_word((unsigned char)line[i])) {
      ++i;
      continue;
    }
    size_t a = i;
    while (a < L && js_word((unsigned char)line[a])) ++a;  // group 1 = [i, a)
    size_t b = a;
    while (b < L && js_space((unsigned char)line[b])) ++b;
    if (b > a && b < L && js_word((unsigned char)line[b])) {
      size_t c = b;
      while (c < L && js_word((unsigned char)line[c])) ++c;  // group 2 = [b, c)
      size_t d = c;
      while (d < L && js_space((unsigned char)line[d])) ++d;
      if (d > c && d < L && js_word((unsigned char)line[d])) {
        size_t e = d;
        while (e < L && js_word((unsigned char)line[e])) ++e;  // group 3 = [d, e)
        *type = line.substr(b, c - b);
        *name = line.substr(d, e - d);
        return true;
      }
    }
    i = a;  // every start inside this word fails the same way
  }
  return false;
}

static Err decode_ply(const uint8_t* buf, uint64_t len, PlyLayout* out) {
  static const char kEnd[] = "end_header";
  uint64_t pos = UINT64_MAX;
  for (uint64_t i = 0; i + 10 <= len; ++i)
    if (memcmp(buf + i, kEnd, 10) == 0) {
      pos = i;
      break;
    }
  if (pos == UINT64_MAX) return Err{GT_ERR_INVALID_ARG, "PLY: no end_header in the buffer"};
  // chunks of 50 bytes up to the one that completes "end_header"
  const uint64_t chunk_end = (pos + 10 + 49) / 50 * 50;
  if (chunk_end > len)
    return Err{GT_ERR_INVALID_ARG,
               "PLY: the file ends inside the 50-byte header chunk that holds end_header (the reference loader "
               "throws here)"};
  for (uint64_t i = 0; i < pos; ++i)
    if (buf[i] >= 0x80) return Err{GT_ERR_INVALID_ARG, "PLY: the header is not ASCII"};

  struct Prop {
    std::string name, type;
  };
  std::vector<Prop> named;            // non-index names, insertion order
  std::map<uint64_t, Prop> indexed;   // array-index names, ascending
  uint64_t count = 0;
  bool count_ok = true;
  uint64_t ls = 0;
  while (ls <= chunk_end) {
    uint64_t le = ls;
    while (le < chunk_end && buf[le] != '\n') ++le;
    uint64_t a = ls, b = le;
    while (a < b && js_space(buf[a])) ++a;
    while (b > a && js_space(buf[b - 1])) --b;
    std::string line((const char*)buf + a, (size_t)(b - a));
    if (line.compare(0, 14, "element vertex") == 0) {
      size_t d = 0;
      while (d < line.size() && !(line[d] >= '0' && line[d] <= '9')) ++d;
      if (d < line.size()) {
        size_t e = d;
        while (e < line.size() && line[e] >= '0' && line[e] <= '9') ++e;
        std::string digits = line.substr(d, e - d);
        size_t nz = digits.find_first_not_of('0');
        digits = nz == std::string::npos ? "0" : digits.substr(nz);
        if (digits.size() > 12) {
          count_ok = false;
        } else {
          count_ok = true;
          count = strtoull(digits.c_str(), nullptr, 10);
        }
      }
    } else if (line.compare(0, 8, "property") == 0) {
      std::string type, name;
      if (property_match(line, &type, &name) && name != "__proto__") {
        uint64_t idx;
        if (array_index(name, &idx)) {
          indexed[idx] = Prop{name, type};
        } else {
          auto it = std::find_if(named.begin(), named.end(), [&](const Prop& p) { return p.name == name; });
          if (it != named.end())
            it->type = type;
          else
            named.push_back(Prop{name, type});
        }
      }
    } else if (line == kEnd) {
      break;
    }
    if (le >= chunk_end) break;
    ls = le + 1;
  }
  if (!count_ok || count >= (1ull << 31)) return Err{GT_ERR_INVALID_ARG, "PLY: at most 2^31 - 1 vertices"};

  std::vector<Prop> props;
  for (auto& kv : indexed) props.push_back(kv.second);
  for (auto& p : named) props.push_back(p);

  uint32_t n_rest = 0;
  for (auto& p : props)
    if (p.name.compare(0, 7, "f_rest_") == 0) ++n_rest;
  const double per_color = (double)n_rest / 3.0;
  const double degf = sqrt(per_color + 1.0) - 1.0;
  if (!(degf == 0.0 || degf == 1.0 || degf == 2.0 || degf == 3.0)) {
    char msg[96];
    snprintf(msg, sizeof msg, "PLY: unsupported SH degree (%u f_rest_ properties)", n_rest);
    return Err{GT_ERR_INVALID_ARG, msg};
  }
  PlyLayout L;
  L.n = count;
  L.data_offset = pos + 11;
  L.degree = (uint32_t)degf;
  L.n_sh = (L.degree + 1) * (L.degree + 1);
  L.stride = 64u + 16u * L.n_sh;
  L.n_props = (uint32_t)props.size();
  // row layout: float and uchar properties in key order
  std::map<std::string, uint32_t> where;
  uint64_t off = 0;
  for (auto& p : props) {
    if (p.type == "float") {
      where[p.name] = (uint32_t)off;
      off += 4;
    } else if (p.type == "uchar") {
      where[p.name] = (uint32_t)off | kPlyUchar;
      off += 1;
    }
    if (off > kPlyMaxRow) return Err{GT_ERR_INVALID_ARG, "PLY: vertex rows larger than 32 KB"};
  }
  L.row_bytes = (uint32_t)off;
  auto need = [&](const std::string& nm, uint32_t* slot) -> Err {
    auto it = where.find(nm);
    if (it == where.end())
      return Err{GT_ERR_INVALID_ARG, "PLY: missing float/uchar vertex property " + nm};
    *slot = it->second;
    return Err{};
  };
  const char* base[11] = {"x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3",
                          "opacity"};
  for (int f = 0; f < 11; ++f) {
    Err e = need(base[f], &L.field[f]);
    if (e.code != GT_OK) return e;
  }
  const uint32_t per = n_rest / 3;
  for (uint32_t j = 0; j < L.n_sh; ++j)
    for (uint32_t c = 0; c < 3; ++c) {
      std::string nm = j == 0 ? "f_dc_" + std::to_string(c) : "f_rest_" + std::to_string(c * per + (j - 1));
      Err e = need(nm, &L.field[11 + 3 * j + c]);
      if (e.code != GT_OK) return e;
    }
  if (L.n > 0 && (len - L.data_offset) / L.row_bytes < L.n)
    return Err{GT_ERR_INVALID_ARG, "PLY: the vertex data is shorter than the header says"};
  *out = L;
  return Err{};
}

// ----------------------------------------------------------------- device
__device__ __forceinline__ double ply_value(const uint8_t* row, uint32_t f) {
  const uint32_t o = f & ~kPlyUchar;
  if (f & kPlyUchar) return (double)row[o] / 255.0;
  const uint32_t bits = (uint32_t)row[o] | ((uint32_t)row[o + 1] << 8) | ((uint32_t)row[o + 2] << 16) |
                        ((uint32_t)row[o + 3] << 24);
  return (double)__uint_as_float(bits);
}

// Packed word w of a record from its vertex row.
__device__ __forceinline__ float ply_word(const uint8_t* row, const PlyFields& F, uint32_t w) {
  if (w < 3) return __double2float_rn(ply_value(row, F.field[w]));
  if (w >= 4 && w < 7) return __double2float_rn(exp(ply_value(row, F.field[3 + (w - 4)])));
  if (w >= 8 && w < 12) {
    const double q0 = ply_value(row, F.field[6]), q1 = ply_value(row, F.field[7]);
    const double q2 = ply_value(row, F.field[8]), q3 = ply_value(row, F.field[9]);
    const double s = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(q0, q0), __dmul_rn(q1, q1)), __dmul_rn(q2, q2)),
                               __dmul_rn(q3, q3));
    const double norm = __dsqrt_rn(s);
    const double q = w == 8 ? q0 : w == 9 ? q1 : w == 10 ? q2 : q3;
    return __double2float_rn(__ddiv_rn(q, norm));
  }
  if (w == 12) {
    const double x = ply_value(row, F.field[10]);
    return __double2float_rn(__ddiv_rn(1.0, __dadd_rn(1.0, exp(-x))));
  }
  if (w >= 16) {
    const uint32_t j = (w - 16) >> 2, c = (w - 16) & 3u;
    if (c < 3 && j < F.n_sh) return __double2float_rn(ply_value(row, F.field[11 + 3 * j + c]));
  }
  return 0.0f;
}

// The activated values in double of vertex i: opacity, scale x y z, rotation
// w x y z (the reference's gaussianData numbers, src/GS_ply.ts:225-235), by
// the same operations as ply_word before its rounding to binary32.
__global__ void k_ply_act64(const uint8_t* __restrict__ body, uint64_t n, const __grid_constant__ PlyFields F,
                            double* __restrict__ act) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t* row = body + i * F.row_bytes;
  double* a = act + 8 * i;
  const double x = ply_value(row, F.field[10]);
  a[0] = __ddiv_rn(1.0, __dadd_rn(1.0, exp(-x)));
#pragma unroll
  for (int c = 0; c < 3; ++c) a[1 + c] = exp(ply_value(row, F.field[3 + c]));
  const double q0 = ply_value(row, F.field[6]), q1 = ply_value(row, F.field[7]);
  const double q2 = ply_value(row, F.field[8]), q3 = ply_value(row, F.field[9]);
  const double s = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(q0, q0), __dmul_rn(q1, q1)), __dmul_rn(q2, q2)),
                             __dmul_rn(q3, q3));
  const double norm = __dsqrt_rn(s);
  a[4] = __ddiv_rn(q0, norm);
  a[5] = __ddiv_rn(q1, norm);
  a[6] = __ddiv_rn(q2, norm);
  a[7] = __ddiv_rn(q3, norm);
}

// One tile of rows per iteration: coalesced loads of the rows into shared
// memory, one (row, word) item per thread step, coalesced 16-byte stores.
__global__ void __launch_bounds__(256) k_ply_pack(const uint8_t* __restrict__ body, uint64_t n,
                                                  const __grid_constant__ PlyFields F, float4* __restrict__ out) {
  extern __shared__ float4 smem[];
  const uint32_t R = F.rows_per_tile;
  const uint32_t in_words = (R * F.row_bytes + 15u) / 16u;  // float4 slots of the row tile
  uint8_t* rows_s = reinterpret_cast<uint8_t*>(smem);
  float* out_s = reinterpret_cast<float*>(smem + in_words);
  const uint32_t words = F.stride / 4u;
  const uint64_t n_tiles = (n + R - 1) / R;
  for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const uint64_t i0 = tile * R;
    const uint32_t rows = n - i0 < R ? (uint32_t)(n - i0) : R;
    const uint8_t* src = body + i0 * F.row_bytes;
    const uint32_t nbytes = rows * F.row_bytes;
    if ((F.row_bytes & 3u) == 0) {  // rows start on 4-byte boundaries (the body is 256-aligned)
      const uint32_t* s32 = reinterpret_cast<const uint32_t*>(src);
      uint32_t* d32 = reinterpret_cast<uint32_t*>(rows_s);
      for (uint32_t i = threadIdx.x; i < nbytes / 4u; i += blockDim.x) d32[i] = __ldg(s32 + i);
    } else {
      for (uint32_t i = threadIdx.x; i < nbytes; i += blockDim.x) rows_s[i] = __ldg(src + i);
    }
    __syncthreads();
    for (uint32_t it = threadIdx.x; it < rows * words; it += blockDim.x) {
      const uint32_t r = it / words, w = it - r * words;
      out_s[it] = ply_word(rows_s + (size_t)r * F.row_bytes, F, w);
    }
    __syncthreads();
    float4* dst = out + i0 * (F.stride / 16u);
    const float4* o4 = reinterpret_cast<const float4*>(out_s);
    for (uint32_t i = threadIdx.x; i < rows * (F.stride / 16u); i += blockDim.x) dst[i] = o4[i];
    __syncthreads();
  }
}

static uint32_t ply_rows_per_tile(const PlyLayout& L) {
  uint32_t per = L.row_bytes + L.stride + 16u;
  return std::max(1u, std::min(64u, 45056u / per));
}

// Packs n vertices of `body_dev` into `out_dev` (n * stride bytes, 16-aligned).
static Err launch_ply_pack(const PlyLayout& L, const uint8_t* body_dev, float* out_dev, int num_sms,
                           cudaStream_t st, uint64_t* launches) {
  if (L.n == 0) return Err{};
  PlyFields F;
  memcpy(F.field, L.field, sizeof F.field);
  F.row_bytes = L.row_bytes;
  F.stride = L.stride;
  F.n_sh = L.n_sh;
  F.rows_per_tile = ply_rows_per_tile(L);
  const uint32_t in_words = (F.rows_per_tile * F.row_bytes + 15u) / 16u;
  const size_t smem = 16u * (size_t)in_words + (size_t)F.rows_per_tile * F.stride;
  const uint64_t tiles = (L.n + F.rows_per_tile - 1) / F.rows_per_tile;
  const uint32_t grid = (uint32_t)std::min<uint64_t>(tiles, (uint64_t)num_sms * 8u);
  k_ply_pack<<<grid, 256, smem, st>>>(body_dev, L.n, F, reinterpret_cast<float4*>(out_dev));
  ++*launches;
  GT_CUDA_TRY(cudaGetLastError());
  return Err{};
}

// Uploads the body of a host PLY buffer and packs it into a new device
// buffer (*packed_dev, L.n * L.stride bytes); with act_dev also the
// activated values in double (8 per vertex) into a second new buffer.
static Err ply_to_device(gt_context* ctx, const uint8_t* data, const PlyLayout& L, float** packed_dev,
                         double** act_dev = nullptr) {
  *packed_dev = nullptr;
  if (act_dev) *act_dev = nullptr;
  if (L.n == 0) return Err{};
  uint8_t* body = nullptr;
  float* packed = nullptr;
  const uint64_t body_bytes = L.n * (uint64_t)L.row_bytes;
  GT_CUDA_TRY(cudaMalloc(&body, body_bytes));
  cudaError_t e = cudaMalloc(&packed, L.n * (uint64_t)L.stride);
  if (e == cudaSuccess) e = cudaMemcpyAsync(body, data + L.data_offset, body_bytes, cudaMemcpyHostToDevice, ctx->stream);
  Err r;
  if (e != cudaSuccess) {
    r = Err{e == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA,
            std::string("PLY upload: ") + cudaGetErrorString(e)};
  } else {
    r = launch_ply_pack(L, body, packed, ctx->num_sms, ctx->stream, &ctx->launches);
    if (r.code == GT_OK && act_dev) {
      double* act = nullptr;
      e = cudaMalloc(&act, L.n * 8 * sizeof(double));
      if (e != cudaSuccess) {
        r = Err{e == cudaErrorMemoryAllocation ? GT_ERR_OOM : GT_ERR_CUDA,
                std::string("PLY activations: ") + cudaGetErrorString(e)};
      } else {
        PlyFields F;
        memcpy(F.field, L.field, sizeof F.field);
        F.row_bytes = L.row_bytes;
        F.stride = L.stride;
        F.n_sh = L.n_sh;
        F.rows_per_tile = 1;
        k_ply_act64<<<(unsigned)((L.n + 255) / 256), 256, 0, ctx->stream>>>(body, L.n, F, act);
        ++ctx->launches;
        e = cudaGetLastError();
        if (e != cudaSuccess) {
          cudaFree(act);
          r = Err{GT_ERR_CUDA, std::string("PLY activations: ") + cudaGetErrorString(e)};
        } else {
          *act_dev = act;
        }
      }
    }
    if (r.code == GT_OK) {
      e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) r = Err{GT_ERR_CUDA, std::string("PLY pack: ") + cudaGetErrorString(e)};
    }
  }
  cudaFree(body);
  if (r.code != GT_OK) {
    cudaFree(packed);
    if (act_dev && *act_dev) {
      cudaFree(*act_dev);
      *act_dev = nullptr;
    }
    return r;
  }
  *packed_dev = packed;
  return Err{};
}

static void fill_info(const PlyLayout& L, gt_ply_info* info) {
  if (!info) return;
  memset(info, 0, sizeof *info);
  info->n_vertices = L.n;
  info->data_offset = L.data_offset;
  info->sh_degree = L.degree;
  info->record_stride = L.stride;
  info->row_bytes = L.row_bytes;
  info->n_properties = L.n_props;
}

static bool read_file(const char* path, std::vector<uint8_t>* out, std::string* err) {
  FILE* f = fopen(path, "rb");
  if (!f) {
    *err = std::string("cannot open ") + path;
    return false;
  }
  if (fseek(f, 0, SEEK_END) != 0) {
    fclose(f);
    *err = std::string("cannot seek ") + path;
    return false;
  }
  long sz = ftell(f);
  if (sz < 0) {
    fclose(f);
    *err = std::string("cannot size ") + path;
    return false;
  }
  rewind(f);
  out->resize((size_t)sz);
  size_t got = sz ? fread(out->data(), 1, (size_t)sz, f) : 0;
  fclose(f);
  if (got != (size_t)sz) {
    *err = std::string("short read of ") + path;
    return false;
  }
  return true;
}

}  // namespace gt

using namespace gt;

// ================================================================== C ABI
extern "C" gt_status gt_ply_parse_header(const void* data, uint64_t len, gt_ply_info* info) {
  if (!data && len) return api_fail(nullptr, GT_ERR_INVALID_ARG, "data is NULL");
  if (!info) return api_fail(nullptr, GT_ERR_INVALID_ARG, "info is NULL");
  PlyLayout L;
  Err e = decode_ply(static_cast<const uint8_t*>(data), len, &L);
  if (e.code != GT_OK) return api_fail(nullptr, e.code, e.msg);
  fill_info(L, info);
  return GT_OK;
}

extern "C" gt_status gt_ply_pack(gt_context* ctx, const void* data, uint64_t len, void* out_packed,
                                 uint64_t out_bytes, uint32_t flags, gt_ply_info* info) {
  if (!ctx) return api_fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (!data && len) return api_fail(ctx, GT_ERR_INVALID_ARG, "data is NULL");
  if (flags & GT_FLAG_INPUT_DEVICE) return api_fail(ctx, GT_ERR_UNSUPPORTED, "PLY data must be a host buffer");
  PlyLayout L;
  Err e = decode_ply(static_cast<const uint8_t*>(data), len, &L);
  if (e.code != GT_OK) return api_fail(ctx, e.code, e.msg);
  const uint64_t need = L.n * (uint64_t)L.stride;
  if (need > 0 && !out_packed) return api_fail(ctx, GT_ERR_INVALID_ARG, "out_packed is NULL");
  if (out_bytes < need) return api_fail(ctx, GT_ERR_INVALID_ARG, "out_packed is smaller than n * record_stride");
  if ((flags & GT_FLAG_OUTPUT_DEVICE) && ((uintptr_t)out_packed & 15u))
    return api_fail(ctx, GT_ERR_INVALID_ARG, "a device out_packed must be 16-byte aligned");
  fill_info(L, info);
  if (need == 0) return GT_OK;
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return api_fail(ctx, GT_ERR_CUDA, cudaGetErrorString(ce));
  cudaEventRecord(ctx->int0, ctx->stream);
  float* packed = nullptr;
  e = ply_to_device(ctx, static_cast<const uint8_t*>(data), L, &packed);
  if (e.code != GT_OK) return api_fail(ctx, e.code, e.msg);
  cudaEventRecord(ctx->int1, ctx->stream);
  ce = cudaMemcpyAsync(out_packed, packed, need,
                       (flags & GT_FLAG_OUTPUT_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       ctx->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
  cudaFree(packed);
  if (ce != cudaSuccess) return api_fail(ctx, GT_ERR_CUDA, std::string("PLY output copy: ") + cudaGetErrorString(ce));
  if (info) cudaEventElapsedTime(&info->ingest_ms, ctx->int0, ctx->int1);
  return GT_OK;
}

extern "C" gt_status gt_scene_create_from_ply(gt_context* ctx, const void* data, uint64_t len, double alpha_min,
                                              uint32_t flags, gt_scene** out, gt_ply_info* info) {
  if (!ctx) return api_fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (!out) return api_fail(ctx, GT_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  if (!data && len) return api_fail(ctx, GT_ERR_INVALID_ARG, "data is NULL");
  if (flags & GT_FLAG_INPUT_DEVICE) return api_fail(ctx, GT_ERR_UNSUPPORTED, "PLY data must be a host buffer");
  if (!(alpha_min > 0.0) || !(alpha_min < 1.0)) return api_fail(ctx, GT_ERR_INVALID_ARG, "alpha_min must be in (0, 1)");
  PlyLayout L;
  Err e = decode_ply(static_cast<const uint8_t*>(data), len, &L);
  if (e.code != GT_OK) return api_fail(ctx, e.code, e.msg);
  fill_info(L, info);
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce != cudaSuccess) return api_fail(ctx, GT_ERR_CUDA, cudaGetErrorString(ce));
  cudaEventRecord(ctx->int0, ctx->stream);
  float* packed = nullptr;
  double* act = nullptr;
  e = ply_to_device(ctx, static_cast<const uint8_t*>(data), L, &packed, &act);
  if (e.code != GT_OK) return api_fail(ctx, e.code, e.msg);
  cudaEventRecord(ctx->int1, ctx->stream);
  // the proxies come from the activated values in double, as the reference's do
  gt_status s = gt_scene_create_ex(ctx, packed, L.n, L.stride, alpha_min, act,
                                   (flags & GT_FLAG_FAST_BUILD) | GT_FLAG_INPUT_DEVICE, out);
  cudaFree(packed);
  cudaFree(act);
  if (s == GT_OK && info) cudaEventElapsedTime(&info->ingest_ms, ctx->int0, ctx->int1);
  return s;
}

extern "C" gt_status gt_scene_create_from_ply_file(gt_context* ctx, const char* path, double alpha_min,
                                                   uint32_t flags, gt_scene** out, gt_ply_info* info) {
  if (!ctx) return api_fail(nullptr, GT_ERR_INVALID_ARG, "context is NULL");
  if (!path) return api_fail(ctx, GT_ERR_INVALID_ARG, "path is NULL");
  if (!out) return api_fail(ctx, GT_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  std::vector<uint8_t> bytes;
  std::string err;
  if (!read_file(path, &bytes, &err)) return api_fail(ctx, GT_ERR_INVALID_ARG, err);
  return gt_scene_create_from_ply(ctx, bytes.data(), bytes.size(), alpha_min, flags, out, info);
}
