// Scene loading on the device: the reference's `.splat` and PLY readers
// (src/splat_format.rs:18-44, src/ply.rs:104-379) and Scene::finalize
// (src/scene.rs:62-94) with the activation (exp scales, sigmoid opacity,
// base colour from f_dc, quaternion normalisation, opacity clamp, 3D
// covariance) done by one thread per splat, written straight into the
// renderer's FP32 or FP16 device layout. The host parses only the PLY header
// (text) and copies the file's records to the device once.
//
// Arithmetic follows the reference's f32 expressions operation by operation
// (this file is built with --fmad=false): a property is read as f64 and
// converted to f32 (ScalarType::read + `as f32`), colours are f_dc * SH_C0 +
// 0.5 (or u8 / 255), opacities 1 / (1 + exp(-x)), scales exp(x), and exp and
// ln are evaluated in double and rounded to f32 (the correctly rounded f32
// result, which the platform's f32 exp/ln return), so the device scene
// equals what splat_cuda_create uploads for the host-parsed, finalized scene.
#include <cuda_fp16.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "geom.cuh"
#include "handle.h"

#define SPLAT_API extern "C" __attribute__((visibility("default")))

using namespace splat;

namespace {

// PLY scalar types (src/ply.rs:26-35) and their sizes.
enum : uint8_t { kNone = 0, kI8, kU8, kI16, kU16, kI32, kU32, kF32, kF64 };
uint32_t type_size(uint8_t t) {
  switch (t) {
    case kI8: case kU8: return 1;
    case kI16: case kU16: return 2;
    case kI32: case kU32: case kF32: return 4;
    case kF64: return 8;
    default: return 0;
  }
}

struct Col {
  uint32_t off;
  uint32_t type;  // kNone: absent
};

constexpr int kMaxRest = 45;

// Where each property the reader uses sits in a vertex record.
struct Layout {
  uint32_t stride;
  uint32_t big_endian;
  Col pos[3], dc[3], rgb[3], opacity, scale[3], rot[4];
  Col rest[kMaxRest];
  uint32_t per_channel;  // rest coefficients per channel used (degree's)
  float rgb_scale;       // 1/255 for u8 colours, else 1
  uint32_t splat_format; // 1: the 32-byte .splat record instead
};

// src/sh.rs:5
constexpr float kShC0 = 0.2820948f;

__device__ __forceinline__ double read_scalar(const uint8_t* p, uint32_t type, bool be) {
  const uint32_t n = type == kF64 ? 8 : (type == kI32 || type == kU32 || type == kF32 ? 4 : (type <= kU8 ? 1 : 2));
  uint64_t v = 0;
  for (uint32_t i = 0; i < n; i++) v |= (uint64_t)p[be ? n - 1 - i : i] << (8 * i);
  switch (type) {
    case kI8: return (double)(int8_t)(uint8_t)v;
    case kU8: return (double)(uint8_t)v;
    case kI16: return (double)(int16_t)(uint16_t)v;
    case kU16: return (double)(uint16_t)v;
    case kI32: return (double)(int32_t)(uint32_t)v;
    case kU32: return (double)(uint32_t)v;
    case kF32: return (double)__uint_as_float((uint32_t)v);
    default: return __longlong_as_double((long long)v);
  }
}

// f32 exp and ln, correctly rounded (double evaluation, one rounding).
__device__ __forceinline__ float exp_f32(float x) { return (float)exp((double)x); }
__device__ __forceinline__ float ln_f32(float x) { return (float)log((double)x); }

// One splat of the file, parsed and finalized.
struct Parsed {
  float pos[3], color[3], opacity, scale[3], q[4];  // q = x, y, z, w (unit)
};

__device__ __forceinline__ void parse_splat(const uint8_t* __restrict__ body, const Layout& L, uint64_t i,
                                            Parsed& s, float* rest /* per_channel * 3, RGB innermost */) {
  if (L.splat_format) {
    // src/splat_format.rs:33-41
    const uint8_t* r = body + i * 32;
    for (int k = 0; k < 3; k++) s.pos[k] = (float)read_scalar(r + 4 * k, kF32, false);
    for (int k = 0; k < 3; k++) s.scale[k] = fabsf((float)read_scalar(r + 12 + 4 * k, kF32, false));
    for (int k = 0; k < 3; k++) s.color[k] = __fdiv_rn((float)r[24 + k], 255.0f);
    s.opacity = __fdiv_rn((float)r[27], 255.0f);
    s.q[0] = __fdiv_rn((float)r[29] - 128.0f, 128.0f);
    s.q[1] = __fdiv_rn((float)r[30] - 128.0f, 128.0f);
    s.q[2] = __fdiv_rn((float)r[31] - 128.0f, 128.0f);
    s.q[3] = __fdiv_rn((float)r[28] - 128.0f, 128.0f);
  } else {
    // src/ply.rs:268-307 (emit)
    const uint8_t* r = body + i * L.stride;
    const bool be = L.big_endian != 0;
    auto f = [&](const Col& c) { return (float)read_scalar(r + c.off, c.type, be); };
    for (int k = 0; k < 3; k++) s.pos[k] = f(L.pos[k]);
    if (L.dc[0].type) {
      for (int k = 0; k < 3; k++) s.color[k] = f(L.dc[k]) * kShC0 + 0.5f;
    } else if (L.rgb[0].type) {
      for (int k = 0; k < 3; k++) s.color[k] = f(L.rgb[k]) * L.rgb_scale;
    } else {
      for (int k = 0; k < 3; k++) s.color[k] = 0.8f;
    }
    s.opacity = L.opacity.type ? 1.0f / (1.0f + exp_f32(-f(L.opacity))) : 1.0f;
    for (int k = 0; k < 3; k++) s.scale[k] = L.scale[0].type ? exp_f32(f(L.scale[k])) : 0.01f;
    if (L.rot[0].type) {  // 3DGS stores (w, x, y, z)
      s.q[0] = f(L.rot[1]);
      s.q[1] = f(L.rot[2]);
      s.q[2] = f(L.rot[3]);
      s.q[3] = f(L.rot[0]);
    } else {
      s.q[0] = s.q[1] = s.q[2] = 0.0f;
      s.q[3] = 1.0f;
    }
    // f_rest is channel-major: all R coefficients, then G, then B.
    const uint32_t pc = L.per_channel;
    for (uint32_t k = 0; k < pc; k++)
      for (int ch = 0; ch < 3; ch++) rest[3 * k + ch] = f(L.rest[ch * pc + k]);
  }
  // Scene::finalize (src/scene.rs:72-86)
  normalize_quat(s.q[0], s.q[1], s.q[2], s.q[3]);
  s.opacity = isfinite(s.opacity) ? fminf(fmaxf(s.opacity, 0.0f), 1.0f) : 0.0f;
}

// k = sqrt(2 ln(opacity / ALPHA_MIN)), the bbox radius both upload paths store.
__device__ __forceinline__ float bbox_k(float o) {
  return o < kAlphaMin ? 0.0f : sqrtf(2.0f * ln_f32(o / kAlphaMin));
}

__device__ __forceinline__ uint16_t half_bits(float v) { return __half_as_ushort(__float2half_rn(v)); }

// FP32 layout: pos_op, cov_a, cov_b (with k), colour planes, SH planes.
__global__ void k_decode_fp32(const uint8_t* __restrict__ body, Layout L, uint64_t n, float4* __restrict__ pos_op,
                              float4* __restrict__ cov_a, float4* __restrict__ cov_b, float* __restrict__ color,
                              float* __restrict__ sh) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    Parsed s;
    float rest[kMaxRest];
    parse_splat(body, L, i, s, rest);
    float c[6];
    covariance_rs(s.scale, s.q[0], s.q[1], s.q[2], s.q[3], c);
    pos_op[i] = make_float4(s.pos[0], s.pos[1], s.pos[2], s.opacity);
    cov_a[i] = make_float4(c[0], c[1], c[2], c[3]);
    cov_b[i] = make_float4(c[4], c[5], bbox_k(s.opacity), 0.0f);
    for (int k = 0; k < 3; k++) color[k * n + i] = s.color[k];
    for (uint32_t k = 0; k < 3 * L.per_channel; k++) sh[(uint64_t)k * n + i] = rest[k];
  }
}

// FP16 layout: pos_k (k from the stored half opacity), geom16 (scale,
// rotation, opacity halves), planes of halves: base colour, then the rest.
__global__ void k_decode_fp16(const uint8_t* __restrict__ body, Layout L, uint64_t n, float4* __restrict__ pos_k,
                              uint4* __restrict__ geom16, uint16_t* __restrict__ sh16) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    Parsed s;
    float rest[kMaxRest];
    parse_splat(body, L, i, s, rest);
    const uint16_t ob = half_bits(s.opacity);
    const float o = fminf(fmaxf(__half2float(__ushort_as_half(ob)), 0.0f), 1.0f);
    pos_k[i] = make_float4(s.pos[0], s.pos[1], s.pos[2], bbox_k(o));
    const uint16_t sc0 = half_bits(s.scale[0]), sc1 = half_bits(s.scale[1]), sc2 = half_bits(s.scale[2]);
    const uint16_t q0 = half_bits(s.q[0]), q1 = half_bits(s.q[1]), q2 = half_bits(s.q[2]), q3 = half_bits(s.q[3]);
    geom16[i] = make_uint4(sc0 | ((uint32_t)sc1 << 16), sc2 | ((uint32_t)q0 << 16), q1 | ((uint32_t)q2 << 16),
                           q3 | ((uint32_t)ob << 16));
    for (int k = 0; k < 3; k++) sh16[k * n + i] = half_bits(s.color[k]);
    for (uint32_t k = 0; k < 3 * L.per_channel; k++) sh16[(uint64_t)(3 + k) * n + i] = half_bits(rest[k]);
  }
}

// ---- host: PLY header (src/ply.rs:104-235) ----------------------------------

struct Prop {
  std::string name;
  uint8_t type;
  bool list;
};
struct Elem {
  std::string name;
  uint64_t count;
  std::vector<Prop> props;
};

uint8_t parse_type(const std::string& s) {
  if (s == "char" || s == "int8") return kI8;
  if (s == "uchar" || s == "uint8") return kU8;
  if (s == "short" || s == "int16") return kI16;
  if (s == "ushort" || s == "uint16") return kU16;
  if (s == "int" || s == "int32") return kI32;
  if (s == "uint" || s == "uint32") return kU32;
  if (s == "float" || s == "float32") return kF32;
  if (s == "double" || s == "float64") return kF64;
  return kNone;
}

int degree_from_rest_count(size_t rest) {
  for (int d = 0; d <= 3; d++)
    if (3 * ((d + 1) * (d + 1) - 1) == (int)rest) return d;
  return -1;
}

struct Decoded {
  Layout layout{};
  uint64_t n = 0;
  uint32_t degree = 0;
  std::vector<uint8_t> ascii_rows;  // ASCII bodies: rows of f64 values
  const uint8_t* body = nullptr;    // binary bodies: the vertex records in the file
  size_t body_bytes = 0;
};

int parse_ply(const uint8_t* data, size_t bytes, Decoded& out, std::string& err) {
  static const char kEnd[] = "end_header";
  const size_t scan = std::min<size_t>(bytes, (size_t)1 << 20);
  size_t pos = (size_t)-1;
  for (size_t i = 0; i + 10 <= scan; i++)
    if (std::memcmp(data + i, kEnd, 10) == 0) {
      pos = i;
      break;
    }
  if (pos == (size_t)-1) {
    err = "PLY header missing end_header";
    return SPLAT_ERR_INVALID_ARG;
  }
  size_t body = pos + 10;
  while (body < bytes && data[body] != '\n') body++;
  body++;
  std::vector<std::string> lines;
  {
    std::string cur;
    for (size_t i = 0; i < pos; i++) {
      const char c = (char)data[i];
      if (c == '\n') {
        lines.push_back(cur);
        cur.clear();
      } else if (c != '\r') {
        cur.push_back(c);
      }
    }
    lines.push_back(cur);
  }
  auto words = [](const std::string& l) {
    std::vector<std::string> w;
    size_t i = 0;
    while (i < l.size()) {
      while (i < l.size() && isspace((unsigned char)l[i])) i++;
      size_t j = i;
      while (j < l.size() && !isspace((unsigned char)l[j])) j++;
      if (j > i) w.push_back(l.substr(i, j - i));
      i = j;
    }
    return w;
  };
  if (lines.empty() || words(lines[0]) != std::vector<std::string>{"ply"}) {
    err = "not a PLY file (missing 'ply' magic)";
    return SPLAT_ERR_INVALID_ARG;
  }
  int format = -1;  // 0 ascii, 1 le, 2 be
  std::vector<Elem> elems;
  for (size_t li = 1; li < lines.size(); li++) {
    const auto w = words(lines[li]);
    if (w.empty() || w[0] == "comment" || w[0] == "obj_info") continue;
    if (w[0] == "format") {
      const std::string f = w.size() > 1 ? w[1] : "";
      if (f == "ascii") format = 0;
      else if (f == "binary_little_endian") format = 1;
      else if (f == "binary_big_endian") format = 2;
      else {
        err = "unsupported PLY format " + f;
        return SPLAT_ERR_INVALID_ARG;
      }
    } else if (w[0] == "element") {
      if (w.size() < 3) {
        err = "element without name or count";
        return SPLAT_ERR_INVALID_ARG;
      }
      char* endp = nullptr;
      const unsigned long long c = strtoull(w[2].c_str(), &endp, 10);
      if (!endp || *endp) {
        err = "bad element count";
        return SPLAT_ERR_INVALID_ARG;
      }
      elems.push_back(Elem{w[1], (uint64_t)c, {}});
    } else if (w[0] == "property") {
      if (elems.empty()) {
        err = "property before element";
        return SPLAT_ERR_INVALID_ARG;
      }
      Prop p{};
      if (w.size() >= 2 && w[1] == "list") {
        if (w.size() < 5 || !parse_type(w[2]) || !parse_type(w[3])) {
          err = "unsupported PLY property type";
          return SPLAT_ERR_INVALID_ARG;
        }
        p = Prop{w[4], parse_type(w[3]), true};
      } else {
        if (w.size() < 3 || !parse_type(w[1])) {
          err = "unsupported PLY property type '" + (w.size() > 1 ? w[1] : std::string()) + "'";
          return SPLAT_ERR_INVALID_ARG;
        }
        p = Prop{w[2], parse_type(w[1]), false};
      }
      elems.back().props.push_back(p);
    } else {
      err = "unexpected PLY header keyword '" + w[0] + "'";
      return SPLAT_ERR_INVALID_ARG;
    }
  }
  if (format < 0) {
    err = "PLY header has no format line";
    return SPLAT_ERR_INVALID_ARG;
  }
  size_t vi = elems.size();
  for (size_t i = 0; i < elems.size(); i++)
    if (elems[i].name == "vertex") {
      vi = i;
      break;
    }
  if (vi == elems.size()) {
    err = "PLY has no vertex element";
    return SPLAT_ERR_INVALID_ARG;
  }
  uint64_t offset = body;
  for (size_t i = 0; i < vi; i++) {
    bool list = false;
    uint64_t stride = 0;
    for (const auto& p : elems[i].props) {
      list = list || p.list;
      stride += type_size(p.type);
    }
    if (format == 0 || list) {
      err = "PLY element '" + elems[i].name + "' before vertex is not supported";
      return SPLAT_ERR_UNSUPPORTED;
    }
    offset += stride * elems[i].count;
  }
  const Elem& el = elems[vi];
  std::unordered_map<std::string, size_t> idx;
  for (size_t i = 0; i < el.props.size(); i++) idx.emplace(el.props[i].name, i);
  for (const auto& p : el.props)
    if (p.name.rfind("packed_", 0) == 0) {
      err = "compressed PLY (SuperSplat packed format) is not supported; decompress it first";
      return SPLAT_ERR_UNSUPPORTED;
    }
  const bool ascii = format == 0;
  // Byte offset of each property in a record (ASCII rows hold f64 values).
  std::vector<uint32_t> offs(el.props.size());
  uint32_t stride = 0;
  for (size_t i = 0; i < el.props.size(); i++) {
    offs[i] = stride;
    stride += ascii ? 8u : type_size(el.props[i].type);
  }
  Layout& L = out.layout;
  L.stride = stride;
  L.big_endian = format == 2;
  auto col = [&](const std::string& name) -> Col {
    auto it = idx.find(name);
    if (it == idx.end()) return Col{0, kNone};
    return Col{offs[it->second], ascii ? (uint32_t)kF64 : (uint32_t)el.props[it->second].type};
  };
  const char* xyz[3] = {"x", "y", "z"};
  for (int k = 0; k < 3; k++) {
    L.pos[k] = col(xyz[k]);
    if (!L.pos[k].type) {
      err = std::string("PLY vertex missing '") + xyz[k] + "'";
      return SPLAT_ERR_INVALID_ARG;
    }
  }
  auto all3 = [&](const char* a, const char* b, const char* c, Col* dst) {
    const Col x = col(a), y = col(b), z = col(c);
    if (x.type && y.type && z.type) {
      dst[0] = x;
      dst[1] = y;
      dst[2] = z;
    }
  };
  all3("f_dc_0", "f_dc_1", "f_dc_2", L.dc);
  all3("red", "green", "blue", L.rgb);
  all3("scale_0", "scale_1", "scale_2", L.scale);
  {
    const Col r0 = col("rot_0"), r1 = col("rot_1"), r2 = col("rot_2"), r3 = col("rot_3");
    if (r0.type && r1.type && r2.type && r3.type) {
      L.rot[0] = r0;
      L.rot[1] = r1;
      L.rot[2] = r2;
      L.rot[3] = r3;
    }
  }
  L.opacity = col("opacity");
  L.rgb_scale = (L.rgb[0].type && el.props[idx["red"]].type == kU8) ? 1.0f / 255.0f : 1.0f;
  std::vector<Col> rest;
  while (true) {
    const Col c = col("f_rest_" + std::to_string(rest.size()));
    if (!c.type) break;
    rest.push_back(c);
  }
  const int deg = degree_from_rest_count(rest.size());
  out.degree = deg < 0 ? 0u : (uint32_t)deg;
  L.per_channel = (out.degree + 1) * (out.degree + 1) - 1;
  for (uint32_t k = 0; k < 3 * L.per_channel; k++) L.rest[k] = rest[k];
  out.n = el.count;
  if (ascii) {
    // The body as rows of f64 values: the same device decode then reads them.
    const char* p = reinterpret_cast<const char*>(data) + std::min<uint64_t>(offset, bytes);
    const char* end = reinterpret_cast<const char*>(data) + bytes;
    const uint64_t nreserve = std::min<uint64_t>(el.count, bytes);
    out.ascii_rows.reserve(nreserve * stride);
    std::string tok;
    auto next = [&](double& v) -> bool {
      while (p < end && isspace((unsigned char)*p)) p++;
      if (p >= end) return false;
      const char* s0 = p;
      while (p < end && !isspace((unsigned char)*p)) p++;
      tok.assign(s0, p);
      char* e2 = nullptr;
      v = strtod(tok.c_str(), &e2);
      return e2 && *e2 == 0;
    };
    for (uint64_t v = 0; v < el.count; v++)
      for (const auto& prop : el.props) {
        double x = 0.0;
        if (!next(x)) {
          err = "ASCII PLY truncated at vertex " + std::to_string(v);
          return SPLAT_ERR_INVALID_ARG;
        }
        if (prop.list) {
          const uint64_t cnt = (uint64_t)x;
          for (uint64_t c = 0; c < cnt; c++)
            if (!next(x)) {
              err = "ASCII PLY truncated at vertex " + std::to_string(v);
              return SPLAT_ERR_INVALID_ARG;
            }
          x = 0.0;
        }
        uint8_t b[8];
        std::memcpy(b, &x, 8);
        out.ascii_rows.insert(out.ascii_rows.end(), b, b + 8);
      }
    out.layout.big_endian = 0;
    out.body = out.ascii_rows.data();
    out.body_bytes = out.ascii_rows.size();
  } else {
    for (const auto& p : el.props)
      if (p.list) {
        err = "list properties on vertices are not supported";
        return SPLAT_ERR_UNSUPPORTED;
      }
    const uint64_t need = offset + (uint64_t)stride * el.count;
    if (bytes < need || need < offset) {
      err = "PLY body truncated: need " + std::to_string(need) + " bytes, file has " + std::to_string(bytes);
      return SPLAT_ERR_INVALID_ARG;
    }
    out.body = data + offset;
    out.body_bytes = (size_t)stride * el.count;
  }
  return SPLAT_OK;
}

int decode_to_handle(const Decoded& dec, uint32_t precision, int device, splat_cuda_handle** out) {
  if (precision != SPLAT_PRECISION_FP32 && precision != SPLAT_PRECISION_FP16) {
    set_create_error("unknown scene precision");
    return SPLAT_ERR_UNSUPPORTED;
  }
  splat_scene_desc d{};
  d.n = dec.n;
  d.sh_degree = dec.degree;
  d.precision = precision;
  std::string err;
  splat_cuda_handle* h = nullptr;
  int rc = create_unfilled(&d, device, &h, &err);
  if (rc) {
    set_create_error(err);
    return rc;
  }
  if (dec.n) {
    uint8_t* body = nullptr;
    cudaError_t e = cudaMalloc(&body, std::max<size_t>(dec.body_bytes, 1));
    // On the decode's own stream: a cudaMemcpy from pageable memory may return
    // before its DMA lands, and that stream does not wait for the legacy one.
    if (e == cudaSuccess) e = cudaMemcpyAsync(body, dec.body, dec.body_bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
      const unsigned grid = (unsigned)std::min<uint64_t>((dec.n + 255) / 256, 16u * (uint64_t)h->num_sms);
      if (precision == SPLAT_PRECISION_FP32)
        k_decode_fp32<<<grid, 256, 0, h->stream>>>(body, dec.layout, dec.n, h->pos_op, h->cov_a, h->cov_b, h->color,
                                                  h->sh);
      else
        k_decode_fp16<<<grid, 256, 0, h->stream>>>(body, dec.layout, dec.n, h->pos_k, h->geom16, h->sh16);
      h->launches += 1;
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    if (body) cudaFree(body);
    if (e != cudaSuccess) {
      set_create_error(std::string("device decode: ") + cudaGetErrorString(e));
      splat_cuda_destroy(h);
      return e == cudaErrorMemoryAllocation ? SPLAT_ERR_OOM : SPLAT_ERR_DEVICE;
    }
    if ((rc = build_binning_order(h))) {
      set_create_error(h->err);
      splat_cuda_destroy(h);
      return rc;
    }
  }
  *out = h;
  return SPLAT_OK;
}

}  // namespace

SPLAT_API int splat_cuda_create_from_splat(const void* data, size_t bytes, uint32_t precision, int device,
                                           splat_cuda_handle** out) {
  if (!out) return SPLAT_ERR_INVALID_ARG;
  *out = nullptr;
  if (!data && bytes) {
    set_create_error("null data");
    return SPLAT_ERR_INVALID_ARG;
  }
  if (bytes % 32 != 0) {
    set_create_error(".splat file size " + std::to_string(bytes) + " is not a multiple of 32 bytes");
    return SPLAT_ERR_INVALID_ARG;
  }
  Decoded dec;
  dec.layout.splat_format = 1;
  dec.n = bytes / 32;
  dec.degree = 0;
  dec.body = static_cast<const uint8_t*>(data);
  dec.body_bytes = bytes;
  return decode_to_handle(dec, precision, device, out);
}

SPLAT_API int splat_cuda_create_from_ply(const void* data, size_t bytes, uint32_t precision, int device,
                                         splat_cuda_handle** out) {
  if (!out) return SPLAT_ERR_INVALID_ARG;
  *out = nullptr;
  if (!data) {
    set_create_error("null data");
    return SPLAT_ERR_INVALID_ARG;
  }
  Decoded dec;
  std::string err;
  const int rc = parse_ply(static_cast<const uint8_t*>(data), bytes, dec, err);
  if (rc) {
    set_create_error(err);
    return rc;
  }
  return decode_to_handle(dec, precision, device, out);
}
