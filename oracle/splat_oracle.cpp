// ORACLE — test infrastructure only. Never linked into, loaded by or called
// from the product library (splat_b200/libsplat_cuda.so). Only tests/, the
// smoke check and bench.py's CPU-baseline leg load it, as the checker.
//
// A CPU restatement of farmerchris/splat's rasterizer hot path (crate
// `splat-tui`, Rust). The Rust crate cannot be built in this environment (no
// cargo/rustc, crates.io dependencies not vendored), so each function below
// restates the reference's algorithm in C++ with the reference's x86
// floating-point semantics: IEEE binary32, no fused multiply-add
// (-ffp-contract=off), no fast-math, the same operation order as the Rust
// source and as glam 0.29.3's scalar Vec3/Mat3 operators.
//
// Parity pins (golden vectors / known answers the reference's own tests hold):
//   fix_ties KAT (src/render/cpu.rs:738-746), sort_hi32 == stable sort
//   (src/render/radix.rs:82-105), exp_neg error < 5e-7 (src/render/simd.rs:
//   338-354), downsample KATs (src/term.rs:141-149, tests/term.rs:20-62),
//   covariance KATs (src/scene.rs:289-302), SH identities (src/sh.rs:70-91),
//   psnr(identical) = inf (src/bench.rs:248-252), semantic image tests
//   (tests/render.rs:78-203) and cpu vs cpu-naive >= 45 dB grids
//   (tests/render.rs:45-76, 215-225). Absolute bit parity with the Rust
//   binary itself is not pinned (it cannot run here).
//
// Reference files are cited as path:line inside the reference project.

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <limits>
#include <vector>

namespace {

// src/render/mod.rs:23-33
constexpr float DILATION = 0.3f;
constexpr float ALPHA_MIN = 1.0f / 255.0f;
constexpr float ALPHA_MAX = 0.99f;
constexpr float T_MIN = 1e-4f;
constexpr uint32_t MAX_DIM = 16384;
// src/render/cpu.rs:34
constexpr uint32_t TILE = 16;
constexpr int LANES = 4;
constexpr size_t MIN_GROUP = 1024;       // src/render/cpu.rs:39
constexpr size_t GROUPS_PER_THREAD = 8;  // src/render/cpu.rs:40
constexpr size_t SMALL = 192;            // src/render/radix.rs:4

// ---------------------------------------------------------------------------
// Rust scalar semantics.

// f32::min / f32::max: a NaN operand yields the other operand.
inline float rmin(float a, float b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a < b ? a : b)); }
inline float rmax(float a, float b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }
inline double rmin(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a < b ? a : b)); }
inline double rmax(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }
// f32::clamp: NaN passes through.
template <class T> inline T rclamp(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }
// `x as u32`: saturating, NaN -> 0.
template <class T> inline uint32_t as_u32(T v) {
  if (!(v > T(0))) return 0;
  if (v >= T(4294967296.0)) return UINT32_MAX;
  return (uint32_t)v;
}
template <class T> inline int32_t as_i32(T v) {
  if (std::isnan(v)) return 0;
  if (v <= T(-2147483648.0)) return INT32_MIN;
  if (v >= T(2147483647.0)) return INT32_MAX;
  return (int32_t)v;
}
inline uint32_t f2u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// glam Vec3 / Mat3 (scalar, column-major), as used by the reference.
template <class T> struct V3 { T x, y, z; };
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <class T> inline V3<T> normalize(V3<T> a) { return a * (T(1) / length(a)); }
// glam normalize_or_zero: reciprocal length, used only when finite and > 0.
template <class T> inline V3<T> normalize_or_zero(V3<T> a) {
  T rcp = T(1) / length(a);
  if (std::isfinite(rcp) && rcp > T(0)) return a * rcp;
  return {T(0), T(0), T(0)};
}
template <class T> struct M3 { V3<T> c[3]; };  // columns (x_axis, y_axis, z_axis)
// glam Mat3::mul_vec3: x_axis*v.x, + y_axis*v.y, + z_axis*v.z.
template <class T> inline V3<T> mul(const M3<T>& m, V3<T> v) {
  V3<T> r = m.c[0] * v.x;
  r = r + m.c[1] * v.y;
  r = r + m.c[2] * v.z;
  return r;
}
template <class T> inline M3<T> transpose(const M3<T>& m) {
  M3<T> r;
  r.c[0] = {m.c[0].x, m.c[1].x, m.c[2].x};
  r.c[1] = {m.c[0].y, m.c[1].y, m.c[2].y};
  r.c[2] = {m.c[0].z, m.c[1].z, m.c[2].z};
  return r;
}
template <class T> inline M3<T> mul(const M3<T>& a, const M3<T>& b) {
  return {{mul(a, b.c[0]), mul(a, b.c[1]), mul(a, b.c[2])}};
}
// glam Mat3::from_quat (quaternion x, y, z, w).
template <class T> inline M3<T> from_quat(T x, T y, T z, T w) {
  T x2 = x + x, y2 = y + y, z2 = z + z;
  T xx = x * x2, xy = x * y2, xz = x * z2;
  T yy = y * y2, yz = y * z2, zz = z * z2;
  T wx = w * x2, wy = w * y2, wz = w * z2;
  M3<T> m;
  m.c[0] = {T(1) - (yy + zz), xy + wz, xz - wy};
  m.c[1] = {xy - wz, T(1) - (xx + zz), yz + wx};
  m.c[2] = {xz + wy, yz - wx, T(1) - (xx + yy)};
  return m;
}

// src/scene.rs:170-178 — covariance R S Sᵀ Rᵀ as its upper triangle.
template <class T> void covariance(const T s[3], const T q[4], T out[6]) {
  M3<T> r = from_quat(q[0], q[1], q[2], q[3]);
  M3<T> d;
  d.c[0] = {s[0], T(0), T(0)};
  d.c[1] = {T(0), s[1], T(0)};
  d.c[2] = {T(0), T(0), s[2]};
  M3<T> m = mul(r, d);
  M3<T> c = mul(m, transpose(m));
  out[0] = c.c[0].x; out[1] = c.c[1].x; out[2] = c.c[2].x;
  out[3] = c.c[1].y; out[4] = c.c[2].y; out[5] = c.c[2].z;
}

// ---------------------------------------------------------------------------
// src/sh.rs:5-22 (3DGS constants) and src/sh.rs:39-64 (eval_rest).
constexpr float SH_C1 = 0.4886025f;
constexpr float SH_C2[5] = {1.0925485f, -1.0925485f, 0.31539157f, -1.0925485f, 0.54627424f};
constexpr float SH_C3[7] = {-0.5900436f, 2.8906114f, -0.4570458f, 0.37317633f, -0.4570458f, 1.4453057f, -0.5900436f};

template <class T> V3<T> eval_rest(uint32_t degree, const T* rest /* per*3, RGB innermost */, V3<T> dir) {
  if (degree == 0) return {T(0), T(0), T(0)};
  auto R = [&](int k) { return V3<T>{rest[3 * k], rest[3 * k + 1], rest[3 * k + 2]}; };
  T x = dir.x, y = dir.y, z = dir.z;
  V3<T> c = T(SH_C1) * (((-y) * R(0) + z * R(1)) - x * R(2));
  if (degree >= 2) {
    T xx = x * x, yy = y * y, zz = z * z;
    T xy = x * y, yz = y * z, xz = x * z;
    V3<T> s = (T(SH_C2[0]) * xy) * R(3);
    s = s + (T(SH_C2[1]) * yz) * R(4);
    s = s + (T(SH_C2[2]) * ((T(2) * zz - xx) - yy)) * R(5);
    s = s + (T(SH_C2[3]) * xz) * R(6);
    s = s + (T(SH_C2[4]) * (xx - yy)) * R(7);
    c = c + s;
    if (degree >= 3) {
      V3<T> u = ((T(SH_C3[0]) * y) * (T(3) * xx - yy)) * R(8);
      u = u + ((T(SH_C3[1]) * xy) * z) * R(9);
      u = u + ((T(SH_C3[2]) * y) * ((T(4) * zz - xx) - yy)) * R(10);
      u = u + ((T(SH_C3[3]) * z) * ((T(2) * zz - T(3) * xx) - T(3) * yy)) * R(11);
      u = u + ((T(SH_C3[4]) * x) * ((T(4) * zz - xx) - yy)) * R(12);
      u = u + ((T(SH_C3[5]) * z) * (xx - yy)) * R(13);
      u = u + ((T(SH_C3[6]) * x) * (xx - T(3) * yy)) * R(14);
      c = c + u;
    }
  }
  return c;
}

// ---------------------------------------------------------------------------
// Views and per-frame constants.

template <class T> struct View {
  V3<T> eye, right, down, fwd;
  T fov_y, near_;
};

// src/render/mod.rs:155-196 (ProjectCtx::new) with src/camera.rs:174-181.
template <class T> struct Ctx {
  M3<T> rot;
  V3<T> eye;
  T focal, cx, cy, width, height, near_, lim_x, lim_y;
};

template <class T> Ctx<T> make_ctx(const View<T>& v, uint32_t width, uint32_t height) {
  Ctx<T> c;
  // View::rotation: Mat3::from_cols(right, down, forward).transpose().
  M3<T> cols;
  cols.c[0] = v.right; cols.c[1] = v.down; cols.c[2] = v.fwd;
  c.rot = transpose(cols);
  c.eye = v.eye;
  // View::focal: height as f32 * 0.5 / (fov_y * 0.5).tan().
  c.focal = (T(height) * T(0.5)) / std::tan(v.fov_y * T(0.5));
  T w = T(width), h = T(height);
  auto lim = [&](T half) {
    T l = T(1.3f) * (half / c.focal);
    return std::isfinite(l) ? l : T(0);
  };
  c.cx = w * T(0.5);
  c.cy = h * T(0.5);
  c.width = w;
  c.height = h;
  c.near_ = v.near_;
  c.lim_x = lim(w * T(0.5));
  c.lim_y = lim(h * T(0.5));
  return c;
}

template <class T> struct Splat2D {
  T x, y, conic[3], color[3], opacity, depth, ext_x, ext_y;
};

// Per-splat inputs of `project` (one gaussian of a Scene).
template <class T> struct SplatIn {
  V3<T> p;
  T opacity;
  V3<T> color;
  const T* cov;   // 6
  const T* rest;  // per*3 or null
  uint32_t degree;
};

// src/render/mod.rs:199-272 (project); identical results to project_fast and
// project4 (src/render/cpu.rs:419-566, pinned bit for bit by cpu.rs:763-804).
// `k_pre` >= 0 substitutes the precomputed bounding radius (cpu.rs:384-388).
// `det_out` (optional) receives the 2D covariance determinant when the
// projection gets that far.
template <class T>
bool project(const SplatIn<T>& s, const Ctx<T>& ctx, Splat2D<T>* out, T k_pre = T(-1), T* det_out = nullptr) {
  const T amin = T(ALPHA_MIN);
  T opacity = s.opacity;
  if (opacity < amin) return false;
  V3<T> t = mul(ctx.rot, s.p - ctx.eye);
  if (!(t.z > ctx.near_)) return false;
  T inv_z = T(1) / t.z;
  T x = ((ctx.focal * t.x) * inv_z) + ctx.cx;
  T y = ((ctx.focal * t.y) * inv_z) + ctx.cy;
  T tx = rclamp(t.x * inv_z, -ctx.lim_x, ctx.lim_x);
  T ty = rclamp(t.y * inv_z, -ctx.lim_y, ctx.lim_y);
  T f = ctx.focal * inv_z;
  V3<T> j0{f, T(0), (-f) * tx};
  V3<T> j1{T(0), f, (-f) * ty};
  M3<T> rt = transpose(ctx.rot);
  V3<T> t0 = mul(rt, j0);
  V3<T> t1 = mul(rt, j1);
  const T* c = s.cov;
  auto sigma = [&](V3<T> v) {
    return V3<T>{(c[0] * v.x + c[1] * v.y) + c[2] * v.z, (c[1] * v.x + c[3] * v.y) + c[4] * v.z,
                 (c[2] * v.x + c[4] * v.y) + c[5] * v.z};
  };
  V3<T> s0 = sigma(t0);
  T a = dot(t0, s0) + T(DILATION);
  T b = dot(t1, s0);
  T cc = dot(t1, sigma(t1)) + T(DILATION);
  T det = a * cc - b * b;
  if (det_out) *det_out = det;
  if (!(det > T(0))) return false;
  T inv_det = T(1) / det;
  T k = k_pre >= T(0) ? k_pre : std::sqrt(T(2) * std::log(opacity / amin));
  T ext_x = k * std::sqrt(a);
  T ext_y = k * std::sqrt(cc);
  if (x + ext_x <= T(0) || x - ext_x >= ctx.width || y + ext_y <= T(0) || y - ext_y >= ctx.height) return false;
  V3<T> color = s.color;
  if (s.degree > 0) {
    V3<T> dir = normalize_or_zero(s.p - ctx.eye);
    color = color + eval_rest(s.degree, s.rest, dir);
  }
  color = {rmax(color.x, T(0)), rmax(color.y, T(0)), rmax(color.z, T(0))};
  if (!(std::isfinite(x) && std::isfinite(y) && std::isfinite(ext_x) && std::isfinite(ext_y))) return false;
  out->x = x;
  out->y = y;
  out->conic[0] = cc * inv_det;
  out->conic[1] = (-b) * inv_det;
  out->conic[2] = a * inv_det;
  out->color[0] = color.x;
  out->color[1] = color.y;
  out->color[2] = color.z;
  out->opacity = opacity;
  out->depth = t.z;
  out->ext_x = ext_x;
  out->ext_y = ext_y;
  return true;
}

// src/render/mod.rs:276-278
template <class T> inline T power(const T conic[3], T dx, T dy) {
  return T(-0.5) * ((conic[0] * dx) * dx + (conic[2] * dy) * dy) - (conic[1] * dx) * dy;
}

// src/render/mod.rs:282-285
template <class T> inline uint8_t to_u8(T v) {
  T c = rclamp(v, T(0), T(1));
  T q = c * T(255) + T(0.5);
  if (!(q > T(0))) return 0;
  if (q >= T(255)) return 255;
  return (uint8_t)(uint32_t)q;
}

// src/render/cpu.rs:94-102
struct BBox { uint16_t x0, y0, x1, y1; };
template <class T> inline BBox pixel_bbox(T x, T y, T ex, T ey, uint32_t width, uint32_t height) {
  uint32_t x0 = as_u32(rmax(std::floor(x - ex), T(0)));
  uint32_t y0 = as_u32(rmax(std::floor(y - ey), T(0)));
  uint32_t x1 = std::min(as_u32(rmax(std::ceil(x + ex), T(0))), width);
  uint32_t y1 = std::min(as_u32(rmax(std::ceil(y + ey), T(0))), height);
  return {(uint16_t)std::min(x0, x1), (uint16_t)std::min(y0, y1), (uint16_t)x1, (uint16_t)y1};
}

// ---------------------------------------------------------------------------
// Scene (flat arrays, the reference's SoA: src/scene.rs:11-28).

struct SceneF {
  size_t n = 0;
  uint32_t degree = 0;
  std::vector<float> pos, opac, col, cov, rest;  // n*3, n, n*3, n*6, n*per*3
  size_t per() const { return degree == 0 ? 0 : (size_t)((degree + 1) * (degree + 1) - 1); }
  SplatIn<float> at(size_t i) const {
    SplatIn<float> s;
    s.p = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    s.opacity = opac[i];
    s.color = {col[3 * i], col[3 * i + 1], col[3 * i + 2]};
    s.cov = &cov[6 * i];
    s.rest = degree ? &rest[i * per() * 3] : nullptr;
    s.degree = degree;
    return s;
  }
};

SceneF scene_from(size_t n, uint32_t degree, const float* pos, const float* opac, const float* col,
                  const float* cov, const float* rest) {
  SceneF s;
  s.n = n;
  s.degree = degree;
  s.pos.assign(pos, pos + 3 * n);
  s.opac.assign(opac, opac + n);
  s.col.assign(col, col + 3 * n);
  s.cov.assign(cov, cov + 6 * n);
  if (degree) s.rest.assign(rest, rest + n * s.per() * 3);
  return s;
}

// f32::total_cmp ordering.
inline int32_t total_key(float f) {
  int32_t i;
  std::memcpy(&i, &f, 4);
  return i ^ (int32_t)(((uint32_t)(i >> 31)) >> 1);
}
bool total_lt(float a, float b) { return total_key(a) < total_key(b); }

struct Bounds { V3<float> center; float radius; };

// src/scene.rs:123-166 (Scene::bounds)
Bounds scene_bounds(const SceneF& s) {
  Bounds def{{0, 0, 0}, 1.0f};
  if (s.n == 0) return def;
  size_t step = std::max<size_t>(s.n / 200000, 1);
  std::vector<V3<float>> pts;
  for (size_t i = 0; i < s.n; i += step) {
    V3<float> p{s.pos[3 * i], s.pos[3 * i + 1], s.pos[3 * i + 2]};
    if (std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(p.z)) pts.push_back(p);
  }
  if (pts.empty()) return def;
  auto median = [](std::vector<float> v) {
    size_t mid = v.size() / 2;
    std::nth_element(v.begin(), v.begin() + mid, v.end(), total_lt);
    return v[mid];
  };
  std::vector<float> xs, ys, zs;
  for (auto& p : pts) { xs.push_back(p.x); ys.push_back(p.y); zs.push_back(p.z); }
  V3<float> center{median(xs), median(ys), median(zs)};
  std::vector<float> d;
  for (auto& p : pts) d.push_back(length(p - center));
  auto pct = [&](float q) {
    size_t idx = std::min<size_t>((size_t)as_u32((float)d.size() * q), d.size() - 1);
    std::nth_element(d.begin(), d.begin() + idx, d.end(), total_lt);
    return d[idx];
  };
  float p90 = pct(0.9f);
  float p50 = pct(0.5f);
  float radius = rmin(p90, 2.0f * p50);
  return {center, radius > 1e-6f ? radius : 1.0f};
}

// ---------------------------------------------------------------------------
// src/render/simd.rs:166-307 (portable 4-lane F4, unfused mul_add) and
// src/render/simd.rs:315-331 (exp_neg).
struct F4 {
  float v[4];
};
inline F4 splat4(float a) { return {{a, a, a, a}}; }
#define F4_OP(name, expr)                                          \
  inline F4 name(F4 a, F4 b) {                                    \
    F4 r;                                                          \
    for (int i = 0; i < 4; i++) { float x = a.v[i], y = b.v[i]; r.v[i] = (expr); } \
    return r;                                                      \
  }
F4_OP(add4, x + y)
F4_OP(sub4, x - y)
F4_OP(mul4, x * y)
F4_OP(min4, rmin(x, y))
F4_OP(max4, rmax(x, y))
#undef F4_OP
// F4::mul_add(self, a, b) = self + a * b (unfused on x86).
inline F4 mul_add4(F4 s, F4 a, F4 b) { return add4(s, mul4(a, b)); }

float exp_neg1(float xin) {
  const float LOG2E = 1.44269504088896340736f;
  const float C1 = 0.6933594f;
  const float C2 = -2.1219444e-4f;
  float x = rmax(xin, -87.0f);
  float n = std::nearbyint(x * LOG2E);  // round_ties_even
  float f = (x - n * C1) - n * C2;
  float p = 1.9875691e-4f;
  p = 1.3981999e-3f + p * f;
  p = 8.333452e-3f + p * f;
  p = 4.1665796e-2f + p * f;
  p = 1.6666665e-1f + p * f;
  p = 0.5f + p * f;
  float f2 = f * f;
  float r = (f + 1.0f) + p * f2;
  uint32_t e = ((uint32_t)(as_i32(n) + 127)) << 23;
  return r * u2f(e);
}
inline F4 exp_neg4(F4 a) {
  F4 r;
  for (int i = 0; i < 4; i++) r.v[i] = exp_neg1(a.v[i]);
  return r;
}

// ---------------------------------------------------------------------------
// src/render/radix.rs:13-57 (sort_hi32): stable LSD sort on the upper 32 bits.
void sort_hi32(uint64_t* keys, uint64_t* tmp, size_t n) {
  if (n <= SMALL) {
    std::sort(keys, keys + n);
    return;
  }
  uint32_t hist[4][256];
  std::memset(hist, 0, sizeof(hist));
  for (size_t i = 0; i < n; i++) {
    uint32_t h = (uint32_t)(keys[i] >> 32);
    hist[0][h & 0xff]++;
    hist[1][(h >> 8) & 0xff]++;
    hist[2][(h >> 16) & 0xff]++;
    hist[3][h >> 24]++;
  }
  uint64_t* src = keys;
  uint64_t* dst = tmp;
  bool in_tmp = false;
  for (int d = 0; d < 4; d++) {
    int shift = 32 + 8 * d;
    uint32_t* h = hist[d];
    if ((size_t)h[(src[0] >> shift) & 0xff] == n) continue;
    uint32_t sum = 0;
    for (int c = 0; c < 256; c++) { uint32_t v = h[c]; h[c] = sum; sum += v; }
    for (size_t i = 0; i < n; i++) {
      uint64_t k = src[i];
      dst[h[(k >> shift) & 0xff]++] = k;
    }
    std::swap(src, dst);
    in_tmp = !in_tmp;
  }
  if (in_tmp) std::memcpy(dst, src, n * 8);
}

// src/render/cpu.rs:396-414 (fix_ties)
void fix_ties(uint64_t* keys, size_t n, const uint32_t* orig) {
  size_t i = 0;
  while (i + 1 < n) {
    uint64_t d = keys[i] >> 32;
    if ((keys[i + 1] >> 32) != d) { i++; continue; }
    size_t j = i + 2;
    while (j < n && (keys[j] >> 32) == d) j++;
    std::sort(keys + i, keys + j, [&](uint64_t a, uint64_t b) { return orig[(uint32_t)a] < orig[(uint32_t)b]; });
    i = j;
  }
}

// ---------------------------------------------------------------------------
// A small persistent thread pool standing in for rayon's global pool.
class Pool {
 public:
  explicit Pool(unsigned n) : n_(std::max(1u, n)) {
    for (unsigned i = 1; i < n_; i++) workers_.emplace_back([this, i] { loop(i); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
      gen_++;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  unsigned size() const { return n_; }
  // Runs fn(item) for item in [0, count), items handed out one at a time.
  void run(size_t count, const std::function<void(size_t)>& fn) {
    if (count == 0) return;
    if (n_ == 1) { for (size_t i = 0; i < count; i++) fn(i); return; }
    {
      std::lock_guard<std::mutex> g(m_);
      fn_ = &fn;
      count_ = count;
      next_.store(0);
      active_ = n_ - 1;
      gen_++;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> l(m_);
    done_cv_.wait(l, [&] { return active_ == 0; });
    fn_ = nullptr;
  }

 private:
  void work() {
    for (;;) {
      size_t i = next_.fetch_add(1);
      if (i >= count_) break;
      (*fn_)(i);
    }
  }
  void loop(unsigned) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
      }
      work();
      {
        std::lock_guard<std::mutex> g(m_);
        if (--active_ == 0) done_cv_.notify_all();
      }
    }
  }
  unsigned n_;
  std::vector<std::thread> workers_;
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(size_t)>* fn_ = nullptr;
  size_t count_ = 0;
  std::atomic<size_t> next_{0};
  unsigned active_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

struct Stats {
  uint64_t visible, overlaps;
  double project_ms, sort_ms, raster_ms, total_ms;
};

double ms_since(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// ---------------------------------------------------------------------------
// src/render/naive.rs:29-101 (CpuNaive::render), templated so that T = double
// gives the FP64 run of the same algorithm.
template <class T>
Stats render_naive(size_t n, const std::function<SplatIn<T>(size_t)>& at, const View<T>& view, uint32_t width,
                   uint32_t height, const T bg[3], uint8_t* rgb, T* linear_out) {
  auto start = std::chrono::steady_clock::now();
  Stats st{};
  if (width == 0 || height == 0) return st;
  Ctx<T> ctx = make_ctx(view, width, height);
  std::vector<Splat2D<T>> splats;
  for (size_t i = 0; i < n; i++) {
    Splat2D<T> s;
    if (project(at(i), ctx, &s)) splats.push_back(s);
  }
  st.visible = splats.size();
  auto t_proj = std::chrono::steady_clock::now();
  // Stable sort by depth (f32::total_cmp; depths are > near > 0).
  std::stable_sort(splats.begin(), splats.end(), [](const Splat2D<T>& a, const Splat2D<T>& b) { return a.depth < b.depth; });
  auto t_sort = std::chrono::steady_clock::now();
  size_t np = (size_t)width * height;
  std::vector<T> color(np * 3, T(0));
  std::vector<T> trans(np, T(1));
  const T tmin = T(T_MIN), amin = T(ALPHA_MIN), amax = T(ALPHA_MAX);
  for (const auto& s : splats) {
    BBox bb = pixel_bbox(s.x, s.y, s.ext_x, s.ext_y, width, height);
    for (uint32_t py = bb.y0; py < bb.y1; py++) {
      T dy = (T(py) + T(0.5)) - s.y;
      for (uint32_t px = bb.x0; px < bb.x1; px++) {
        size_t i = (size_t)py * width + px;
        T t = trans[i];
        if (t < tmin) continue;
        T pw = power(s.conic, (T(px) + T(0.5)) - s.x, dy);
        if (pw > T(0)) continue;
        T alpha = rmin(s.opacity * std::exp(pw), amax);
        if (alpha < amin) continue;
        T w = alpha * t;
        for (int c = 0; c < 3; c++) color[3 * i + c] = color[3 * i + c] + s.color[c] * w;
        trans[i] = t * (T(1) - alpha);
      }
    }
  }
  st.overlaps = splats.size();
  for (size_t i = 0; i < np; i++) {
    T t = trans[i];
    for (int c = 0; c < 3; c++) {
      T v = color[3 * i + c] + t * bg[c];
      if (linear_out) linear_out[3 * i + c] = v;
      rgb[3 * i + c] = to_u8(v);
    }
  }
  auto end = std::chrono::steady_clock::now();
  st.project_ms = ms_since(start, t_proj);
  st.sort_ms = ms_since(t_proj, t_sort);
  st.raster_ms = ms_since(t_sort, end);
  st.total_ms = ms_since(start, end);
  return st;
}

// ---------------------------------------------------------------------------
// src/render/cpu.rs (CpuTiled): Morton-reordered scene copy (Prep, cpu.rs:
// 321-394), grouped projection emitting (tile, key) pairs (cpu.rs:232-319),
// counting sort by tile (cpu.rs:149-199), per-tile sort_hi32 + fix_ties +
// raster_tile (cpu.rs:202-214, 604-719).

inline uint32_t spread3(uint32_t v) {  // src/render/cpu.rs:338-346
  uint32_t x = v & 0x3ff;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

struct RSplat {  // src/render/cpu.rs:42-54
  float x, y, conic[3], color[3], opacity;
  uint16_t bbox[4];
};

struct Group {  // src/render/cpu.rs:56-66
  std::vector<uint64_t> keys;
  std::vector<std::pair<uint32_t, uint32_t>> tiles;
  std::vector<uint32_t> counts;
};

struct CpuTiled {
  SceneF scene;  // reordered
  std::vector<uint32_t> orig;
  std::vector<float> k;
  std::vector<Group> groups;
  std::vector<uint64_t> keys, sort_tmp;
  std::vector<RSplat> splats;
  std::vector<uint32_t> tile_start;
  std::unique_ptr<Pool> pool;

  CpuTiled(const SceneF& src, unsigned threads) : pool(new Pool(threads)) {
    size_t n = src.n;
    Bounds b = scene_bounds(src);
    V3<float> lo = b.center - V3<float>{4.0f * b.radius, 4.0f * b.radius, 4.0f * b.radius};
    float scale = 1024.0f / (8.0f * b.radius);
    std::vector<uint64_t> order(n);
    for (size_t i = 0; i < n; i++) {
      V3<float> p{src.pos[3 * i], src.pos[3 * i + 1], src.pos[3 * i + 2]};
      V3<float> q = (p - lo) * scale;
      // Vec3::clamp(ZERO, 1023) = max(ZERO).min(1023)
      float qx = rmin(rmax(q.x, 0.0f), 1023.0f), qy = rmin(rmax(q.y, 0.0f), 1023.0f),
            qz = rmin(rmax(q.z, 0.0f), 1023.0f);
      uint32_t code = spread3(as_u32(qx)) | spread3(as_u32(qy)) << 1 | spread3(as_u32(qz)) << 2;
      order[i] = ((uint64_t)code << 32) | i;
    }
    std::sort(order.begin(), order.end());
    orig.resize(n);
    for (size_t j = 0; j < n; j++) orig[j] = (uint32_t)order[j];
    scene.n = n;
    scene.degree = src.degree;
    size_t per3 = src.per() * 3;
    scene.pos.resize(3 * n); scene.opac.resize(n); scene.col.resize(3 * n); scene.cov.resize(6 * n);
    scene.rest.resize(n * per3);
    for (size_t j = 0; j < n; j++) {
      size_t i = orig[j];
      std::memcpy(&scene.pos[3 * j], &src.pos[3 * i], 12);
      scene.opac[j] = src.opac[i];
      std::memcpy(&scene.col[3 * j], &src.col[3 * i], 12);
      std::memcpy(&scene.cov[6 * j], &src.cov[6 * i], 24);
      if (per3) std::memcpy(&scene.rest[j * per3], &src.rest[i * per3], per3 * 4);
    }
    k.resize(n);
    for (size_t j = 0; j < n; j++) {
      float o = scene.opac[j];
      k[j] = o < ALPHA_MIN ? 0.0f : std::sqrt(2.0f * std::log(o / ALPHA_MIN));
    }
  }

  Stats render(const View<float>& view, uint32_t width, uint32_t height, const float bg[3], uint8_t* frame) {
    auto start = std::chrono::steady_clock::now();
    Stats st{};
    if (width == 0 || height == 0) return st;
    size_t n = scene.n;
    Ctx<float> ctx = make_ctx(view, width, height);
    uint32_t tiles_x = (width + TILE - 1) / TILE, tiles_y = (height + TILE - 1) / TILE;
    size_t num_tiles = (size_t)tiles_x * tiles_y;
    size_t threads = pool->size();
    size_t jobs = std::max<size_t>(std::min<size_t>((n + MIN_GROUP - 1) / MIN_GROUP, threads * GROUPS_PER_THREAD), 1);
    size_t group = std::max<size_t>((n + jobs - 1) / jobs, 1);
    size_t ngroups = (n + group - 1) / group;
    groups.resize(ngroups);
    if (splats.size() != n) splats.assign(n, RSplat{});
    // 1. Project + emit overlap pairs, per index group.
    pool->run(ngroups, [&](size_t gi) {
      Group& g = groups[gi];
      g.keys.clear();
      g.tiles.clear();
      g.counts.assign(num_tiles, 0);
      size_t base = gi * group, end = std::min(n, base + group);
      for (size_t i = base; i < end; i++) {
        Splat2D<float> s;
        if (!project(scene.at(i), ctx, &s, k[i])) continue;
        BBox bb = pixel_bbox(s.x, s.y, s.ext_x, s.ext_y, width, height);
        uint32_t rec = (uint32_t)g.keys.size();
        RSplat& r = splats[i];
        r.x = s.x; r.y = s.y;
        std::memcpy(r.conic, s.conic, 12);
        std::memcpy(r.color, s.color, 12);
        r.opacity = s.opacity;
        r.bbox[0] = bb.x0; r.bbox[1] = bb.y0; r.bbox[2] = bb.x1; r.bbox[3] = bb.y1;
        g.keys.push_back(((uint64_t)f2u(s.depth) << 32) | (uint64_t)i);
        if (bb.x0 >= bb.x1 || bb.y0 >= bb.y1) continue;
        uint32_t tx0 = bb.x0 / TILE, ty0 = bb.y0 / TILE;
        uint32_t tx1 = (bb.x1 + TILE - 1) / TILE, ty1 = (bb.y1 + TILE - 1) / TILE;
        for (uint32_t ty = ty0; ty < ty1; ty++)
          for (uint32_t tx = tx0; tx < tx1; tx++) {
            uint32_t t = ty * tiles_x + tx;
            g.tiles.push_back({t, rec});
            g.counts[t]++;
          }
      }
    });
    for (auto& g : groups) st.visible += g.keys.size();
    auto t_proj = std::chrono::steady_clock::now();
    // 2. Counting sort by tile.
    tile_start.assign(num_tiles + 1, 0);
    uint64_t total = 0;
    for (size_t t = 0; t < num_tiles; t++) {
      tile_start[t] = (uint32_t)total;
      for (auto& g : groups) {
        uint32_t c = g.counts[t];
        g.counts[t] = (uint32_t)total;
        total += c;
      }
    }
    tile_start[num_tiles] = (uint32_t)total;
    st.overlaps = total;
    keys.resize(total);
    pool->run(ngroups, [&](size_t gi) {
      Group& g = groups[gi];
      for (auto& tr : g.tiles) keys[g.counts[tr.first]++] = g.keys[tr.second];
    });
    if (sort_tmp.size() < total) sort_tmp.resize(total);
    std::vector<uint32_t> order(num_tiles);
    for (size_t t = 0; t < num_tiles; t++) order[t] = (uint32_t)t;
    // Largest tiles first (scheduling only; src/render/cpu.rs:198-199).
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
      return (tile_start[a + 1] - tile_start[a]) > (tile_start[b + 1] - tile_start[b]);
    });
    auto t_sort = std::chrono::steady_clock::now();
    // 3. Per tile: sort by depth, fix ties, blend.
    pool->run(num_tiles, [&](size_t oi) {
      uint32_t t = order[oi];
      size_t b = tile_start[t], e = tile_start[t + 1];
      sort_hi32(&keys[b], &sort_tmp[b], e - b);
      fix_ties(&keys[b], e - b, orig.data());
      raster_tile(&keys[b], e - b, (t % tiles_x) * TILE, (t / tiles_x) * TILE, width, height, bg, frame);
    });
    auto end = std::chrono::steady_clock::now();
    st.project_ms = ms_since(start, t_proj);
    st.sort_ms = ms_since(t_proj, t_sort);
    st.raster_ms = ms_since(t_sort, end);
    st.total_ms = ms_since(start, end);
    return st;
  }

  // src/render/cpu.rs:604-719
  void raster_tile(const uint64_t* tkeys, size_t nkeys, uint32_t ox, uint32_t oy, uint32_t width, uint32_t height,
                   const float bg[3], uint8_t* out) const {
    constexpr int ROW_GROUPS = TILE / LANES;
    constexpr int TILE_GROUPS = TILE * TILE / LANES;
    size_t tw = std::min(TILE, width - ox), th = std::min(TILE, height - oy);
    F4 tr[TILE_GROUPS], cr[TILE_GROUPS], cg[TILE_GROUPS], cb[TILE_GROUPS];
    for (int i = 0; i < TILE_GROUPS; i++) { tr[i] = splat4(1.0f); cr[i] = cg[i] = cb[i] = splat4(0.0f); }
    uint32_t full_row = (uint32_t)((1ull << tw) - 1);
    uint32_t live[TILE] = {0};
    for (size_t y = 0; y < th; y++) live[y] = full_row;
    size_t live_rows = th;
    float fx = (float)ox, fy = (float)oy;
    const F4 lane = {{0.0f, 1.0f, 2.0f, 3.0f}};
    const F4 zero = splat4(0.0f), one = splat4(1.0f);
    const F4 amin = splat4(ALPHA_MIN), amax = splat4(ALPHA_MAX), tmin = splat4(T_MIN);
    F4 dxs[ROW_GROUPS], qx[ROW_GROUPS];
    for (size_t ki = 0; ki < nkeys; ki++) {
      const RSplat& s = splats[(uint32_t)tkeys[ki]];
      size_t bx0 = s.bbox[0], by0 = s.bbox[1], bx1 = s.bbox[2], by1 = s.bbox[3];
      size_t lx0 = bx0 > ox ? bx0 - ox : 0;
      size_t lx1 = std::min(bx1 > ox ? bx1 - ox : 0, tw);
      size_t ly0 = by0 > oy ? by0 - oy : 0;
      size_t ly1 = std::min(by1 > oy ? by1 - oy : 0, th);
      if (lx0 >= lx1) continue;
      uint32_t bbox_bits = ((uint32_t)((1ull << lx1) - 1)) & ~((1u << lx0) - 1);
      size_t g0 = lx0 / LANES, g1 = (lx1 + LANES - 1) / LANES;
      float a = s.conic[0], b = s.conic[1], c = s.conic[2];
      float cx0 = (fx + 0.5f) - s.x;
      for (size_t g = g0; g < g1; g++) {
        F4 dx = add4(lane, splat4((float)(g * LANES) + cx0));
        dxs[g] = dx;
        qx[g] = mul4(mul4(dx, dx), splat4(-0.5f * a));
      }
      F4 op = splat4(s.opacity), sr = splat4(s.color[0]), sg = splat4(s.color[1]), sb = splat4(s.color[2]);
      for (size_t ly = ly0; ly < ly1; ly++) {
        uint32_t lm = live[ly] & bbox_bits;
        if (lm == 0) continue;
        float dy = ((fy + (float)ly) + 0.5f) - s.y;
        F4 qy = splat4(((-0.5f * c) * dy) * dy);
        F4 bdy = splat4((-b) * dy);
        uint32_t sat = 0;
        for (size_t g = g0; g < g1; g++) {
          uint32_t gm = (lm >> (g * LANES)) & 0xF;
          if (gm == 0) continue;
          size_t i = ly * ROW_GROUPS + g;
          F4 pw = mul_add4(add4(qx[g], qy), bdy, dxs[g]);
          F4 alpha = min4(mul4(exp_neg4(pw), op), amax);
          F4 t = tr[i];
          F4 w, nt;
          uint32_t m = 0;
          for (int l = 0; l < 4; l++) {
            bool on = ((gm >> l) & 1) && (pw.v[l] <= zero.v[l]) && (alpha.v[l] >= amin.v[l]);
            if (!on) alpha.v[l] = 0.0f;
            m |= (uint32_t)on << l;
          }
          w = mul4(alpha, t);
          cr[i] = mul_add4(cr[i], sr, w);
          cg[i] = mul_add4(cg[i], sg, w);
          cb[i] = mul_add4(cb[i], sb, w);
          nt = mul4(t, sub4(one, alpha));
          tr[i] = nt;
          uint32_t sm = 0;
          for (int l = 0; l < 4; l++) sm |= (uint32_t)((nt.v[l] < tmin.v[l]) && ((m >> l) & 1)) << l;
          sat |= sm << (g * LANES);
        }
        if (sat != 0) {
          live[ly] &= ~sat;
          if (live[ly] == 0) live_rows--;
        }
      }
      if (live_rows == 0) break;
    }
    for (size_t ly = 0; ly < th; ly++) {
      uint8_t* row = out + ((size_t)(oy + ly) * width + ox) * 3;
      for (size_t px = 0; px < tw; px++) {
        size_t i = ly * ROW_GROUPS + px / LANES;
        int l = (int)(px % LANES);
        float t = tr[i].v[l];
        row[3 * px + 0] = to_u8(cr[i].v[l] + t * bg[0]);
        row[3 * px + 1] = to_u8(cg[i].v[l] + t * bg[1]);
        row[3 * px + 2] = to_u8(cb[i].v[l] + t * bg[2]);
      }
    }
  }
};

View<float> view_from(const float* v) {
  View<float> r;
  r.eye = {v[0], v[1], v[2]};
  r.right = {v[3], v[4], v[5]};
  r.down = {v[6], v[7], v[8]};
  r.fwd = {v[9], v[10], v[11]};
  r.fov_y = v[12];
  r.near_ = v[13];
  return r;
}

void write_stats(const Stats& s, double* out) {
  if (!out) return;
  out[0] = (double)s.visible;
  out[1] = (double)s.overlaps;
  out[2] = s.project_ms;
  out[3] = s.sort_ms;
  out[4] = s.raster_ms;
  out[5] = s.total_ms;
}

bool bad_dims(uint32_t w, uint32_t h) { return w > MAX_DIM || h > MAX_DIM; }

}  // namespace

// ===========================================================================
// C API for ctypes (tests and the CPU-baseline leg only).
//
// Scene arrays follow the reference's Scene SoA: positions n*3, opacities n,
// colors n*3, cov3d n*6, sh_rest n*per*3 (splat-major, coefficient, RGB).
// A view is 14 floats: eye[3], right[3], down[3], forward[3], fov_y, near.
// Stats are 6 doubles: visible, overlaps, project_ms, sort_ms, raster_ms,
// total_ms (src/render/mod.rs:72-83).

extern "C" {

int oracle_abi_version() { return 1; }

// src/render/mod.rs:169-196; out: rot (9, row-major = rows right/down/fwd),
// eye(3), focal, cx, cy, width, height, near, lim_x, lim_y
void oracle_project_ctx(const float* view, uint32_t w, uint32_t h, float* out) {
  Ctx<float> c = make_ctx(view_from(view), w, h);
  for (int r = 0; r < 3; r++) {
    out[3 * r + 0] = r == 0 ? c.rot.c[0].x : (r == 1 ? c.rot.c[0].y : c.rot.c[0].z);
    out[3 * r + 1] = r == 0 ? c.rot.c[1].x : (r == 1 ? c.rot.c[1].y : c.rot.c[1].z);
    out[3 * r + 2] = r == 0 ? c.rot.c[2].x : (r == 1 ? c.rot.c[2].y : c.rot.c[2].z);
  }
  out[9] = c.eye.x; out[10] = c.eye.y; out[11] = c.eye.z;
  out[12] = c.focal; out[13] = c.cx; out[14] = c.cy; out[15] = c.width; out[16] = c.height;
  out[17] = c.near_; out[18] = c.lim_x; out[19] = c.lim_y;
}

// Per-splat project(): out is n*12 floats (x, y, conic[3], color[3], opacity,
// depth, ext_x, ext_y), visible n bytes.
void oracle_project(uint64_t n, uint32_t degree, const float* pos, const float* opac, const float* col,
                    const float* cov, const float* rest, const float* view, uint32_t w, uint32_t h, float* out,
                    uint8_t* visible) {
  SceneF s = scene_from(n, degree, pos, opac, col, cov, rest);
  Ctx<float> ctx = make_ctx(view_from(view), w, h);
  for (size_t i = 0; i < n; i++) {
    Splat2D<float> p;
    bool ok = project(s.at(i), ctx, &p);
    visible[i] = ok;
    float* o = out + 12 * i;
    if (ok) {
      o[0] = p.x; o[1] = p.y; o[2] = p.conic[0]; o[3] = p.conic[1]; o[4] = p.conic[2];
      o[5] = p.color[0]; o[6] = p.color[1]; o[7] = p.color[2]; o[8] = p.opacity; o[9] = p.depth;
      o[10] = p.ext_x; o[11] = p.ext_y;
    } else {
      std::memset(o, 0, 48);
    }
  }
}

// The 2D covariance determinant project() computes per splat (+inf where the
// splat is culled before it), for locating near-singular conics.
void oracle_project_det(uint64_t n, uint32_t degree, const float* pos, const float* opac, const float* col,
                        const float* cov, const float* rest, const float* view, uint32_t w, uint32_t h,
                        float* det) {
  SceneF s = scene_from(n, degree, pos, opac, col, cov, rest);
  Ctx<float> ctx = make_ctx(view_from(view), w, h);
  for (size_t i = 0; i < n; i++) {
    Splat2D<float> p;
    det[i] = std::numeric_limits<float>::infinity();
    project(s.at(i), ctx, &p, -1.0f, &det[i]);
  }
}

// sh::eval_rest for one direction. rest: per*3.
void oracle_eval_rest(uint32_t degree, const float* rest, const float* dir, float* out) {
  V3<float> c = eval_rest<float>(degree, rest, V3<float>{dir[0], dir[1], dir[2]});
  out[0] = c.x; out[1] = c.y; out[2] = c.z;
}

void oracle_covariance(const float* scale, const float* quat_xyzw, float* out6) {
  covariance<float>(scale, quat_xyzw, out6);
}

void oracle_exp_neg(const float* x, float* out, uint64_t n) {
  for (size_t i = 0; i < n; i++) out[i] = exp_neg1(x[i]);
}

void oracle_sort_hi32(uint64_t* keys, uint64_t n) {
  std::vector<uint64_t> tmp(n);
  sort_hi32(keys, tmp.data(), n);
}

void oracle_fix_ties(uint64_t* keys, uint64_t n, const uint32_t* orig) { fix_ties(keys, n, orig); }

uint32_t oracle_spread3(uint32_t v) { return spread3(v); }

// Scene::bounds: out = center[3], radius
void oracle_bounds(uint64_t n, const float* pos, float* out) {
  SceneF s;
  s.n = n;
  s.pos.assign(pos, pos + 3 * n);
  Bounds b = scene_bounds(s);
  out[0] = b.center.x; out[1] = b.center.y; out[2] = b.center.z; out[3] = b.radius;
}

// src/term.rs:73-99 (downsample). dst must hold (w/f)*(h/f)*3 bytes.
void oracle_downsample(const uint8_t* src, uint32_t w, uint32_t h, uint32_t factor, uint8_t* dst) {
  factor = std::max(factor, 1u);
  uint32_t ow = w / factor, oh = h / factor;
  if (factor == 1) { std::memcpy(dst, src, (size_t)ow * oh * 3); return; }
  uint32_t n = factor * factor;
  for (uint32_t y = 0; y < oh; y++)
    for (uint32_t x = 0; x < ow; x++) {
      uint32_t acc[3] = {0, 0, 0};
      for (uint32_t sy = 0; sy < factor; sy++) {
        const uint8_t* row = src + ((size_t)(y * factor + sy) * w + x * factor) * 3;
        for (uint32_t sx = 0; sx < factor; sx++)
          for (int c = 0; c < 3; c++) acc[c] += row[3 * sx + c];
      }
      for (int c = 0; c < 3; c++) dst[((size_t)y * ow + x) * 3 + c] = (uint8_t)(acc[c] / n);
    }
}

// src/bench.rs:152-170
double oracle_psnr(const uint8_t* a, const uint8_t* b, uint64_t npix) {
  if (npix == 0) return 0.0;
  double se = 0.0;
  for (size_t i = 0; i < npix * 3; i++) {
    double d = (double)a[i] - (double)b[i];
    se += d * d;
  }
  double mse = se / (double)(npix * 3);
  if (mse == 0.0) return INFINITY;
  return 10.0 * std::log10(255.0 * 255.0 / mse);
}

// CpuNaive::render (FP32). rgb: w*h*3.
int oracle_render_naive(uint64_t n, uint32_t degree, const float* pos, const float* opac, const float* col,
                        const float* cov, const float* rest, const float* view, uint32_t w, uint32_t h,
                        const float* bg, uint8_t* rgb, double* stats) {
  if (bad_dims(w, h)) return 1;
  SceneF s = scene_from(n, degree, pos, opac, col, cov, rest);
  std::function<SplatIn<float>(size_t)> at = [&](size_t i) { return s.at(i); };
  Stats st = render_naive<float>(n, at, view_from(view), w, h, bg, rgb, nullptr);
  write_stats(st, stats);
  return 0;
}

// FP64 run of the naive rasterizer for scenes stored with FP16 parameters:
// inputs are the decoded values (positions fp32; scales, rotations (x,y,z,w),
// opacities, base colours and SH rest as decoded from FP16). The covariance,
// projection, SH and blending are all computed in double. linear (optional):
// w*h*3 doubles before quantisation.
int oracle_render_naive_f64(uint64_t n, uint32_t degree, const float* pos, const float* scale, const float* rot,
                            const float* opac, const float* col, const float* rest, const float* view, uint32_t w,
                            uint32_t h, const float* bg, uint8_t* rgb, double* linear, double* stats) {
  if (bad_dims(w, h)) return 1;
  size_t per3 = degree ? (size_t)((degree + 1) * (degree + 1) - 1) * 3 : 0;
  std::vector<double> cov(6 * n), rest_d(n * per3);
  for (size_t i = 0; i < n; i++) {
    double s[3] = {scale[3 * i], scale[3 * i + 1], scale[3 * i + 2]};
    double q[4] = {rot[4 * i], rot[4 * i + 1], rot[4 * i + 2], rot[4 * i + 3]};
    double len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    if (std::isfinite(len) && len > 1e-12) {
      for (int k = 0; k < 4; k++) q[k] /= len;
    } else {
      q[0] = q[1] = q[2] = 0.0; q[3] = 1.0;
    }
    covariance<double>(s, q, &cov[6 * i]);
  }
  for (size_t j = 0; j < n * per3; j++) rest_d[j] = rest[j];
  std::function<SplatIn<double>(size_t)> at = [&](size_t i) {
    SplatIn<double> si;
    si.p = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    double o = opac[i];
    si.opacity = std::isfinite(o) ? std::min(std::max(o, 0.0), 1.0) : 0.0;
    si.color = {col[3 * i], col[3 * i + 1], col[3 * i + 2]};
    si.cov = &cov[6 * i];
    si.rest = per3 ? &rest_d[i * per3] : nullptr;
    si.degree = degree;
    return si;
  };
  View<float> vf = view_from(view);
  View<double> vd;
  vd.eye = {vf.eye.x, vf.eye.y, vf.eye.z};
  vd.right = {vf.right.x, vf.right.y, vf.right.z};
  vd.down = {vf.down.x, vf.down.y, vf.down.z};
  vd.fwd = {vf.fwd.x, vf.fwd.y, vf.fwd.z};
  vd.fov_y = vf.fov_y;
  vd.near_ = vf.near_;
  double bgd[3] = {bg[0], bg[1], bg[2]};
  Stats st = render_naive<double>(n, at, vd, w, h, bgd, rgb, linear);
  write_stats(st, stats);
  return 0;
}

// CpuTiled: create once per scene (Prep), render many views.
void* oracle_cpu_create(uint64_t n, uint32_t degree, const float* pos, const float* opac, const float* col,
                        const float* cov, const float* rest, uint32_t threads) {
  if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
  SceneF s = scene_from(n, degree, pos, opac, col, cov, rest);
  return new CpuTiled(s, threads);
}

int oracle_cpu_render(void* handle, const float* view, uint32_t w, uint32_t h, const float* bg, uint8_t* rgb,
                      double* stats) {
  if (bad_dims(w, h)) return 1;
  auto* c = static_cast<CpuTiled*>(handle);
  Stats st = c->render(view_from(view), w, h, bg, rgb);
  write_stats(st, stats);
  return 0;
}

uint32_t oracle_cpu_threads(void* handle) { return static_cast<CpuTiled*>(handle)->pool->size(); }

void oracle_cpu_destroy(void* handle) { delete static_cast<CpuTiled*>(handle); }

// The CPU recomputation behind the bit-exact key/range gate: from projected
// x, y, ext_x, ext_y and depth (any source; the test feeds the device's own
// values) and visibility flags, emit one (tile << 32 | depth bits, splat)
// pair per tile of each visible splat's pixel_bbox, row-major, in splat-index
// order (src/render/cpu.rs:251-277), then sort stably by key. ranges holds
// [begin, end) per tile. Returns the pair count, or -1 if it exceeds cap.
// tile_w x tile_h tiles (the reference's are 16 x 16).
int64_t oracle_bin_sort(uint64_t n, const float* x, const float* y, const float* ext_x, const float* ext_y,
                        const float* depth, const uint8_t* visible, uint32_t w, uint32_t h, uint32_t tile_w,
                        uint32_t tile_h, uint64_t* keys, uint32_t* values, uint64_t cap, uint32_t* ranges) {
  uint32_t tiles_x = (w + tile_w - 1) / tile_w, tiles_y = (h + tile_h - 1) / tile_h;
  std::vector<std::pair<uint64_t, uint32_t>> pairs;
  for (size_t i = 0; i < n; i++) {
    if (!visible[i]) continue;
    BBox bb = pixel_bbox(x[i], y[i], ext_x[i], ext_y[i], w, h);
    if (bb.x0 >= bb.x1 || bb.y0 >= bb.y1) continue;
    uint32_t tx0 = bb.x0 / tile_w, ty0 = bb.y0 / tile_h;
    uint32_t tx1 = (bb.x1 + tile_w - 1) / tile_w, ty1 = (bb.y1 + tile_h - 1) / tile_h;
    for (uint32_t ty = ty0; ty < ty1; ty++)
      for (uint32_t tx = tx0; tx < tx1; tx++)
        pairs.push_back({((uint64_t)(ty * tiles_x + tx) << 32) | f2u(depth[i]), (uint32_t)i});
  }
  std::stable_sort(pairs.begin(), pairs.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  if (pairs.size() > cap) return -1;
  size_t num_tiles = (size_t)tiles_x * tiles_y;
  for (size_t t = 0; t < 2 * num_tiles; t++) ranges[t] = 0;
  for (size_t p = 0; p < pairs.size(); p++) {
    keys[p] = pairs[p].first;
    values[p] = pairs[p].second;
    uint32_t t = (uint32_t)(pairs[p].first >> 32);
    if (p == 0 || (uint32_t)(pairs[p - 1].first >> 32) != t) ranges[2 * t] = (uint32_t)p;
    if (p + 1 == pairs.size() || (uint32_t)(pairs[p + 1].first >> 32) != t) ranges[2 * t + 1] = (uint32_t)(p + 1);
  }
  return (int64_t)pairs.size();
}

}  // extern "C"
