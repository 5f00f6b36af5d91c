// Kernel (a): fused EWA projection, culling and SH colour, one thread per
// splat. Follows `project` (src/render/mod.rs:199-272, equal bit for bit to
// project_fast/project4 of src/render/cpu.rs:419-566) and `sh::eval_rest`
// (src/sh.rs:39-64) operation by operation. This translation unit is built
// with --fmad=false and IEEE division/sqrt, so every result is the correctly
// rounded f32 of the same expression tree the reference evaluates on x86
// (no fused multiply-adds): the projected splats equal the oracle's bit for
// bit. The kernel also emits each visible splat's tile rectangle (pixel_bbox,
// src/render/cpu.rs:94-102 and the tile loop of cpu.rs:262-276), its pair
// count and depth bits for the binning, and counts the visible splats.
#include <cuda_fp16.h>

#include <algorithm>
#include <cstddef>

#include "common.cuh"
#include "geom.cuh"
#include "mlp.cuh"
#include "sh.cuh"

namespace splat {
namespace {

// `x as u32` of a float: saturating, NaN -> 0.
__device__ __forceinline__ uint32_t sat_u32(float v) {
  if (!(v > 0.0f)) return 0u;
  if (v >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)v;
}

// f32::clamp (NaN passes through).
__device__ __forceinline__ float rclamp(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ float h2f(uint32_t bits16) { return __half2float(__ushort_as_half((unsigned short)bits16)); }

template <class T>
__device__ __forceinline__ void conic_terms(const T c[6], T t0x, T t0y, T t0z, T t1x, T t1y, T t1z, T& a, T& bb,
                                            T& cc) {
  const T s0x = (c[0] * t0x + c[1] * t0y) + c[2] * t0z;
  const T s0y = (c[1] * t0x + c[3] * t0y) + c[4] * t0z;
  const T s0z = (c[2] * t0x + c[4] * t0y) + c[5] * t0z;
  const T s1x = (c[0] * t1x + c[1] * t1y) + c[2] * t1z;
  const T s1y = (c[1] * t1x + c[3] * t1y) + c[4] * t1z;
  const T s1z = (c[2] * t1x + c[4] * t1y) + c[5] * t1z;
  a = ((t0x * s0x + t0y * s0y) + t0z * s0z) + T(kDilation);
  bb = (t1x * s0x + t1y * s0y) + t1z * s0z;
  cc = ((t1x * s1x + t1y * s1y) + t1z * s1z) + T(kDilation);
}

__device__ __forceinline__ void l2_prefetch(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// F16: the scene is stored in FP16 (positions FP32); the 3D covariance is
// formed here in FP32, and a 2D covariance whose FP32 determinant falls below
// kFp64DetBelow is recomputed in FP64.
// Projects splat i < s.n of the view: writes its record (when visible), its
// tile rectangle and the optional debug values; reports visibility and
// whether its conic took the FP64 path.
// LEARNED: the colour comes from the learned-colour MLP afterwards; the
// record's colour is left 0 and `dir` receives normalize_or_zero(p - eye),
// the direction the SH colour would be evaluated at.
// Where the FP32 scene values of splat i are read: global memory (through
// the read-only path), or a CTA's copy in shared memory (k_project_tma).
struct GlobalScene {
  const SceneDev& s;
  __device__ __forceinline__ float4 pos(uint64_t i) const { return __ldg(&s.pos_op[i]); }
  __device__ __forceinline__ float4 cov_a(uint64_t i) const { return __ldg(&s.cov_a[i]); }
  __device__ __forceinline__ float4 cov_b(uint64_t i) const { return __ldg(&s.cov_b[i]); }
  __device__ __forceinline__ float color(int ch, uint64_t i) const { return __ldg(s.color + (uint64_t)ch * s.n + i); }
  __device__ __forceinline__ float sh(int plane, uint64_t i) const {
    return __ldg(s.sh + (uint64_t)plane * s.n + i);
  }
  static constexpr bool kGlobal = true;
};

template <class Src>
__device__ __forceinline__ Src scene_source(const SceneDev& s, const Src* given) {
  if constexpr (Src::kGlobal)
    return Src{s};
  else
    return *given;
}

template <int DEG, bool F16, bool LEARNED = false, class Src = GlobalScene>
__device__ __forceinline__ void project_splat(const FrameParams& fp, const SceneDev& s, uint64_t i,
                                              Record* __restrict__ rec, BinInfo* __restrict__ bin,
                                              BinSkip* __restrict__ skip, float* __restrict__ dbg_proj,
                                              float* __restrict__ dbg_color,
                                              bool& vis, bool& used_fp64, float* dir = nullptr,
                                              const Src* given = nullptr) {
  const Src src = scene_source<Src>(s, given);
  if constexpr (!LEARNED && DEG > 0 && Src::kGlobal) {
    // The warp's 32 entries of every SH plane are brought into L2 now; the
    // loads that read them come after the geometry and the culling tests.
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t base = i - lane, last = min(base + 31, s.n - 1);
    constexpr uint32_t kPlanes = F16 ? (DEG + 1) * (DEG + 1) * 3 : ((DEG + 1) * (DEG + 1) - 1) * 3;
    for (uint32_t p = lane; p < kPlanes; p += 32) {
      if (F16) {
        l2_prefetch(s.sh16 + (uint64_t)p * s.n + base);
        l2_prefetch(s.sh16 + (uint64_t)p * s.n + last);
      } else {
        l2_prefetch(s.sh + (uint64_t)p * s.n + base);
        l2_prefetch(s.sh + (uint64_t)p * s.n + last);
      }
    }
  }
  {
    float px, py, pz, opacity, k;
    uint4 g16 = make_uint4(0, 0, 0, 0);
    if (F16) {
      const float4 pk = __ldg(&s.pos_k[i]);
      px = pk.x;
      py = pk.y;
      pz = pk.z;
      k = pk.w;
      g16 = __ldg(&s.geom16[i]);
      opacity = fminf(fmaxf(h2f(g16.w >> 16), 0.0f), 1.0f);  // Scene::finalize's clamp; NaN -> 0
    } else {
      const float4 po = src.pos(i);
      px = po.x;
      py = po.y;
      pz = po.z;
      opacity = po.w;
      k = 0.0f;
    }
    BinInfo b{kCulled, 0u, 0u, 0u};
    BinSkip bk;
    bool wide = false;  // bk is stored
    float out_x = 0.f, out_y = 0.f, out_ex = 0.f, out_ey = 0.f, out_depth = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
    float col[3] = {0.f, 0.f, 0.f};
    do {
      if (opacity < kAlphaMin) break;
      // t = rot * (p - eye), glam Mat3::mul_vec3 order.
      const float dx = px - fp.eye[0], dy = py - fp.eye[1], dz = pz - fp.eye[2];
      const float tx_ = (fp.rot[0] * dx + fp.rot[1] * dy) + fp.rot[2] * dz;
      const float ty_ = (fp.rot[3] * dx + fp.rot[4] * dy) + fp.rot[5] * dz;
      const float tz = (fp.rot[6] * dx + fp.rot[7] * dy) + fp.rot[8] * dz;
      if (!(tz > fp.near_plane)) break;
      const float inv_z = 1.0f / tz;
      const float x = ((fp.focal * tx_) * inv_z) + fp.cx;
      const float y = ((fp.focal * ty_) * inv_z) + fp.cy;
      // Jacobian at the clamped mean; rows of T = J R are rot^T * j.
      const float jx = rclamp(tx_ * inv_z, -fp.lim_x, fp.lim_x);
      const float jy = rclamp(ty_ * inv_z, -fp.lim_y, fp.lim_y);
      const float f = fp.focal * inv_z;
      const float j0z = (-f) * jx, j1z = (-f) * jy;
      const float t0x = (fp.rot[0] * f + fp.rot[3] * 0.0f) + fp.rot[6] * j0z;
      const float t0y = (fp.rot[1] * f + fp.rot[4] * 0.0f) + fp.rot[7] * j0z;
      const float t0z = (fp.rot[2] * f + fp.rot[5] * 0.0f) + fp.rot[8] * j0z;
      const float t1x = (fp.rot[0] * 0.0f + fp.rot[3] * f) + fp.rot[6] * j1z;
      const float t1y = (fp.rot[1] * 0.0f + fp.rot[4] * f) + fp.rot[7] * j1z;
      const float t1z = (fp.rot[2] * 0.0f + fp.rot[5] * f) + fp.rot[8] * j1z;
      float cov[6];
      float sc[3], q[4];
      if (F16) {
        sc[0] = h2f(g16.x & 0xFFFFu);
        sc[1] = h2f(g16.x >> 16);
        sc[2] = h2f(g16.y & 0xFFFFu);
        q[0] = h2f(g16.y >> 16);
        q[1] = h2f(g16.z & 0xFFFFu);
        q[2] = h2f(g16.z >> 16);
        q[3] = h2f(g16.w & 0xFFFFu);
        covariance_from<float>(sc, q[0], q[1], q[2], q[3], cov);
      } else {
        const float4 ca = src.cov_a(i);
        const float4 cb = src.cov_b(i);
        cov[0] = ca.x;
        cov[1] = ca.y;
        cov[2] = ca.z;
        cov[3] = ca.w;
        cov[4] = cb.x;
        cov[5] = cb.y;
        k = cb.z;  // sqrt(2 ln(opacity / ALPHA_MIN)), precomputed at upload
      }
      float a, bb, cc;
      conic_terms<float>(cov, t0x, t0y, t0z, t1x, t1y, t1z, a, bb, cc);
      float det = a * cc - bb * bb;
      float inv_det = 0.0f;
      bool conic_done = false;
      if (F16 && !(det >= kFp64DetBelow)) {
        // Near-singular: the 2D covariance and its inverse in FP64.
        double scd[3] = {sc[0], sc[1], sc[2]}, cd[6];
        covariance_from<double>(scd, (double)q[0], (double)q[1], (double)q[2], (double)q[3], cd);
        double ad, bd, ccd;
        conic_terms<double>(cd, t0x, t0y, t0z, t1x, t1y, t1z, ad, bd, ccd);
        const double detd = ad * ccd - bd * bd;
        if (!(detd > 0.0)) break;
        const double inv = 1.0 / detd;
        c0 = (float)(ccd * inv);
        c1 = (float)(-bd * inv);
        c2 = (float)(ad * inv);
        a = (float)ad;
        cc = (float)ccd;
        conic_done = true;
        used_fp64 = true;
      } else {
        if (!(det > 0.0f)) break;
        inv_det = 1.0f / det;
      }
      const float ext_x = k * sqrtf(a);
      const float ext_y = k * sqrtf(cc);
      if (x + ext_x <= 0.0f || x - ext_x >= fp.width || y + ext_y <= 0.0f || y - ext_y >= fp.height) break;
      if constexpr (LEARNED) {
        const float len = sqrtf((dx * dx + dy * dy) + dz * dz);
        const float rcp = 1.0f / len;
        if (isfinite(rcp) && rcp > 0.0f) {
          dir[0] = dx * rcp;
          dir[1] = dy * rcp;
          dir[2] = dz * rcp;
        }
      } else {
        if (F16) {
          col[0] = h2f(__ldg(s.sh16 + i));
          col[1] = h2f(__ldg(s.sh16 + s.n + i));
          col[2] = h2f(__ldg(s.sh16 + 2 * s.n + i));
        } else {
          col[0] = src.color(0, i);
          col[1] = src.color(1, i);
          col[2] = src.color(2, i);
        }
        if constexpr (DEG > 0) {
          // normalize_or_zero(p - eye)
          const float len = sqrtf((dx * dx + dy * dy) + dz * dz);
          const float rcp = 1.0f / len;
          float nx = 0.f, ny = 0.f, nz = 0.f;
          if (isfinite(rcp) && rcp > 0.0f) {
            nx = dx * rcp;
            ny = dy * rcp;
            nz = dz * rcp;
          }
          if (F16)
            sh::eval_sh<DEG>([&](int coef, int ch) { return h2f(__ldg(s.sh16 + (uint64_t)((coef + 1) * 3 + ch) * s.n + i)); },
                         nx, ny, nz, col);
          else
            sh::eval_sh<DEG>([&](int coef, int ch) { return src.sh(coef * 3 + ch, i); }, nx, ny, nz, col);
        }
        col[0] = fmaxf(col[0], 0.0f);
        col[1] = fmaxf(col[1], 0.0f);
        col[2] = fmaxf(col[2], 0.0f);
      }
      if (!(isfinite(x) && isfinite(y) && isfinite(ext_x) && isfinite(ext_y))) break;
      if (!conic_done) {
        c0 = cc * inv_det;
        c1 = (-bb) * inv_det;
        c2 = a * inv_det;
      }
      // pixel_bbox (src/render/cpu.rs:96-102)
      const uint32_t x0 = sat_u32(fmaxf(floorf(x - ext_x), 0.0f));
      const uint32_t y0 = sat_u32(fmaxf(floorf(y - ext_y), 0.0f));
      const uint32_t x1 = min(sat_u32(fmaxf(ceilf(x + ext_x), 0.0f)), fp.w);
      const uint32_t y1 = min(sat_u32(fmaxf(ceilf(y + ext_y), 0.0f)), fp.h);
      const uint32_t bx0 = min(x0, x1), by0 = min(y0, y1);
      Record r;
      r.r0 = make_float4(x, y, -0.5f * c0, -c1);
      r.r1 = make_float4(-0.5f * c2, opacity, col[0], col[1]);
      r.r2 = make_float4(col[2], __uint_as_float(bx0 | (x1 << 16)), __uint_as_float(by0 | (y1 << 16)), tz);
      rec[i] = r;
      b.depth_bits = __float_as_uint(tz);
      wide = window_rect(fp, bx0, x1, by0, y1, r, b, bk);
      vis = true;
      out_x = x;
      out_y = y;
      out_ex = ext_x;
      out_ey = ext_y;
      out_depth = tz;
    } while (false);
    bin[i] = b;
    if (wide) skip[i] = bk;
    if (dbg_proj) {
      float* d = dbg_proj + 8 * i;
      d[0] = out_x; d[1] = out_y; d[2] = out_ex; d[3] = out_ey; d[4] = out_depth; d[5] = c0; d[6] = c1; d[7] = c2;
    }
    if (!LEARNED && dbg_color) {
      dbg_color[3 * i] = vis ? col[0] : 0.f;
      dbg_color[3 * i + 1] = vis ? col[1] : 0.f;
      dbg_color[3 * i + 2] = vis ? col[2] : 0.f;
    }
  }
}

__device__ __forceinline__ void count_visible(bool vis, bool used_fp64, const FrameCounters& fc, uint32_t view) {
  const int nvis = __syncthreads_count(vis);
  const int n64 = __syncthreads_count(used_fp64);
  if (threadIdx.x == 0) {
    if (nvis) {
      atomicAdd(&fc.st->visible, (unsigned long long)nvis);
      atomicAdd(&fc.view_visible[view], (unsigned long long)nvis);
    }
    if (n64) atomicAdd(&fc.st->fp64_conics, (unsigned)n64);
  }
}

// One view, passed by value; CTA 0 also stores it as the view table's only
// entry for the launches that follow.
template <int DEG, bool F16>
__global__ void __launch_bounds__(256) k_project(ViewTask t, ViewTask* __restrict__ table,
                                                 float* __restrict__ dbg_proj, float* __restrict__ dbg_color,
                                                 FrameCounters fc) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *table = t;
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool vis = false, used_fp64 = false;
  if (i < t.s.n) project_splat<DEG, F16>(t.fp, t.s, i, t.rec, t.bin, t.skip, dbg_proj, dbg_color, vis, used_fp64);
  count_visible(vis, used_fp64, fc, 0);
}

// FP32 scenes: the same projection with each CTA's slice of every scene
// array (positions, covariance, colour and SH planes: 232 bytes per splat at
// degree 3) brought into shared memory by bulk asynchronous copies (TMA,
// cp.async.bulk) that complete on one mbarrier, so that every byte the CTA
// reads is in flight at once and the threads wait once instead of on each
// load. A plane's slice need not start on the 16 bytes a bulk copy needs: the
// copy starts at the 16-byte boundary below it (the plane buffers carry 16
// bytes of slack at their end for the rounded-up last copy) and the slice is
// read at its offset. The arithmetic is project_splat's, unchanged.
constexpr uint32_t kTmaSplats = kProjectSplatsPerCta;  // 128: 32 KB of slices per CTA (SH3), 7 CTAs per SM
constexpr uint32_t kTmaPlaneFloats = kTmaSplats + 8;  // the slice, its offset and the rounding

template <int DEG>
struct TmaLayout {
  static constexpr uint32_t kShPlanes = ((DEG + 1) * (DEG + 1) - 1) * 3;
  static constexpr uint32_t kPlanes = 3 + kShPlanes;  // colour, then SH
  static constexpr size_t kBytes = 3 * kTmaSplats * sizeof(float4) + kPlanes * kTmaPlaneFloats * sizeof(float) + 16;
};

struct SmemScene {
  const float4* p_pos;
  const float4* p_ca;
  const float4* p_cb;
  const float* planes;  // kTmaPlaneFloats floats per plane
  const uint32_t* off;  // per plane: the slice's offset in its copy
  uint64_t base;
  __device__ __forceinline__ float4 pos(uint64_t i) const { return p_pos[i - base]; }
  __device__ __forceinline__ float4 cov_a(uint64_t i) const { return p_ca[i - base]; }
  __device__ __forceinline__ float4 cov_b(uint64_t i) const { return p_cb[i - base]; }
  __device__ __forceinline__ float color(int ch, uint64_t i) const {
    return planes[ch * kTmaPlaneFloats + off[ch] + (i - base)];
  }
  __device__ __forceinline__ float sh(int plane, uint64_t i) const {
    return planes[(3 + plane) * kTmaPlaneFloats + off[3 + plane] + (i - base)];
  }
  static constexpr bool kGlobal = false;
};

__device__ __forceinline__ void bulk_copy(void* smem_dst, const void* gmem_src, uint32_t bytes, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          umma::smem_u32(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(mbar)
      : "memory");
}

// One CTA's slice of kTmaSplats splats from `base` of the FP32 view t,
// staged through shared memory (smem_raw: TmaLayout<DEG>::kBytes; s_off:
// TmaLayout<DEG>::kPlanes words; s_mbar: an mbarrier used once) and
// projected: the body of k_project_tma and, per CTA, of k_project_batch.
template <int DEG>
__device__ __forceinline__ void project_slice_tma(const ViewTask& t, uint64_t base, uint8_t* smem_raw, uint32_t* s_off,
                                                  uint64_t* s_mbar, float* dbg_proj, float* dbg_color,
                                                  const FrameCounters& fc, bool& vis, bool& used_fp64) {
  using L = TmaLayout<DEG>;
  float4* s_pos = reinterpret_cast<float4*>(smem_raw);
  float4* s_ca = s_pos + kTmaSplats;
  float4* s_cb = s_ca + kTmaSplats;
  float* s_planes = reinterpret_cast<float*>(s_cb + kTmaSplats);
  const uint32_t tid = threadIdx.x;
  const uint64_t n = t.s.n;
  const uint32_t cnt = (uint32_t)min((uint64_t)kTmaSplats, n - base);
  const uint32_t mbar = umma::smem_u32(s_mbar);
  // Copy sizes: whole float4 records; plane slices rounded out to 16 bytes.
  auto plane_src = [&](uint32_t p) -> const float* {
    return p < 3 ? t.s.color + (uint64_t)p * n : t.s.sh + (uint64_t)(p - 3) * n;
  };
  if (tid < L::kPlanes) {
    const uint64_t first = (uint64_t)(plane_src(tid) - (tid < 3 ? t.s.color : t.s.sh)) + base;
    s_off[tid] = (uint32_t)(first & 3u);
  }
  if (tid == 0) {
    umma::mbar_init(mbar, 1);
    uint32_t bytes = 3 * cnt * (uint32_t)sizeof(float4);
    for (uint32_t p = 0; p < L::kPlanes; p++) {
      const uintptr_t a = reinterpret_cast<uintptr_t>(plane_src(p) + base);
      const uintptr_t lo = a & ~(uintptr_t)15, hi = (a + cnt * sizeof(float) + 15) & ~(uintptr_t)15;
      bytes += (uint32_t)(hi - lo);
    }
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
  }
  __syncthreads();
  // The copies, spread over the first warps' lanes.
  if (tid < 3) {
    const float4* src = tid == 0 ? t.s.pos_op : tid == 1 ? t.s.cov_a : t.s.cov_b;
    bulk_copy(s_pos + tid * kTmaSplats, src + base, cnt * (uint32_t)sizeof(float4), mbar);
  } else if (tid >= 32 && tid < 32 + L::kPlanes) {
    const uint32_t p = tid - 32;
    const uintptr_t a = reinterpret_cast<uintptr_t>(plane_src(p) + base);
    const uintptr_t lo = a & ~(uintptr_t)15, hi = (a + cnt * sizeof(float) + 15) & ~(uintptr_t)15;
    bulk_copy(s_planes + p * kTmaPlaneFloats, reinterpret_cast<const void*>(lo), (uint32_t)(hi - lo), mbar);
  }
  if (!umma::mbar_wait(mbar, 0)) {
    // Copies that did not land in time: the frame reports an error, and the
    // CTA leaves only once they have (bounded) or given up on them.
    if (tid == 0) atomicExch(&fc.st->error, 2u);
    umma::mbar_wait(mbar, 0, 100000000ull);
  } else if (tid < cnt) {
    const SmemScene src{s_pos, s_ca, s_cb, s_planes, s_off, base};
    project_splat<DEG, false, false, SmemScene>(t.fp, t.s, base + tid, t.rec, t.bin, t.skip, dbg_proj, dbg_color, vis,
                                                used_fp64, nullptr, &src);
  }
}

template <int DEG>
__global__ void __launch_bounds__(kTmaSplats) k_project_tma(ViewTask t, ViewTask* __restrict__ table,
                                                            float* __restrict__ dbg_proj, float* __restrict__ dbg_color,
                                                            FrameCounters fc) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  __shared__ uint32_t s_off[TmaLayout<DEG>::kPlanes];
  __shared__ __align__(8) uint64_t s_mbar;
  if (blockIdx.x == 0 && threadIdx.x == 0) *table = t;
  bool vis = false, used_fp64 = false;
  project_slice_tma<DEG>(t, (uint64_t)blockIdx.x * kTmaSplats, smem_raw, s_off, &s_mbar, dbg_proj, dbg_color, fc, vis,
                         used_fp64);
  count_visible(vis, used_fp64, fc, 0);
}

// Every view of the table: CTA c projects kTmaSplats splats of the view
// whose proj_cta0 is the largest one <= c (views of different scenes, SH
// degrees and storage precisions in one launch); FP32 views through the
// bulk-copy staging of k_project_tma (shared memory sized for degree 3).
__global__ void __launch_bounds__(kTmaSplats) k_project_batch(const ViewTask* __restrict__ table, uint32_t n_views,
                                                              FrameCounters fc) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  __shared__ ViewTask s_t;
  __shared__ uint32_t s_off[TmaLayout<3>::kPlanes];
  __shared__ __align__(8) uint64_t s_mbar;
  const uint32_t v = find_view(table, n_views, blockIdx.x, offsetof(ViewTask, proj_cta0));
  static_assert(sizeof(ViewTask) % 16 == 0 && sizeof(ViewTask) / 16 <= kTmaSplats, "ViewTask copies as uint4");
  if (threadIdx.x < sizeof(ViewTask) / 16)
    reinterpret_cast<uint4*>(&s_t)[threadIdx.x] = __ldg(reinterpret_cast<const uint4*>(table + v) + threadIdx.x);
  __syncthreads();
  const uint64_t base = (uint64_t)(blockIdx.x - s_t.proj_cta0) * kTmaSplats, i = base + threadIdx.x;
  bool vis = false, used_fp64 = false;
  if (!s_t.s.fp16) {  // base < n: the view has a CTA per kTmaSplats of its splats
    switch (s_t.s.sh_degree) {
      case 0: project_slice_tma<0>(s_t, base, smem_raw, s_off, &s_mbar, nullptr, nullptr, fc, vis, used_fp64); break;
      case 1: project_slice_tma<1>(s_t, base, smem_raw, s_off, &s_mbar, nullptr, nullptr, fc, vis, used_fp64); break;
      case 2: project_slice_tma<2>(s_t, base, smem_raw, s_off, &s_mbar, nullptr, nullptr, fc, vis, used_fp64); break;
      default: project_slice_tma<3>(s_t, base, smem_raw, s_off, &s_mbar, nullptr, nullptr, fc, vis, used_fp64); break;
    }
  } else if (i < s_t.s.n) {
    switch (s_t.s.sh_degree) {
      case 0: project_splat<0, true>(s_t.fp, s_t.s, i, s_t.rec, s_t.bin, s_t.skip, nullptr, nullptr, vis, used_fp64); break;
      case 1: project_splat<1, true>(s_t.fp, s_t.s, i, s_t.rec, s_t.bin, s_t.skip, nullptr, nullptr, vis, used_fp64); break;
      case 2: project_splat<2, true>(s_t.fp, s_t.s, i, s_t.rec, s_t.bin, s_t.skip, nullptr, nullptr, vis, used_fp64); break;
      default: project_splat<3, true>(s_t.fp, s_t.s, i, s_t.rec, s_t.bin, s_t.skip, nullptr, nullptr, vis, used_fp64); break;
    }
  }
  count_visible(vis, used_fp64, fc, v);
}

// Learned colour (FP16 storage): the projection of k_project, then the
// colour MLP of each 128-splat tile (mlp.cuh), fused: persistent CTAs of 128
// threads, thread t = splat t of the tile = TMEM lane t. The MLP's input row
// is the splat's 16 latents and its view direction; the three layers are
// tcgen05.mma groups with their epilogues between. The record is written by
// the projection and its colour filled in after.
constexpr uint32_t kLearnedThreads = 128;
constexpr uint32_t kLearnedTmemCols = 64;  // z1, then z2, then z3 (16)

struct LearnedSmem {
  mlp::ForwardTiles t;
  ViewTask vt;  // the current tile's view
  uint64_t mbar;
  uint64_t lost;  // never arrived on: the injected lost completion (SceneDev::lost_wait_us)
  uint32_t tmem;
};
// At most 7 CTAs fit an SM by shared memory (228 KB, 1 KB reserved per CTA),
// so the CTAs of an SM never ask for more than 7 x 64 of its 512 TMEM columns.
constexpr size_t kLearnedSmem = sizeof(LearnedSmem);
static_assert((228 * 1024) / (kLearnedSmem + 1024) * kLearnedTmemCols <= 512, "TMEM oversubscribed");

// BATCH = false: one view, `t0`; CTA 0 also stores it as the view table's
// only entry. BATCH = true: the learned views of a batch, `table` holding
// n_views of them with proj_cta0 = the view's first tile in this launch's
// tile space (total_tiles tiles) and pad[0] = its index in the batch.
template <bool BATCH>
__global__ void __launch_bounds__(kLearnedThreads, 7)
    k_project_learned(ViewTask t0, ViewTask* __restrict__ table, uint32_t n_views, uint64_t total_tiles,
                      float* __restrict__ dbg_proj, float* __restrict__ dbg_color, FrameCounters fc) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  LearnedSmem& S = *reinterpret_cast<LearnedSmem*>(smem_raw);
  const uint32_t tid = threadIdx.x;
  if (!BATCH && blockIdx.x == 0 && tid == 0) *table = t0;
  if (tid == 0) {
    umma::mbar_init(umma::smem_u32(&S.mbar), 1);
    umma::mbar_init(umma::smem_u32(&S.lost), 1);
  }
  if (tid < 32) umma::tmem_alloc(&S.tmem, kLearnedTmemCols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = S.tmem, mbar = umma::smem_u32(&S.mbar);
  const uint32_t act = umma::smem_u32(S.t.act);
  uint32_t phase = 0;
  bool timed_out = false, aborted = false, inflight = false;
  uint64_t lost_ns = BATCH ? 0ull : 1000ull * t0.s.lost_wait_us;
  // Waits for the MMAs committed to `mbar`; after a wait that gave up, the
  // phase stays the one still in flight, which the exit path waits for.
  auto wait_mma = [&]() {
    if (umma::mbar_wait(mbar, phase)) {
      phase ^= 1u;
      inflight = false;
    } else {
      timed_out = true;
    }
    if (lost_ns) {
      if (!umma::mbar_wait(umma::smem_u32(&S.lost), 0, lost_ns)) timed_out = true;
      lost_ns = 0;
    }
    umma::fence_after_sync();
  };
  auto sync_or_abort = [&]() -> bool {
    umma::fence_async_smem();
    umma::fence_before_sync();
    return __syncthreads_or(timed_out) != 0;
  };
  const uint64_t tiles = BATCH ? total_tiles : (t0.s.n + mlp::kRows - 1) / mlp::kRows;
  uint32_t cur = 0xFFFFFFFFu;              // view staged in S.vt
  const uint16_t* weights = nullptr;       // parameters staged in S.t
  for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const uint32_t v = BATCH ? find_view(table, n_views, (uint32_t)tile, offsetof(ViewTask, proj_cta0)) : 0u;
    if (v != cur) {  // uniform over the CTA
      static_assert(sizeof(ViewTask) % 16 == 0, "ViewTask copies as uint4");
      __syncthreads();
      if (tid < sizeof(ViewTask) / 16)
        reinterpret_cast<uint4*>(&S.vt)[tid] =
            BATCH ? __ldg(reinterpret_cast<const uint4*>(table + v) + tid) : reinterpret_cast<const uint4*>(&t0)[tid];
      __syncthreads();
      cur = v;
      if (S.vt.s.mlp16 != weights) {
        weights = S.vt.s.mlp16;
        mlp::load_forward_weights(S.t, weights);  // the previous tile's MMAs are complete
      }
    }
    const ViewTask& t = S.vt;
    const uint64_t n = t.s.n;
    const uint64_t i = (tile - (BATCH ? t.proj_cta0 : 0u)) * mlp::kRows + tid;
    bool vis = false, used_fp64 = false;
    float dir[3] = {0.f, 0.f, 0.f};
    uint4 l0 = make_uint4(0, 0, 0, 0), l1 = l0;
    // The CTA's next tile of the same view is brought into L2 while this
    // one is projected and run through the MLP.
    const uint64_t i_next = i + (uint64_t)gridDim.x * mlp::kRows;
    if (i_next < n) {
      l2_prefetch(t.s.pos_k + i_next);
      l2_prefetch(t.s.geom16 + i_next);
      l2_prefetch(t.s.lat16 + 2 * i_next);
    }
    if (i < n) {
      l0 = __ldg(t.s.lat16 + 2 * i);  // in flight during the projection
      l1 = __ldg(t.s.lat16 + 2 * i + 1);
      project_splat<0, true, true>(t.fp, t.s, i, t.rec, t.bin, t.skip, dbg_proj, nullptr, vis, used_fp64, dir);
    }
    mlp::store_input(S.t.act, 0, tid, l0, l1, dir[0], dir[1], dir[2]);
    if (sync_or_abort()) { aborted = true; break; }
    if (tid == 0) {
      umma::fence_after_sync();
      mlp::gemm_k(tmem, act, 0, umma::smem_u32(S.t.w1f), 64, 2, mlp::kIdN64);
      umma::commit(mbar);
    }
    inflight = true;
    wait_mma();
    mlp::relu_epilogue(tmem, 0, nullptr, S.t.act, tid);  // h1 over x (layer 1 is done)
    if (sync_or_abort()) { aborted = true; break; }
    if (tid == 0) {
      umma::fence_after_sync();
      mlp::gemm_k(tmem, act, 0, umma::smem_u32(S.t.w2f), 64, 4, mlp::kIdN64);
      umma::commit(mbar);
    }
    inflight = true;
    wait_mma();
    mlp::relu_epilogue(tmem, 0, S.t.b2, S.t.act, tid);  // h2 over h1 (layer 2 is done)
    if (sync_or_abort()) { aborted = true; break; }
    if (tid == 0) {
      umma::fence_after_sync();
      mlp::gemm_k(tmem, act, 0, umma::smem_u32(S.t.w3f), 16, 4, mlp::kIdN16);
      umma::commit(mbar);
    }
    inflight = true;
    wait_mma();
    float z[16];
    umma::tmem_ld16(umma::tmem_warp_addr(tmem, 0), z);
    float rgb[3];
    for (int c = 0; c < 3; c++) rgb[c] = mlp::sigmoidf(z[c] + S.t.b3[c]);
    if (vis) {
      float* r = reinterpret_cast<float*>(t.rec + i);
      r[6] = rgb[0];  // r1.z, r1.w, r2.x
      r[7] = rgb[1];
      r[8] = rgb[2];
    }
    if (!BATCH && dbg_color && i < n)
      for (int c = 0; c < 3; c++) dbg_color[3 * i + c] = vis ? rgb[c] : 0.0f;
    count_visible(vis, used_fp64, fc, BATCH ? t.pad[0] : 0u);
    umma::fence_before_sync();
  }
  if (!aborted && __syncthreads_or(timed_out)) aborted = true;
  if (aborted) {
    if (tid == 0) atomicExch(&fc.st->error, 1u);
    if (inflight) umma::mbar_wait(mbar, phase, 100000000ull);  // the MMA still in flight
  }
  umma::fence_before_sync();
  __syncthreads();
  if (tid < 32) {
    umma::fence_after_sync();
    umma::tmem_free(tmem, kLearnedTmemCols);
  }
}

int learned_ctas_per_sm_times_sms() {
  static int sms[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  int& ns = sms[dev & 63];
  if (!ns && cudaDeviceGetAttribute(&ns, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) ns = 148;
  return 7 * ns;
}

}  // namespace

cudaError_t launch_project(const ViewTask& t, ViewTask* table, float* dbg_proj, float* dbg_color,
                           const FrameCounters& fc, cudaStream_t stream, uint32_t* launches) {
  if (t.s.learned) {
    const uint64_t tiles = (t.s.n + mlp::kRows - 1) / mlp::kRows;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(tiles, learned_ctas_per_sm_times_sms()));
    k_project_learned<false>
        <<<grid, kLearnedThreads, kLearnedSmem, stream>>>(t, table, 1u, 0ull, dbg_proj, dbg_color, fc);
    *launches += 1;
    return cudaGetLastError();
  }
  // An empty scene still stores the view table.
  const unsigned grid = t.s.n ? (unsigned)((t.s.n + 255) / 256) : 1u;
  const unsigned grid_tma = t.s.n ? (unsigned)((t.s.n + kTmaSplats - 1) / kTmaSplats) : 1u;
#define SPLAT_PROJECT(D)                                                                                        \
  do {                                                                                                          \
    if (t.s.fp16 || t.s.n == 0) {                                                                               \
      if (t.s.fp16)                                                                                             \
        k_project<D, true><<<grid, 256, 0, stream>>>(t, table, dbg_proj, dbg_color, fc);                        \
      else                                                                                                      \
        k_project<D, false><<<grid, 256, 0, stream>>>(t, table, dbg_proj, dbg_color, fc);                       \
    } else {                                                                                                    \
      /* raised once per device, outside capture: a scene's first frame is never captured */                 \
      static bool attr_set[64] = {};                                                                            \
      int dev = 0;                                                                                              \
      if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;                                                          \
      if (!attr_set[dev & 63]) {                                                                                \
        const cudaError_t ae = cudaFuncSetAttribute(k_project_tma<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                                    (int)TmaLayout<D>::kBytes);                                 \
        if (ae != cudaSuccess) return ae;                                                                       \
        attr_set[dev & 63] = true;                                                                              \
      }                                                                                                         \
      k_project_tma<D><<<grid_tma, kTmaSplats, TmaLayout<D>::kBytes, stream>>>(t, table, dbg_proj, dbg_color, fc);  \
    }                                                                                                           \
  } while (0)
  switch (t.s.sh_degree) {
    case 0: SPLAT_PROJECT(0); break;
    case 1: SPLAT_PROJECT(1); break;
    case 2: SPLAT_PROJECT(2); break;
    default: SPLAT_PROJECT(3); break;
  }
#undef SPLAT_PROJECT
  *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_project_learned_batch(ViewTask* table, uint32_t n_views, uint64_t total_tiles,
                                         const FrameCounters& fc, cudaStream_t stream, uint32_t* launches) {
  if (n_views == 0 || total_tiles == 0) return cudaSuccess;
  const unsigned grid =
      (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(total_tiles, learned_ctas_per_sm_times_sms()));
  k_project_learned<true><<<grid, kLearnedThreads, kLearnedSmem, stream>>>(ViewTask{}, table, n_views, total_tiles,
                                                                            nullptr, nullptr, fc);
  *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_project_batch(const ViewTask* table, uint32_t n_views, uint32_t total_ctas,
                                 const FrameCounters& fc, cudaStream_t stream, uint32_t* launches) {
  if (total_ctas == 0) return cudaSuccess;
  k_project_batch<<<total_ctas, kTmaSplats, TmaLayout<3>::kBytes, stream>>>(table, n_views, fc);
  *launches += 1;
  return cudaGetLastError();
}

}  // namespace splat
