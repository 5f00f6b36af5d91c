// Kernel (d): per-tile front-to-back blend with the terminal box-filter
// downsample fused in.
//
// A persistent kernel over the tiles of every view of the view table: each
// CTA of NT threads runs NT / G tile groups of G = min(NT, TW*TH) threads,
// and each group takes the next tile from a global counter until none is
// left (views of uneven resolution share one launch). A thread blends
// PPT = TW*TH / G pixels of its tile (one column, PPT consecutive rows); each
// warp covers an 8 x 4*PPT block of the tile, so a splat whose pixel bbox
// misses the block is skipped by the whole warp. The tile's depth-sorted
// splat list is walked in batches of G: the group gathers the batch's
// 48-byte records into shared memory (one per thread, the next batch's
// gather in flight while the current one blends), storing each splat's bbox
// as column and row bit masks; each warp lists the entries that touch its
// block (ballot compaction) and every pixel blends the batch front to back.
// A pixel stops once its transmittance drops below T_MIN; the group stops
// when a vote finds no live pixel (the reference stops a tile when all its
// row masks are empty, src/render/cpu.rs:693-702).
//
// Tile shapes 8x8, 16x16 (the reference's) and 32x16 with 128, 256 or 512
// threads are instantiated; the image does not depend on the choice (each
// pixel sees the same splats in the same order).
//
// Per pixel and splat the arithmetic is that of raster_tile
// (src/render/cpu.rs:638-703): power = (-a/2 dx^2 + -c/2 dy^2) + (-b dy) dx
// inside the splat's pixel bbox, alpha = min(opacity * exp(power), 0.99),
// masked by power <= 0 and alpha >= 1/255, C += colour * alpha * T,
// T *= 1 - alpha. EXACT = true evaluates it with the reference's x86 f32
// semantics (unfused multiply-adds, the polynomial exp_neg of
// src/render/simd.rs:315-331, and dx associated as the reference's 4-wide
// lanes of a 16-pixel tile do), which reproduces the cpu backend's image bit
// for bit; EXACT = false uses FMA and the hardware exp2 (the default).
// The result is quantised with to_u8 (src/render/mod.rs:282-285) and, for a
// downsample factor f dividing the tile shape, averaged over f x f blocks in
// shared memory with term::downsample's truncating integer division
// (src/term.rs:74-99); other factors go through a full-resolution scratch
// frame and k_downsample.
#include <atomic>
#include <cstddef>

#include "common.cuh"
#include "tilesort.cuh"
#include "umma.cuh"

namespace splat {
namespace {

constexpr float kLog2e = 1.44269504088896340736f;
constexpr float kLog2AlphaMin = -7.99435343685886f;  // log2(1/255)
constexpr float kLog2AlphaMax = -0.0144995696951f;   // log2(0.99)

// src/render/simd.rs:315-331 with the portable F4's unfused mul_add.
__device__ __forceinline__ float exp_neg_exact(float xin) {
  const float C1 = 0.6933594f;
  const float C2 = -2.1219444e-4f;
  const float x = fmaxf(xin, -87.0f);
  const float n = rintf(__fmul_rn(x, kLog2e));
  const float f = __fsub_rn(__fsub_rn(x, __fmul_rn(n, C1)), __fmul_rn(n, C2));
  float p = 1.9875691e-4f;
  p = __fadd_rn(1.3981999e-3f, __fmul_rn(p, f));
  p = __fadd_rn(8.333452e-3f, __fmul_rn(p, f));
  p = __fadd_rn(4.1665796e-2f, __fmul_rn(p, f));
  p = __fadd_rn(1.6666665e-1f, __fmul_rn(p, f));
  p = __fadd_rn(0.5f, __fmul_rn(p, f));
  const float f2 = __fmul_rn(f, f);
  const float r = __fadd_rn(__fadd_rn(f, 1.0f), __fmul_rn(p, f2));
  return __fmul_rn(r, __int_as_float(((int)n + 127) << 23));
}

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// to_u8 (src/render/mod.rs:282-285)
__device__ __forceinline__ uint32_t to_u8(float v) {
  const float c = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);  // f32::clamp; NaN passes
  const float q = __fadd_rn(__fmul_rn(c, 255.0f), 0.5f);
  if (!(q > 0.0f)) return 0u;
  if (q >= 255.0f) return 255u;
  return (uint32_t)q;
}


// Default path staging. With the splat's centre in the pixel coordinates
// of the 32 x 16 block of the frame that holds the tile (xs, ys; the same
// block whatever the tile shape), its conic
// times log2 e (A, B, C: power = A dx^2 + B dx dy + C dy^2 in log2 units,
// dx = x - xs, dy = y - ys) and lop = log2 opacity, the exponent
// pw' = power + lop is expanded once per splat into a quadratic in the
// pixel's own tile coordinates (x, y):
//   pw' = A x^2 + B x y + C y^2 + D x + E y + F,
//   D = -2 A xs - B ys, E = -2 C ys - B xs, F = A xs^2 + B xs ys + C ys^2 + lop,
// so that a pixel evaluates it in five fused multiply-adds. alpha =
// 2^min(pw', cap) with cap = min(lop, log2 0.99) is min(opacity exp(power),
// 0.99) with power <= 0 enforced, and the alpha test is pw' >= log2(1/255).
// The expansion's terms stay within the ellipse's own scale wherever the
// splat contributes (a pixel in reach is within its k-sigma extent), so the
// f32 cancellation it adds is about 1e-6 in log2 units.
// a = (A, B, C, D), b = (E, F, cap, red), c = (green, blue).
__device__ __forceinline__ void stage_splat(const Record& r, float ox05, float oy05, float4& a, float4& b, float2& c) {
  const float lop = __log2f(r.r1.y);
  const float xs = r.r0.x - ox05, ys = r.r0.y - oy05;
  const float A = r.r0.z * kLog2e, B = r.r0.w * kLog2e, C = r.r1.x * kLog2e;
  const float D = -2.0f * A * xs - B * ys, E = -2.0f * C * ys - B * xs;
  const float F = (A * xs * xs + B * xs * ys) + (C * ys * ys + lop);
  a = make_float4(A, B, C, D);
  b = make_float4(E, F, fminf(lop, kLog2AlphaMax), r.r1.z);
  c = make_float2(r.r1.w, r.r2.x);
}

// Default path alpha from the staged splat (stage_splat) at the pixel's
// coordinates (x, y) in the 32 x 16 block; 0 when below the alpha threshold.
// Every blend shape evaluates this same expression with the same operands,
// so images do not depend on the shape.
__device__ __forceinline__ float fast_alpha(const float4& a, const float4& b, float x, float y) {
  const float pw = fminf(fmaf(x, fmaf(a.x, x, fmaf(a.y, y, a.w)), fmaf(y, fmaf(a.z, y, b.x), b.y)), b.z);
  return pw >= kLog2AlphaMin ? ex2_approx(pw) : 0.0f;
}

template <bool EXACT>
__device__ __forceinline__ float splat_alpha(bool inbox, const float4& a, const float4& b, float fx05, float gbase,
                                             float lanef, float rowc, float lxf, float lyf) {
  if (EXACT) {
    const float cx0 = __fsub_rn(fx05, a.x);
    const float dx = __fadd_rn(lanef, __fadd_rn(gbase, cx0));
    const float qx = __fmul_rn(__fmul_rn(dx, dx), a.z);
    const float dy = __fsub_rn(rowc, a.y);
    const float qy = __fmul_rn(__fmul_rn(b.x, dy), dy);
    const float bdy = __fmul_rn(a.w, dy);
    const float pw = __fadd_rn(__fadd_rn(qx, qy), __fmul_rn(bdy, dx));
    const float alpha = fminf(__fmul_rn(exp_neg_exact(pw), b.y), kAlphaMax);
    const bool on = (pw <= 0.0f) && (alpha >= kAlphaMin) && inbox;
    return on ? alpha : 0.0f;
  } else {
    // A pixel outside the splat's bbox is at least half a pixel beyond the
    // ellipse on which opacity * exp(power) = 1/255 (the bbox is the k-sigma
    // extent rounded outwards and pixels are sampled at their centres), so
    // the alpha test alone excludes it here; the exact path also tests the
    // bbox, as the reference does.
    return fast_alpha(a, b, lxf, lyf);
  }
}

// C += colour * alpha * T, T *= 1 - alpha.
template <bool EXACT>
__device__ __forceinline__ void accumulate(float alpha, float red, float green, float blue, float& T, float& cr,
                                           float& cg, float& cb) {
  if (EXACT) {
    const float w = __fmul_rn(alpha, T);
    cr = __fadd_rn(cr, __fmul_rn(red, w));
    cg = __fadd_rn(cg, __fmul_rn(green, w));
    cb = __fadd_rn(cb, __fmul_rn(blue, w));
    T = __fmul_rn(T, __fsub_rn(1.0f, alpha));
  } else {
    const float w = alpha * T;
    cr = fmaf(red, w, cr);
    cg = fmaf(green, w, cg);
    cb = fmaf(blue, w, cb);
    T = T - w;
  }
}
// The staged colour: exact path (red, green) in b.zw and blue in c.x; default
// path red in b.w, (green, blue) in c (stage_splat).
template <bool EXACT>
__device__ __forceinline__ void staged_colour(const float4& b, const float2& c, float& red, float& green,
                                              float& blue) {
  if (EXACT) {
    red = b.z;
    green = b.w;
    blue = c.x;
  } else {
    red = b.w;
    green = c.x;
    blue = c.y;
  }
}

// Bits [lo, hi) of a 32-bit mask (0 <= lo <= hi <= 32).
__device__ __forceinline__ uint32_t bit_range(int lo, int hi) {
  return (uint32_t)(((1ull << hi) - 1ull) & ~((1ull << lo) - 1ull));
}

// Barrier over the `count` threads of named barrier `id` (0 = the whole CTA).
__device__ __forceinline__ void group_sync(uint32_t id, uint32_t count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Barrier with a population count of `pred` over the same threads.
__device__ __forceinline__ uint32_t group_count(uint32_t id, uint32_t count, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.popc.u32 %0, %2, %3, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(id), "r"(count)
      : "memory");
  return r;
}

template <int TW, int TH, int NT>
struct BlendShape {
  static constexpr int P = TW * TH;         // pixels per tile
  static constexpr int G = NT < P ? NT : P;  // threads per tile group
  static constexpr int NG = NT / G;          // tile groups per CTA
  static constexpr int PPT = P / G;          // pixels per thread
  static constexpr int GW = G / 32;          // warps per group
  static constexpr int BH = 4 * PPT;         // warp block height (width 8)
  static constexpr int WCOLS = TW / 8;       // warp blocks per tile row
  static_assert(TW % 8 == 0 && TH % BH == 0 && WCOLS * (TH / BH) == GW, "tile shape and threads");
  static_assert(TW <= 32 && TH <= 16, "bbox masks hold 32 columns and 16 rows");
  static_assert(NG <= 8, "named barriers 1..8");
};

// A batch of G staged splats: centre, conic, opacity, colour, bbox masks.
template <int G>
struct __align__(16) StagedBatch {
  float4 a[G];  // see stage_splat (exact path: the record's r0)
  float4 b[G];  // see stage_splat (exact path: the record's r1)
  float2 c[G];  // see staged_colour
  uint32_t mx[G];
  uint32_t my[G];
  uint32_t wm[G];  // the warp blocks the splat reaches (block_mask)
};

// The warp blocks of the tile at (ox, oy) that hold a pixel centre the
// splat (record r) reaches: bit w for the group's warp w (block column
// w % WCOLS, row w / WCOLS, 8 x BH pixels), among those its bbox masks
// (mx, my) meet. As the projection bounds the tiles (ellipse_skips): with
// the conic (a, b, c) and K = 2 ln(255 opacity), alpha >= 1/255 where
// a dx^2 + 2 b dx dy + c dy^2 <= K; per block row, the ellipse's x range in
// the row's band of pixel-centre rows, from its leftmost and rightmost
// points clamped into the band (K widened by 0.2 % + 0.002, the range by
// 0.01 px). A block left out holds only pixels whose alpha test fails, so
// leaving it out of the warp's list changes no pixel. A splat the test
// cannot bound keeps every block its bbox meets.
template <class S>
__device__ __forceinline__ uint32_t block_mask(const Record& r, uint32_t ox, uint32_t oy, uint32_t mx, uint32_t my) {
  constexpr int BROWS = S::GW / S::WCOLS;
  uint32_t box = 0;  // the blocks the bbox meets
#pragma unroll
  for (int by = 0; by < BROWS; by++)
    if (my & (((1u << S::BH) - 1u) << (by * S::BH)))
#pragma unroll
      for (int bx = 0; bx < S::WCOLS; bx++)
        if (mx & (0xFFu << (bx * 8))) box |= 1u << (by * S::WCOLS + bx);
  if (__popc(box) <= 1) return box;
  const float a = -2.0f * r.r0.z, bb = -r.r0.w, c = -2.0f * r.r1.x;
  const float p = bb * bb, det = fmaf(a, c, -p) - fmaf(bb, bb, -p);
  const float K = fmaf(1.38629436f * (lg2_hw(r.r1.y) + 7.99435344f), 1.002f, 0.002f);
  if (!(det > 0.0f && a > 0.0f && c > 0.0f && K > 0.0f)) return box;
  const float inv_det = rcp_hw(det), inv_a = rcp_hw(a), aK = a * K;
  const float ey = sqrt_hw(aK * inv_det), xm = sqrt_hw(c * K * inv_det);
  const float dyr = -bb * xm * rcp_hw(c);
  uint32_t m = 0;
#pragma unroll
  for (int by = 0; by < BROWS; by++) {
    if (!((box >> (by * S::WCOLS)) & ((1u << S::WCOLS) - 1u))) continue;
    const float band0 = (float)(oy + by * S::BH) + 0.5f - r.r0.y, band1 = band0 + (float)(S::BH - 1);
    if (band1 < -ey || band0 > ey) continue;
    const float lo = fmaxf(band0, -ey), hi = fminf(band1, ey);
    const float yr = fminf(fmaxf(dyr, lo), hi), yl = fminf(fmaxf(-dyr, lo), hi);
    const float sr = sqrt_hw(fmaxf(aK - det * yr * yr, 0.0f)), sl = sqrt_hw(fmaxf(aK - det * yl * yl, 0.0f));
    const float xu = r.r0.x + (sr - bb * yr) * inv_a + 0.01f, xl = r.r0.x - (sl + bb * yl) * inv_a - 0.01f;
#pragma unroll
    for (int bx = 0; bx < S::WCOLS; bx++) {
      const float c0 = (float)(ox + bx * 8) + 0.5f;
      if (c0 + 7.0f >= xl && c0 <= xu) m |= 1u << (by * S::WCOLS + bx);
    }
  }
  return m & box;
}

// The default shape (16x16 tiles, two groups of 256 threads per CTA) sorts
// each tile of at most kMidSortCap pairs itself, before blending it (the
// other shapes leave that to k_sort_small / k_sort_mid).
template <int TW, int TH, int NT>
constexpr bool kSortsTiles = TW == 16 && TH == 16 && NT == 512;

// Shared memory of one tile group: two staged batches (the group blends one
// while it stages the next), the warps' lists of batch entries, the tile's
// quantised pixels for the fused downsample, the group's tile and its pair-
// count class. Groups that sort their tiles overlay the tile's words (and,
// before them, the sort's counters) on the blend's arrays, which are idle
// while the tile is sorted, and keep the sorted order in `slot`.
template <int TW, int TH, int NT>
struct __align__(16) GroupSmem {
  using S = BlendShape<TW, TH, NT>;
  static constexpr bool kSort = kSortsTiles<TW, TH, NT>;
  struct Blend {
    StagedBatch<S::G> bt[2];
    uint16_t list[S::GW][S::G];
    uint32_t px[S::P];
  };
  // The tile's words as the bulk copy brings them in (with one word of
  // alignment slack in front and one behind) and the counting sort's 4096
  // 16-bit counters, overlaid on the blend's arrays while the tile is sorted.
  struct Sort {
    uint64_t words[kSort ? kMidSortCap + 2 : 1];
    uint32_t hist[kSort ? kCountBuckets / 2 : 1];
  };
  union {
    Blend b;
    Sort srt;
  };
  uint16_t slot[kSort ? kMidSortCap : 1];
  uint32_t red[2][S::GW];
  uint32_t wsum[S::GW];
  uint64_t mbar;  // completion of the tile's bulk copy
  uint32_t work, cls;
};

// The per-tile depth sort of a tile of n <= kMidSortCap pairs by its group
// of 256 threads (thread t). The tile's words (w, in the pair buffer) come
// into shared memory by one bulk asynchronous copy (TMA, cp.async.bulk,
// completing on the group's mbarrier; the copy starts at the 16-byte boundary
// at or below the tile and the pair buffer has slack for its rounded-up
// end), and the sort reads them there: the counting pass of smem_count_sort
// (a 12-bit monotone quantisation of the depth over the tile's range,
// positions from shared-memory atomics on 16-bit packed counters), then runs
// of equal key ordered by the full word (a run longer than one thread orders
// sends the whole tile through a bitonic sort). The result is the
// reference's (depth, scene index) order, as k_sort_small / k_sort_mid
// produce it; it is left in sm.slot (the group stages word w[slot[k]] as the
// k-th: the function returns true) unless the words had to be reordered
// (the bitonic sort) or write_back asks for them (the frame keeps its sorted
// pairs for inspection): then they are written back to w in order and the
// function returns false. A copy that does not land within the bounded wait
// sets the frame's error flag; the sort then reads the words from w. sync()
// is the group's barrier, any(p) its vote, phase the mbarrier's parity.
template <class Sm, class Sync, class Any>
__device__ __forceinline__ bool group_sort_tile(uint64_t* w, uint32_t n, Sm& sm, uint32_t t, Sync&& sync, Any&& any,
                                                bool write_back, uint32_t& phase, DevState* st) {
  constexpr uint32_t kThreads = 256;
  static_assert(kCountBuckets == 16 * kThreads, "16 counters per thread");
  const uint32_t lane = t & 31, warp = t >> 5;
  uint32_t* hist = sm.srt.hist;
  const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&sm.mbar);
  const uint32_t off = (uint32_t)((reinterpret_cast<uintptr_t>(w) >> 3) & 1u);  // words below the 16-byte boundary
  if (t == 0) {
    const uint32_t bytes = ((n + off) * 8u + 15u) & ~15u;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            (uint32_t)__cvta_generic_to_shared(sm.srt.words)),
        "l"(w - off), "r"(bytes), "r"(mbar)
        : "memory");
  }
  for (uint32_t b = t; b < kCountBuckets / 2; b += kThreads) hist[b] = 0u;
  bool landed = umma::mbar_wait(mbar, phase);
  if (!any(!landed)) {
    landed = true;
  } else {  // the whole group takes the same path: wait (bounded) for the copy, read w
    if (t == 0) atomicExch(&st->error, 3u);
    umma::mbar_wait(mbar, phase, 100000000ull);
    landed = false;
  }
  phase ^= 1u;
  const uint64_t* src = landed ? sm.srt.words + off : w;
  uint32_t mn = 0xFFFFFFFFu, mx = 0u;
  for (uint32_t e = t; e < n; e += kThreads) {
    const uint32_t d = (uint32_t)(src[e] >> 32);
    mn = min(mn, d);
    mx = max(mx, d);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if (lane == 0) {
    sm.red[0][warp] = mn;
    sm.red[1][warp] = mx;
  }
  sync();
#pragma unroll
  for (int k = 0; k < 8; k++) {
    mn = min(mn, sm.red[0][k]);
    mx = max(mx, sm.red[1][k]);
  }
  const float dmin = __uint_as_float(mn), range = __uint_as_float(mx) - dmin;
  const float scale = range > 0.0f ? (float)(kCountBuckets - 1) / range : 0.0f;
  auto quant = [&](uint64_t x) -> uint32_t {
    const float q = (__uint_as_float((uint32_t)(x >> 32)) - dmin) * scale;
    return q >= (float)(kCountBuckets - 1) ? kCountBuckets - 1 : (uint32_t)q;
  };
  for (uint32_t e = t; e < n; e += kThreads) {
    const uint32_t q = quant(src[e]);
    atomicAdd(&hist[q >> 1], 1u << (16 * (q & 1u)));
  }
  sync();
  // Exclusive scan of the 4096 counters, 16 per thread.
  uint32_t c[16], sum = 0;
  uint4* h4 = reinterpret_cast<uint4*>(hist + 8 * t);
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const uint4 v = h4[k];
    const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      c[8 * k + 2 * j] = w4[j] & 0xFFFFu;
      c[8 * k + 2 * j + 1] = w4[j] >> 16;
    }
  }
#pragma unroll
  for (int k = 0; k < 16; k++) sum += c[k];
  uint32_t x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm.wsum[warp] = x;
  sync();
  uint32_t run = x - sum;
  for (uint32_t k = 0; k < warp; k++) run += sm.wsum[k];
  uint32_t pk[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const uint32_t lo = run;
    run += c[2 * j];
    pk[j] = lo | (run << 16);
    run += c[2 * j + 1];
  }
  h4[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
  h4[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  sync();
  for (uint32_t e = t; e < n; e += kThreads) {
    const uint32_t q = quant(src[e]), sh = 16 * (q & 1u);
    sm.slot[(atomicAdd(&hist[q >> 1], 1u << sh) >> sh) & 0xFFFFu] = (uint16_t)e;
  }
  sync();
  const bool long_run = sort_short_runs(
      sm.slot, n, t, kThreads, [&](uint16_t i) { return quant(src[i]); }, [&](uint16_t i) { return src[i]; });
  const bool any_long = any(long_run);  // also the barrier after the runs
  if (!any_long && !write_back) return true;
  if (!landed) return true;  // degraded (the frame reports the error): long runs stay unordered
  uint64_t* sw = sm.srt.words + off;
  if (any_long) {
    bitonic_sort(sw, n, t, kThreads, sync);
    for (uint32_t e = t; e < n; e += kThreads) w[e] = sw[e];
  } else {
    for (uint32_t e = t; e < n; e += kThreads) w[e] = sw[sm.slot[e]];
  }
  sync();  // the group's staging reads the sorted words next
  return false;
}

// COUNT: also counts the pixel/splat evaluations (the blend's unit of work
// after early termination) into st->evals; a separate instantiation, used
// only when SPLAT_OPT_COUNT_EVALS asks for it.
//
// The pair words are read with ordinary (coherent) loads: groups of the
// default shape sort their tile in place before they stage it.
template <bool EXACT, int TW, int TH, int NT, bool ROWS, bool COUNT = false>
__global__ void __launch_bounds__(NT, NT == 512 ? 2 : (NT == 256 ? 5 : 8)) k_blend(const ViewTask* __restrict__ table, uint32_t n_views, uint32_t n_tiles,
                                              uint64_t* pairs, const uint2* __restrict__ ranges,
                                              const uint32_t* __restrict__ order, DevState* st) {
  using S = BlendShape<TW, TH, NT>;
  using Smem = GroupSmem<TW, TH, NT>;
  constexpr int G = S::G, PPT = S::PPT;
  extern __shared__ __align__(16) unsigned char s_raw[];
  const int tid = threadIdx.x, lane = tid & 31;
  const int g = tid / G, gt = tid % G, gw = gt >> 5;
  Smem& sm = reinterpret_cast<Smem*>(s_raw)[g];
  const uint32_t bar = S::NG == 1 ? 0u : 1u + (uint32_t)g;
  auto sync = [&]() {
    if (S::NG == 1)
      __syncthreads();
    else
      group_sync(bar, G);
  };
  auto count = [&](bool p) -> uint32_t {
    if (S::NG == 1) return (uint32_t)__syncthreads_count(p);
    return group_count(bar, G, p);
  };

  const uint32_t wbx = gw % S::WCOLS, wby = gw / S::WCOLS;
  const uint32_t lx = wbx * 8 + (lane & 7);
  const uint32_t ly0 = wby * S::BH + (lane >> 3) * PPT;

  // Tiles are taken by pair-count class (tile_class), each class's list in
  // the order k_tile_ranges appended it.
  __shared__ uint32_t s_cls[kTileClasses];
  if (tid < kTileClasses) s_cls[tid] = st->cls[tid];
  if constexpr (Smem::kSort) {
    if (gt == 0) umma::mbar_init((uint32_t)__cvta_generic_to_shared(&sm.mbar), 1);
  }
  uint32_t sort_phase = 0;  // parity of the group's next bulk-copy completion
  __syncthreads();
  for (;;) {
    if (gt == 0) {
      uint32_t w = atomicAdd(&st->blend_next, 1u), tl = 0xFFFFFFFFu, cl = kTileClasses;
#pragma unroll
      for (int i = 0; i < kTileClasses; i++) {
        // Frames in mapped host memory (ROWS) take the empty and the lightest
        // tiles first: their rows then cross the bus while the heavy tiles
        // compute, instead of in one burst at the end of the frame (classes
        // 6, 5, 0, 1, 2, 3, 4); device frames take the heaviest first.
        const int k = ROWS ? (i < 2 ? kTileClasses - 1 - i : i - 2) : i;
        if (w < s_cls[k]) {
          tl = order[(size_t)k * n_tiles + w];
          cl = (uint32_t)k;
          break;
        }
        w -= s_cls[k];
      }
      sm.work = tl;
      sm.cls = cl;
    }
    sync();
    const uint32_t tile = sm.work;
    if (tile >= n_tiles) break;
    const uint32_t v = find_view(table, n_views, tile, offsetof(ViewTask, tile0));
    const ViewTask* tv = table + v;
    const uint32_t local = tile - tv->tile0;
    const uint32_t tiles_x = tv->fp.tiles_x;
    if (local >= tiles_x * tv->fp.tiles_y) {  // alignment padding between views
      sync();
      continue;
    }
    // Rows [Y0, Y1) and columns [X0, X1) of the frame are rendered; output
    // row = frame row - OY.
    const uint32_t W = tv->fp.w, Y0 = tv->fp.win_y0, Y1 = min(tv->fp.h, Y0 + tv->fp.win_rows);
    const uint32_t X0 = tv->fp.win_x0, X1 = min(W, X0 + tv->fp.win_cols), OY = tv->fp.out_y0;
    const Record* __restrict__ rec = tv->rec;
    const uint32_t ox = (local % tiles_x + tv->fp.win_tx0) * TW, oy = (local / tiles_x + tv->fp.win_ty0) * TH;
    const uint32_t px = ox + lx;

    // EXACT: dx = lane + ((g*4) + ((ox16 + 0.5) - x)), dy = (py + 0.5) - y
    // in the reference's association, ox16 the pixel's 16-pixel tile origin
    // (src/render/cpu.rs:658-671).
    const float fx05 = __fadd_rn((float)(px & ~15u), 0.5f);
    const float gbase = (float)(px & 12u), lanef = (float)(px & 3u);
    // Default path: the staged exponent is a quadratic in pixel coordinates
    // relative to the 32 x 16 block of the frame that holds the tile (qx0,
    // qy0), the same block for every tile shape, so that a pixel's
    // arithmetic and image do not depend on the shape.
    const uint32_t qx0 = ox & ~31u, qy0 = oy & ~15u;
    const float ox05 = (float)qx0 + 0.5f, oy05 = (float)qy0 + 0.5f;
    const float qxf = (float)(px - qx0);

    float T[PPT], cr[PPT], cg[PPT], cb[PPT];
    uint32_t evals = 0;
    bool done[PPT];
    bool all_done = true;
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      T[k] = 1.0f;
      cr[k] = cg[k] = cb[k] = 0.0f;
      done[k] = !(px >= X0 && px < X1 && oy + ly0 + k >= Y0 && oy + ly0 + k < Y1);
      all_done = all_done && done[k];
    }

    const uint2 range = ranges[tile];
    const uint32_t begin = range.x, n = range.y > range.x ? range.y - range.x : 0u;
    bool use_slot = false;
    if constexpr (Smem::kSort) {
      // Tiles of classes 1-5 (2 .. kMidSortCap pairs) are sorted here; longer
      // ones were sorted by k_sort_long.
      use_slot = sm.cls >= 1 && sm.cls <= 5 && n >= 2 &&
                 group_sort_tile(pairs + begin, n, sm, (uint32_t)gt, sync, [&](bool p) { return count(p) != 0; },
                                 (tv->fp.flags & kFrameKeepSortedPairs) != 0u, sort_phase, st);
    }
    // The k-th pair word of the tile in depth order.
    auto word_at = [&](uint32_t k) -> uint64_t { return pairs[begin + (use_slot ? (uint32_t)sm.slot[k] : k)]; };
    // Batch k is staged into buffer k & 1 by the group while it blends batch
    // k - 1 from the other buffer; the barrier that ends batch k - 1 (the
    // early-exit vote) publishes it. The records of batch k + 1 are in
    // flight during the blend of batch k.
    Record nr{};
    bool has = false;
    auto stage = [&](StagedBatch<G>& d) {
      const uint32_t bx = __float_as_uint(nr.r2.y), by = __float_as_uint(nr.r2.z);
      const int x0 = min(max((int)(bx & 0xFFFFu) - (int)ox, 0), TW), x1 = min(max((int)(bx >> 16) - (int)ox, 0), TW);
      const int y0 = min(max((int)(by & 0xFFFFu) - (int)oy, 0), TH), y1 = min(max((int)(by >> 16) - (int)oy, 0), TH);
      d.mx[gt] = x1 > x0 ? bit_range(x0, x1) : 0u;
      d.my[gt] = y1 > y0 ? bit_range(y0, y1) : 0u;
      d.wm[gt] = block_mask<S>(nr, ox, oy, d.mx[gt], d.my[gt]);
      if (EXACT) {
        d.a[gt] = nr.r0;
        d.b[gt] = nr.r1;
        d.c[gt] = make_float2(nr.r2.x, 0.0f);
      } else {
        float4 a, b;
        float2 c;
        stage_splat(nr, ox05, oy05, a, b, c);
        d.a[gt] = a;
        d.b[gt] = b;
        d.c[gt] = c;
      }
    };
    if (n > 0) {
      if ((uint32_t)gt < n) {
        nr = rec[(uint32_t)word_at(gt)];
        stage(sm.b.bt[0]);
      }
      has = (uint32_t)gt + G < n;
      if (has) nr = rec[(uint32_t)word_at(G + gt)];
      sync();
    }
    for (uint32_t start = 0, buf = 0; start < n; start += G, buf ^= 1u) {
      const StagedBatch<G>& bt = sm.b.bt[buf];
      const uint32_t cnt = min((uint32_t)G, n - start);
      // This warp's list of batch entries whose bbox meets its block.
      uint32_t len = 0;
      if (__any_sync(0xffffffffu, !all_done)) {
        for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
          const uint32_t e = c0 + lane;
          const bool hit = e < cnt && ((bt.wm[e] >> gw) & 1u);
          const uint32_t bal = __ballot_sync(0xffffffffu, hit);
          if (hit) sm.b.list[gw][len + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)e;
          len += __popc(bal);
        }
        __syncwarp();
      }
      if (!all_done) {
        if constexpr (PPT == 1) {
          // Two splats per iteration, without branches on alpha: a splat
          // below the alpha test contributes alpha = 0, which leaves C and T
          // unchanged bit for bit; the second splat is dropped (alpha = 0)
          // when the first one saturated the pixel.
          const float rowc = (float)(oy + ly0) + 0.5f, lxf = qxf, lyf = (float)(oy + ly0 - qy0);
          const uint32_t ybit = 1u << ly0, xbit = 1u << lx;
          const uint16_t* lst = sm.b.list[gw];
          uint32_t k = 0;
          for (; k + 1 < len; k += 2) {
            const uint32_t jj = *reinterpret_cast<const uint32_t*>(lst + k);  // k even: 4-byte aligned
            const uint32_t j0 = jj & 0xFFFFu, j1 = jj >> 16;
            const float4 a0 = bt.a[j0], b0 = bt.b[j0];
            const float4 a1 = bt.a[j1], b1 = bt.b[j1];
            const bool in0 = !EXACT || ((bt.mx[j0] & xbit) && (bt.my[j0] & ybit));
            const bool in1 = !EXACT || ((bt.mx[j1] & xbit) && (bt.my[j1] & ybit));
            const float al0 = splat_alpha<EXACT>(in0, a0, b0, fx05, gbase, lanef, rowc, lxf, lyf);
            const float al1 = splat_alpha<EXACT>(in1, a1, b1, fx05, gbase, lanef, rowc, lxf, lyf);
            float r_, g_, b_;
            if (COUNT) evals += 2;
            staged_colour<EXACT>(b0, bt.c[j0], r_, g_, b_);
            accumulate<EXACT>(al0, r_, g_, b_, T[0], cr[0], cg[0], cb[0]);
            const bool sat0 = T[0] < kTMin;
            staged_colour<EXACT>(b1, bt.c[j1], r_, g_, b_);
            accumulate<EXACT>(sat0 ? 0.0f : al1, r_, g_, b_, T[0], cr[0], cg[0], cb[0]);
            if (sat0 || T[0] < kTMin) {
              done[0] = true;
              break;
            }
          }
          if (!done[0] && k < len) {
            const uint32_t j0 = lst[k];
            const float4 a0 = bt.a[j0], b0 = bt.b[j0];
            const bool in0 = !EXACT || ((bt.mx[j0] & xbit) && (bt.my[j0] & ybit));
            const float al0 = splat_alpha<EXACT>(in0, a0, b0, fx05, gbase, lanef, rowc, lxf, lyf);
            float r_, g_, b_;
            if (COUNT) evals += 1;
            staged_colour<EXACT>(b0, bt.c[j0], r_, g_, b_);
            accumulate<EXACT>(al0, r_, g_, b_, T[0], cr[0], cg[0], cb[0]);
            if (T[0] < kTMin) done[0] = true;
          }
          all_done = done[0];
        } else {
          const uint32_t xbit = 1u << lx;
          for (uint32_t k = 0; k < len && !all_done; k++) {
            const uint32_t j = sm.b.list[gw][k];
            const float4 a = bt.a[j], b = bt.b[j];
            const uint32_t mx = bt.mx[j], my = bt.my[j];
            float red, green, blue;
            staged_colour<EXACT>(b, bt.c[j], red, green, blue);
            all_done = true;
#pragma unroll
            for (int q = 0; q < PPT; q++) {
              if (!done[q]) {
                const uint32_t ly = ly0 + q;
                const bool in = !EXACT || ((mx & xbit) && ((my >> ly) & 1u));
                const float al = splat_alpha<EXACT>(in, a, b, fx05, gbase, lanef, (float)(oy + ly) + 0.5f,
                                                    qxf, (float)(oy + ly - qy0));
                if (COUNT) evals += 1;
                if (al > 0.0f) {
                  accumulate<EXACT>(al, red, green, blue, T[q], cr[q], cg[q], cb[q]);
                  if (T[q] < kTMin) done[q] = true;
                }
              }
              all_done = all_done && done[q];
            }
          }
        }
      }
      const uint32_t nxt = start + 2 * G + gt;
      if (has) stage(sm.b.bt[buf ^ 1u]);  // batch start + G
      has = nxt < n;
      if (has) nr = rec[(uint32_t)word_at(nxt)];
      if (count(!all_done) == 0) break;
    }

    if (COUNT) {
      uint32_t e = evals;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
      if (lane == 0 && e) atomicAdd(&st->evals, (unsigned long long)e);
    }
    // C + T * bg, quantised (the reference adds unfused: c + (t * bg)).
    const uint32_t f = tv->fp.downsample;
    uint8_t* __restrict__ out = tv->out;
    const float bg0 = tv->fp.bg[0], bg1 = tv->fp.bg[1], bg2 = tv->fp.bg[2];
    const bool fused = f > 1 && TW % f == 0 && TH % f == 0;
    // ROWS (frames in mapped pinned host memory; f == 1, the tile inside the
    // frame, rows 4-byte aligned): the tile leaves as whole 4-byte words of
    // its rows, consecutive threads writing consecutive words, so the bus
    // carries contiguous row segments rather than single bytes. Device
    // frames keep the per-pixel byte stores (a separate instantiation: the
    // word path costs the device-frame kernel about 4 %).
    constexpr uint32_t kRowWords = (TW * 3) / 4;  // TW is a multiple of 8
    const bool rows = ROWS && f == 1 && W % 4u == 0 && ox >= X0 && ox + TW <= X1 &&
                      (reinterpret_cast<uintptr_t>(out) & 3u) == 0;
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      const uint32_t ly = ly0 + k, py = oy + ly;
      const uint32_t qr = to_u8(__fadd_rn(cr[k], __fmul_rn(T[k], bg0)));
      const uint32_t qg = to_u8(__fadd_rn(cg[k], __fmul_rn(T[k], bg1)));
      const uint32_t qb = to_u8(__fadd_rn(cb[k], __fmul_rn(T[k], bg2)));
      if (fused || rows) {
        sm.b.px[ly * TW + lx] = qr | (qg << 8) | (qb << 16);
      } else if (px >= X0 && px < X1 && py >= Y0 && py < Y1) {
        // f == 1: the frame (window); other factors: the full-resolution
        // scratch frame (whole frames: OY = 0).
        uint8_t* o = (f == 1 ? out : tv->full) + ((size_t)(py - OY) * W + px) * 3;
        o[0] = (uint8_t)qr;
        o[1] = (uint8_t)qg;
        o[2] = (uint8_t)qb;
      }
    }
    if (ROWS && rows) {
      sync();
      for (uint32_t e = gt; e < TH * kRowWords; e += G) {
        const uint32_t ly = e / kRowWords, b0 = 4u * (e % kRowWords), py = oy + ly;  // b0: byte of the row
        if (py >= Y0 && py < Y1) {
          uint32_t v = 0u;
#pragma unroll
          for (uint32_t r = 0; r < 4; r++) {
            const uint32_t bb = b0 + r;
            v |= ((sm.b.px[ly * TW + bb / 3u] >> (8u * (bb % 3u))) & 255u) << (8u * r);
          }
          *reinterpret_cast<uint32_t*>(out + ((size_t)(py - OY) * W + ox) * 3 + b0) = v;
        }
      }
    }
    if (fused) {
      sync();
      const uint32_t pw_ = TW / f, ph_ = TH / f;  // output pixels of the tile
      if ((uint32_t)gt < pw_ * ph_) {
        const uint32_t bxl = gt % pw_, byl = gt / pw_;
        const uint32_t obx = ox / f + bxl, oby = oy / f + byl;
        if (obx < tv->fp.out_w && oby < tv->fp.out_h) {
          uint32_t acc[3] = {0u, 0u, 0u};
          for (uint32_t sy = 0; sy < f; sy++)
            for (uint32_t sx = 0; sx < f; sx++) {
              const uint32_t p = sm.b.px[(byl * f + sy) * TW + bxl * f + sx];
              acc[0] += p & 255u;
              acc[1] += (p >> 8) & 255u;
              acc[2] += (p >> 16) & 255u;
            }
          const uint32_t nn = f * f;
          uint8_t* o = out + ((size_t)oby * tv->fp.out_w + obx) * 3;
          o[0] = (uint8_t)(acc[0] / nn);
          o[1] = (uint8_t)(acc[1] / nn);
          o[2] = (uint8_t)(acc[2] / nn);
        }
      }
    }
    // The group's shared memory is reused by its next tile; a tile sort's bulk
    // copy writes it through the async proxy, after the blend's generic
    // accesses (each thread's ordered by its proxy fence, all by the barrier).
    if constexpr (Smem::kSort) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    sync();
  }
}

// term::downsample (src/term.rs:74-99) for factors that do not divide the tile.
__global__ void k_downsample(FrameParams fp, const uint8_t* __restrict__ full, uint8_t* __restrict__ out) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= fp.out_w || y >= fp.out_h) return;
  const uint32_t f = fp.downsample;
  uint32_t acc[3] = {0u, 0u, 0u};
  for (uint32_t sy = 0; sy < f; sy++) {
    const uint8_t* row = full + ((size_t)(y * f + sy) * fp.w + x * f) * 3;
    for (uint32_t sx = 0; sx < f; sx++) {
      acc[0] += row[3 * sx];
      acc[1] += row[3 * sx + 1];
      acc[2] += row[3 * sx + 2];
    }
  }
  const uint32_t nn = f * f;
  uint8_t* o = out + ((size_t)y * fp.out_w + x) * 3;
  o[0] = (uint8_t)(acc[0] / nn);
  o[1] = (uint8_t)(acc[1] / nn);
  o[2] = (uint8_t)(acc[2] / nn);
}

}  // namespace

bool blend_sorts_tiles(const BlendConfig& c) { return c.tile_w == 16 && c.tile_h == 16 && c.threads == 512; }
bool blend_writes_host_rows(const BlendConfig& c, bool exact) { return !exact && blend_sorts_tiles(c); }

bool blend_config_supported(const BlendConfig& c) {
  const bool shape = (c.tile_w == 8 && c.tile_h == 8) || (c.tile_w == 16 && c.tile_h == 16) ||
                     (c.tile_w == 32 && c.tile_h == 16);
  return shape && (c.threads == 128 || c.threads == 256 || c.threads == 512);
}

namespace {

template <bool EXACT, int TW, int TH, int NT, bool ROWS, bool COUNT = false>
cudaError_t launch_blend_t(const ViewTask* table, uint32_t n_views, uint32_t n_tiles, uint64_t* pairs,
                           const uint2* ranges, const uint32_t* order, DevState* st, int num_sms,
                           cudaStream_t stream) {
  using S = BlendShape<TW, TH, NT>;
  const auto kernel = k_blend<EXACT, TW, TH, NT, ROWS, COUNT>;
  const int smem = (int)(S::NG * sizeof(GroupSmem<TW, TH, NT>));
  // Resident CTAs per SM, looked up once per instantiation.
  static std::atomic<int> occ{0};
  int o = occ.load(std::memory_order_relaxed);
  if (o == 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kernel, NT, smem);
    if (e != cudaSuccess) return e;
    if (o < 1) o = 1;
    occ.store(o, std::memory_order_relaxed);
  }
  const uint64_t want = ((uint64_t)n_tiles + S::NG - 1) / S::NG;
  const uint32_t grid = (uint32_t)std::min<uint64_t>(want, (uint64_t)num_sms * (uint64_t)o);
  kernel<<<grid, NT, smem, stream>>>(table, n_views, n_tiles, pairs, ranges, order, st);
  return cudaGetLastError();
}

template <bool EXACT>
cudaError_t launch_blend_e(const ViewTask* table, uint32_t n_views, uint32_t n_tiles, uint64_t* pairs,
                           const uint2* ranges, const uint32_t* order, const BlendConfig& c, DevState* st,
                           int num_sms, cudaStream_t s, bool rows, bool count) {
  // The row-word variant for mapped host frames and the evaluation-counting
  // variant exist for the default blend (16x16 tiles, 512 threads); other
  // shapes write mapped frames byte by byte, which is as correct, and do not
  // count.
#define SPLAT_BLEND(TW, TH, NT)                                                                        \
  if (c.tile_w == TW && c.tile_h == TH && c.threads == NT) {                                           \
    if constexpr (!EXACT && TW == 16 && TH == 16 && NT == 512) {                                       \
      if (count) return launch_blend_t<EXACT, TW, TH, NT, false, true>(table, n_views, n_tiles, pairs, \
                                                                       ranges, order, st, num_sms, s); \
      if (rows) return launch_blend_t<EXACT, TW, TH, NT, true>(table, n_views, n_tiles, pairs, ranges, \
                                                               order, st, num_sms, s);                 \
    }                                                                                                  \
    return launch_blend_t<EXACT, TW, TH, NT, false>(table, n_views, n_tiles, pairs, ranges, order, st, \
                                                    num_sms, s);                                       \
  }
  SPLAT_BLEND(16, 16, 256)
  SPLAT_BLEND(16, 16, 128)
  SPLAT_BLEND(16, 16, 512)
  SPLAT_BLEND(8, 8, 128)
  SPLAT_BLEND(8, 8, 256)
  SPLAT_BLEND(8, 8, 512)
  SPLAT_BLEND(32, 16, 128)
  SPLAT_BLEND(32, 16, 256)
  SPLAT_BLEND(32, 16, 512)
#undef SPLAT_BLEND
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_blend(const ViewTask* table, uint32_t n_views, uint32_t n_tiles, uint64_t* pairs,
                         const uint2* ranges, const uint32_t* order, bool exact, const BlendConfig& cfg, DevState* st,
                         int num_sms, cudaStream_t stream, uint32_t* launches, bool host_rows, bool count) {
  if (n_tiles == 0) return cudaSuccess;
  const cudaError_t e =
      exact ? launch_blend_e<true>(table, n_views, n_tiles, pairs, ranges, order, cfg, st, num_sms, stream, host_rows,
                                   count)
            : launch_blend_e<false>(table, n_views, n_tiles, pairs, ranges, order, cfg, st, num_sms, stream,
                                    host_rows, count);
  if (e == cudaSuccess) *launches += 1;
  return e;
}

cudaError_t launch_downsample(const FrameParams& fp, const uint8_t* full, uint8_t* out, cudaStream_t stream,
                              uint32_t* launches) {
  if (fp.out_w == 0 || fp.out_h == 0) return cudaSuccess;
  dim3 grid((fp.out_w + 127) / 128, fp.out_h);
  k_downsample<<<grid, 128, 0, stream>>>(fp, full, out);
  *launches += 1;
  return cudaGetLastError();
}

}  // namespace splat
