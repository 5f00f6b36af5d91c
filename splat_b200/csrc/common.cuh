// Shared definitions of the sm_100a rasterizer kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/splat_cuda.h"

namespace splat {

// src/render/mod.rs:23-33
constexpr float kDilation = 0.3f;
constexpr float kAlphaMin = 1.0f / 255.0f;
constexpr float kAlphaMax = 0.99f;
constexpr float kTMin = 1e-4f;
// FP16 storage: a 2D covariance determinant below this is recomputed in FP64.
constexpr float kFp64DetBelow = 1e-6f;
constexpr uint32_t kMaxDim = 16384;
// src/render/cpu.rs:34: the reference's 16x16 tiles (the default tile shape
// here; 8x8 and 32x16 are the other shapes the tuner may choose).
constexpr uint32_t kTile = 16;
// Tile starts of consecutive views in a batch are aligned to this many tiles,
// and the tile scan works on chunks of kScanChunk tiles.
constexpr uint32_t kTileAlign = 32;
constexpr uint32_t kScanChunk = 2048;

// Marks a culled splat in BinInfo::rect_lo.
constexpr uint32_t kCulled = 0xFFFFFFFFu;

// Largest pair capacity (pair offsets and tile ranges are 32-bit).
constexpr uint64_t kMaxPairs = (1ull << 30) - 1;

// Per-frame constants (ProjectCtx, src/render/mod.rs:155-196) plus grid sizes.
struct FrameParams {
  float rot[9];  // row-major: rows are right, down, forward (View::rotation)
  float eye[3];
  float focal, cx, cy, width, height, near_plane, lim_x, lim_y;
  float bg[3];
  uint32_t w, h;
  uint32_t tile_w, tile_h;      // tile shape (powers of two)
  uint32_t tile_sx, tile_sy;    // log2 of the tile shape
  uint32_t tiles_x, tiles_y;
  uint32_t downsample;      // 1 = none
  uint32_t out_w, out_h;    // floor(w/f), floor(h/f)
  // The window of the w x h frame that is rendered: rows [win_y0, win_y0 +
  // win_rows), columns [win_x0, win_x0 + win_cols) (the whole frame: 0, h,
  // 0, w); the tile grid then covers tile rows [win_ty0, win_ty0 + tiles_y)
  // and tile columns [win_tx0, win_tx0 + tiles_x). Frame row y is output row
  // y - out_y0 (row windows into a buffer of their own rows: out_y0 =
  // win_y0; windows drawn into the whole frame: 0). A window that does not
  // start at column 0 or end at the frame's edge is aligned to tiles.
  uint32_t win_y0, win_rows, win_ty0, out_y0;
  uint32_t win_x0, win_cols, win_tx0;
  uint32_t flags;  // kFrame* bits
};
// The frame's pair buffer keeps every tile's pairs in depth order after the
// blend (for inspection; otherwise tiles the blend sorts itself may be left
// in bucket order, their order held in shared memory only).
constexpr uint32_t kFrameKeepSortedPairs = 1u;
// The frame pairs each splat with every tile of its pixel bbox, as the
// reference does (src/render/cpu.rs:251-277). Otherwise a tile whose pixel
// centres all lie outside the splat's alpha = 1/255 ellipse (its blend
// contribution there is zero) gets no pair; see window_rect.
constexpr uint32_t kFrameBboxPairs = 2u;

// Device-resident scene, FP32 storage (layout chosen for coalesced loads).
struct SceneDev {
  // FP32 storage
  const float4* pos_op;   // x, y, z, opacity
  const float4* cov_a;    // xx, xy, xz, yy
  const float4* cov_b;    // yz, zz, k = sqrt(2 ln(op / ALPHA_MIN)), 0
  const float* color;     // 3 planes of n: r, g, b (base colour)
  const float* sh;        // rest*3 planes of n: plane (coef*3 + channel)
  // FP16 storage (128 bytes per splat)
  const float4* pos_k;    // x, y, z, k
  const uint4* geom16;    // 8 halves: scale x, y, z, rotation x, y, z, w, opacity
  const uint16_t* sh16;   // (rest+1)*3 planes of n halves: base colour, then the rest
  uint64_t n;
  uint32_t sh_degree;
  uint32_t fp16;
  // Learned colour (FP16 storage only): per-splat latents, 16 halves each
  // (two uint4), and the MLP's fp16 parameters (mlp.cuh layout).
  const uint4* lat16;
  const uint16_t* mlp16;
  uint32_t learned;
  // The order in which the binning visits the splats: a static permutation
  // of the scene that follows a 3D Morton curve through the splat positions,
  // so that the splats one CTA bins lie close together on screen and its
  // pairs fall into few tiles, in runs (null: scene order).
  const uint32_t* order;
  // Fault injection (tests of the timeout path): when nonzero, each CTA of
  // the learned-colour projection also waits, at its first tensor-core wait,
  // for a completion that never arrives, giving up after this many
  // microseconds, as a lost completion would make it do.
  uint32_t lost_wait_us;
};

// A projected splat as the blend reads it: 48 bytes, three float4.
//  r0 = x, y, -0.5*conic_a, -conic_b
//  r1 = -0.5*conic_c, opacity, red, green
//  r2 = blue, bbox x0 | x1 << 16, bbox y0 | y1 << 16, depth
struct __align__(16) Record {
  float4 r0, r1, r2;
};

// Per-splat binning input written by the projection: the tile rectangle of
// its pixel bbox clipped to the rendered window and counted from the
// window's first tile row and column (tx0 | ty0 << 16, tx1 | ty1 << 16),
// depth bits, and which tiles of the rectangle it pairs with: for a
// rectangle of at most kMaskTiles tiles, `cm` has bit k set for its k-th
// tile in row-major order (its pair count is the number of bits); for a
// larger one, `cm` is its pair count and the splat's BinSkip says which
// tiles are kept. rect_lo == kCulled marks a culled splat; a visible splat
// whose bbox holds no pixel has no pairs (empty rectangle, cm = 0).
struct __align__(16) BinInfo {
  uint32_t rect_lo, rect_hi, depth_bits, cm;
};
// The kept tiles of a rectangle of more than kMaskTiles tiles, written only
// for those: per row r < kSkipRows, the tiles at the row's two ends that the
// splat does not reach (byte r: left | right << 4, each at most 15;
// kSkipEmpty: none of the row), row r pairing with tiles [tx0 + left,
// tx1 - right); all zero: the whole rectangle.
struct __align__(16) BinSkip {
  uint32_t skip[4];
};
constexpr uint32_t kSkipRows = 16;
constexpr uint32_t kSkipEmpty = 0xFFu;
constexpr uint32_t kMaskTiles = 32;

__host__ __device__ __forceinline__ uint32_t low_bits(uint32_t n) { return n >= 32u ? ~0u : (1u << n) - 1u; }

__device__ __forceinline__ uint32_t rect_area(const BinInfo& b) {
  return ((b.rect_hi & 0xFFFFu) - (b.rect_lo & 0xFFFFu)) * ((b.rect_hi >> 16) - (b.rect_lo >> 16));
}
// The splat's pair count (0 for a culled splat).
__device__ __forceinline__ uint32_t bin_count(const BinInfo& b) {
  if (b.rect_lo == kCulled) return 0u;
  return rect_area(b) <= kMaskTiles ? (uint32_t)__popc(b.cm) : b.cm;
}

__device__ __forceinline__ bool has_skips(const BinSkip& k) {
  return (k.skip[0] | k.skip[1] | k.skip[2] | k.skip[3]) != 0u;
}

// Row r's tile span [a, e) of the rectangle [tx0, tx1) (empty: a == e).
__device__ __forceinline__ void row_span(const BinSkip& k, uint32_t r, uint32_t tx0, uint32_t tx1, uint32_t& a,
                                         uint32_t& e) {
  // The word by selects, not by a dynamic index (which would put k in local memory).
  const uint32_t word = r < 8u ? (r < 4u ? k.skip[0] : k.skip[1]) : (r < 12u ? k.skip[2] : k.skip[3]);
  const uint32_t sk = r < kSkipRows ? (word >> (8u * (r & 3u))) & 255u : 0u;
  a = sk == kSkipEmpty ? tx1 : tx0 + (sk & 15u);
  e = sk == kSkipEmpty ? tx1 : tx1 - (sk >> 4);
}

// Hardware approximations as inline PTX: the same instruction, hence the
// same result, in every translation unit whatever its contraction flags.
__device__ __forceinline__ float lg2_hw(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_hw(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sqrt_hw(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// For each row of a splat's tile rectangle, the tiles at its two ends whose
// pixel centres all lie outside the splat's alpha = 1/255 ellipse, from the
// splat's record r (centre, -conic/2 terms, opacity): with the conic (a, b,
// c) and K = 2 ln(255 opacity), alpha >= 1/255 exactly where
// Q = a dx^2 + 2 b dx dy + c dy^2 <= K (the same K that sizes the pixel bbox,
// k^2). In the band of a tile row's pixel-centre rows [Y0, Y1] the ellipse
// reaches x from min L(dy) to max U(dy), U/L(dy) = (-b dy +/- sqrt(a K -
// det dy^2)) / a (det = ac - b^2), extremes at the ellipse's leftmost and
// rightmost points (dy = +/- b sqrt(K c / det) / c) clamped into the band;
// a tile column whose pixel-centre x range misses [x + L, x + U] holds no
// pixel the splat reaches. K is widened by 0.2 % + 0.002 and the x range by
// 0.01 px (the hardware square roots and reciprocals err by a few units in
// the last place), so no tile a pixel needs is dropped; the blend's images do
// not change (a dropped tile's pixels would all have failed the alpha test).
//
// The spans are those of the whole bbox rectangle [ftx0, ftx1) x [fty0,
// fty1) (its rows past kSkipRows, and every row of a 1 x 1 rectangle, whole;
// at most 15 tiles dropped at either end), intersected with the window's
// part [wtx0, wtx1) x [wty0, wty1): a frame drawn in windows has exactly the
// pairs of the frame drawn at once. Every operation rounds explicitly, so
// the projection and the records' binning input (different translation
// units and contraction flags) compute the same skips. Sets b.cm (the mask,
// or the pair count) and, for a rectangle of more than kMaskTiles tiles, k.
__device__ __forceinline__ void ellipse_skips(const FrameParams& fp, const Record& r, uint32_t ftx0, uint32_t ftx1,
                                              uint32_t fty0, uint32_t fty1, uint32_t wtx0, uint32_t wtx1,
                                              uint32_t wty0, uint32_t wty1, BinInfo& b, BinSkip& k) {
  const uint32_t wcols = wtx1 - wtx0, wrows = wty1 - wty0, all = wcols * wrows;
  const bool masked = all <= kMaskTiles;
  b.cm = masked ? low_bits(all) : all;  // whole, unless narrowed below
  if (ftx1 - ftx0 == 1u && fty1 - fty0 == 1u) return;  // the centre's own tile
  const float a = __fmul_rn(-2.0f, r.r0.z), bb = -r.r0.w, c = __fmul_rn(-2.0f, r.r1.x);
  // det = ac - b^2 with b^2's rounding error carried (two-product): no
  // cancellation for thin ellipses.
  const float p = __fmul_rn(bb, bb), pe = __fmaf_rn(bb, bb, -p);
  const float det = __fsub_rn(__fmaf_rn(a, c, -p), pe);
  // K = 2 ln 2 (log2 op + log2 255), widened.
  const float K0 = __fmul_rn(1.38629436f, __fadd_rn(lg2_hw(r.r1.y), 7.99435344f));
  const float K = __fadd_rn(__fmul_rn(K0, 1.002f), 0.002f);
  if (!(det > 0.0f && a > 0.0f && c > 0.0f && K > 0.0f)) return;
  const float inv_det = rcp_hw(det), inv_a = rcp_hw(a);
  const float aK = __fmul_rn(a, K);
  const float ey = sqrt_hw(__fmul_rn(aK, inv_det));                          // vertical half-extent
  const float xm = sqrt_hw(__fmul_rn(__fmul_rn(c, K), inv_det));             // horizontal half-extent
  const float dyr = __fmul_rn(__fmul_rn(-bb, xm), rcp_hw(c));                // dy of the rightmost point
  const float tw = (float)fp.tile_w, th = (float)fp.tile_h, inv_tw = 1.0f / (float)fp.tile_w;  // exact: powers of 2
  const uint32_t dy0 = wty0 - fty0;  // bbox rows above the window
  const uint32_t rows = min(wrows, kSkipRows);
  uint32_t count = (wrows - rows) * wcols;
  uint32_t mask = masked ? low_bits(all) & ~low_bits(rows * wcols) : 0u;  // rows past kSkipRows: whole
  for (uint32_t q = 0; q < rows; q++) {
    const uint32_t rb = q + dy0;  // the row of the whole rectangle
    uint32_t sa = ftx0, se = ftx1;  // its span, whole past kSkipRows
    if (rb < kSkipRows) {
      const float ty = (float)(fty0 + rb);
      const float band0 = __fsub_rn(__fadd_rn(__fmul_rn(ty, th), 0.5f), r.r0.y);
      const float band1 = __fadd_rn(band0, th - 1.0f);
      if (band1 >= -ey && band0 <= ey) {
        const float lo = fmaxf(band0, -ey), hi = fminf(band1, ey);
        const float yr = fminf(fmaxf(dyr, lo), hi), yl = fminf(fmaxf(-dyr, lo), hi);
        const float sr = sqrt_hw(fmaxf(__fsub_rn(aK, __fmul_rn(det, __fmul_rn(yr, yr))), 0.0f));
        const float sl = sqrt_hw(fmaxf(__fsub_rn(aK, __fmul_rn(det, __fmul_rn(yl, yl))), 0.0f));
        const float U = __fmul_rn(__fadd_rn(__fmul_rn(-bb, yr), sr), inv_a);
        const float L = __fmul_rn(__fsub_rn(__fmul_rn(-bb, yl), sl), inv_a);
        // Tile columns whose pixel centres [tx tw + 0.5, tx tw + tw - 0.5] meet [x + L, x + U].
        const float xl = __fsub_rn(__fadd_rn(r.r0.x, L), 0.01f), xu = __fadd_rn(__fadd_rn(r.r0.x, U), 0.01f);
        const float ta = ceilf(__fmul_rn(__fsub_rn(xl, tw - 0.5f), inv_tw));
        const float tb = floorf(__fmul_rn(__fsub_rn(xu, 0.5f), inv_tw));
        const uint32_t left = (uint32_t)fminf(fmaxf(__fsub_rn(ta, (float)ftx0), 0.0f), 15.0f);
        uint32_t right = (uint32_t)fminf(fmaxf(__fsub_rn((float)(ftx1 - 1u), tb), 0.0f), 15.0f);
        if (left == 15u && right == 15u) right = 14u;  // 15 | 15 << 4 is kSkipEmpty
        sa = ftx0 + left;
        se = max(sa, ftx1 - min(right, ftx1 - ftx0));
      } else {
        sa = se = ftx1;  // the ellipse misses the band
      }
    }
    // The span inside the window's columns.
    const uint32_t ca = min(max(sa, wtx0), wtx1), ce = max(min(se, wtx1), ca);
    count += ce - ca;
    if (masked) {
      mask |= low_bits(ce - ca) << (q * wcols + (ca - wtx0));
      continue;
    }
    const uint32_t byte = ce == ca ? kSkipEmpty : (ca - wtx0) | ((wtx1 - ce) << 4);
    const uint32_t sh = 8u * (q & 3u);
    if (q < 4u)
      k.skip[0] |= byte << sh;
    else if (q < 8u)
      k.skip[1] |= byte << sh;
    else if (q < 12u)
      k.skip[2] |= byte << sh;
    else
      k.skip[3] |= byte << sh;
  }
  b.cm = masked ? mask : count;
}

// The tile rectangle of a splat whose pixel bbox (pixel_bbox,
// src/render/cpu.rs:96-102) is [bx0, x1) x [by0, y1): its tile rows and
// columns clipped to the frame's rendered window and counted from the
// window's first tile row and column (the whole frame: unchanged). A bbox
// that holds no pixel of the window gives the empty rectangle (no pairs).
// Unless the frame asks for the bbox pairs (kFrameBboxPairs), the rows' end
// tiles the splat's ellipse does not reach are skipped (ellipse_skips, from
// the splat's record r). Returns whether k is needed (a rectangle of more
// than kMaskTiles tiles: the caller stores it).
__device__ __forceinline__ bool window_rect(const FrameParams& fp, uint32_t bx0, uint32_t x1, uint32_t by0,
                                            uint32_t y1, const Record& r, BinInfo& b, BinSkip& k) {
  const uint32_t ftx0 = bx0 >> fp.tile_sx, ftx1 = (x1 + fp.tile_w - 1) >> fp.tile_sx;
  const uint32_t fty0 = by0 >> fp.tile_sy, fty1 = (y1 + fp.tile_h - 1) >> fp.tile_sy;
  const uint32_t wty0 = max(fty0, fp.win_ty0), wty1 = min(fty1, fp.win_ty0 + fp.tiles_y);
  const uint32_t wtx0 = max(ftx0, fp.win_tx0), wtx1 = min(ftx1, fp.win_tx0 + fp.tiles_x);
  k.skip[0] = k.skip[1] = k.skip[2] = k.skip[3] = 0u;
  if (bx0 < x1 && by0 < y1 && wty0 < wty1 && wtx0 < wtx1) {
    const uint32_t tx0 = wtx0 - fp.win_tx0, ty0 = wty0 - fp.win_ty0;
    const uint32_t tx1 = wtx1 - fp.win_tx0, ty1 = wty1 - fp.win_ty0;
    b.rect_lo = tx0 | (ty0 << 16);
    b.rect_hi = tx1 | (ty1 << 16);
    const uint32_t area = (tx1 - tx0) * (ty1 - ty0);
    if (fp.flags & kFrameBboxPairs)
      b.cm = area <= kMaskTiles ? low_bits(area) : area;
    else
      ellipse_skips(fp, r, ftx0, ftx1, fty0, fty1, wtx0, wtx1, wty0, wty1, b, k);
    return area > kMaskTiles;
  }
  b.rect_lo = 0u;  // visible, but its bbox holds no pixel of the window: no pairs
  b.rect_hi = 0u;
  b.cm = 0u;
  return false;
}

// Per-tile depth sort sizes: tiles up to kWarpSortCap pairs are sorted by one
// warp, up to kMidSortCap by one CTA in shared memory, longer ones in chunks.
constexpr uint32_t kWarpSortCap = 512;
constexpr uint32_t kMidSortCap = 4096;

// Tiles by pair count, heaviest class first: > 4096 (the long sort), 2049 -
// 4096, 1025 - 2048, 513 - 1024 (the mid sort), 257 - 512, 1 - 256, empty.
// k_tile_ranges appends every tile to its class's list (kTileClasses lists
// of n_tiles entries each); the blend and the mid sort take their tiles in
// class order, so no long tile starts last.
constexpr int kTileClasses = 7;
__host__ __device__ constexpr uint32_t tile_class(uint32_t len) {
  return len > kMidSortCap ? 0u
         : len > 2048u     ? 1u
         : len > 1024u     ? 2u
         : len > kWarpSortCap ? 3u
         : len > 256u      ? 4u
         : len > 0u        ? 5u
                           : 6u;
}

// Frame state in device memory, cleared at the start of every frame (or
// batch). Followed in the same allocation by the per-view counters and the
// tile-scan chunk sums, cleared with it (FrameCounters).
struct DevState {
  unsigned long long visible;      // splats that survived culling (all views)
  unsigned long long total_pairs;  // (splat, tile) pairs, may exceed the capacity
  unsigned int error;
  unsigned int fp64_conics;        // splats whose 2D conic was recomputed in FP64
  unsigned int blend_next;         // the persistent blend's next work item
  unsigned int mid_next;           // the mid sort's next work item
  unsigned int cls[kTileClasses];  // tiles per class (tile_class)
  unsigned int pad;
  unsigned long long evals;        // pixel/splat evaluations of the blend (when counted)
};

// The cleared counters of a frame or batch of n_views views over n_chunks
// tile-scan chunks: DevState, then visible splats per view, pairs per view,
// pair totals per scan chunk (all unsigned long long).
struct FrameCounters {
  DevState* st;
  unsigned long long* view_visible;
  unsigned long long* view_pairs;
  unsigned long long* chunk_sum;
};
inline size_t frame_counters_bytes(uint32_t n_views, uint32_t n_chunks) {
  return sizeof(DevState) + sizeof(unsigned long long) * (2 * (size_t)n_views + n_chunks);
}
inline FrameCounters frame_counters_at(void* base, uint32_t n_views) {
  FrameCounters c;
  c.st = static_cast<DevState*>(base);
  c.view_visible = reinterpret_cast<unsigned long long*>(c.st + 1);
  c.view_pairs = c.view_visible + n_views;
  c.chunk_sum = c.view_pairs + n_views;
  return c;
}

// One view of a frame or of a batch, as every kernel of the pipeline reads
// it from the view table (device memory). Each launch covers all views: a
// CTA finds its view by binary search over the views' first CTA (or first
// tile) for that launch.
struct ViewTask {
  FrameParams fp;
  SceneDev s;
  Record* rec;          // n records of this view
  BinInfo* bin;         // n tile rectangles of this view
  BinSkip* skip;        // n kept-tile lists (for rectangles of more than kMaskTiles tiles)
  uint32_t* counts;     // rows x tiles count matrix
  uint8_t* out;         // device frame, out_w * out_h * 3 bytes
  uint8_t* full;        // full-resolution scratch for a downsample factor
                        // that does not divide the tile shape (or null)
  uint32_t rows;        // CTAs of the count and scatter launches for this view
  uint32_t tile0;       // first global tile (a multiple of kTileAlign)
  uint32_t proj_cta0;   // first CTA of the view in the projection launch
  uint32_t bin_cta0;    // ... in the count and scatter launches
  uint32_t col_cta0;    // ... in the column-scan launch
  uint32_t pad[3];      // pad[0], learned-colour batch table: the view's batch index
};

// The view whose `field` (a first-CTA or first-tile member) is the largest
// one <= x; views are in increasing order of every such field.
__device__ __forceinline__ uint32_t find_view(const ViewTask* __restrict__ table, uint32_t n_views, uint32_t x,
                                              size_t field_offset) {
  uint32_t lo = 0, hi = n_views;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    const uint32_t v =
        __ldg(reinterpret_cast<const uint32_t*>(reinterpret_cast<const char*>(table + mid) + field_offset));
    if (v <= x)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Blend configuration: tile shape and threads per CTA.
struct BlendConfig {
  uint32_t tile_w, tile_h, threads;
};
bool blend_config_supported(const BlendConfig& c);
// Whether the blend of this configuration sorts the tiles of at most
// kMidSortCap pairs itself (then the binning launches no small/mid sorts).
bool blend_sorts_tiles(const BlendConfig& c);
// Whether the blend of this configuration has the row-word variant for
// frames in mapped host memory (whole 4-byte words of tile rows; the other
// variants store bytes, which over the host link are an order of magnitude
// slower than drawing into device memory and copying the frame).
bool blend_writes_host_rows(const BlendConfig& c, bool exact);

// Launchers (each returns the cudaGetLastError of its launches and adds the
// number of kernels it launched to *launches).
// (a) projection of one view (`t` by value; CTA 0 also stores it as table[0]),
// or of every view of the table (batch).
cudaError_t launch_project(const ViewTask& t, ViewTask* table, float* dbg_proj, float* dbg_color,
                           const FrameCounters& fc, cudaStream_t stream, uint32_t* launches);
// (Each CTA of the batch projection takes kProjectSplatsPerCta splats of one view.)
constexpr uint32_t kProjectSplatsPerCta = 128;
cudaError_t launch_project_batch(const ViewTask* table, uint32_t n_views, uint32_t total_ctas,
                                 const FrameCounters& fc, cudaStream_t stream, uint32_t* launches);
// The learned-colour views of a batch: `table` holds n_views copies of them
// with proj_cta0 = first tile of 128 splats in this launch and pad[0] = the
// view's index in the batch.
cudaError_t launch_project_learned_batch(ViewTask* table, uint32_t n_views, uint64_t total_tiles,
                                         const FrameCounters& fc, cudaStream_t stream, uint32_t* launches);
// Count-matrix rows (CTAs of the count and scatter launches) for n splats:
// about per_cta splats each, at most two CTAs per SM. A single view takes
// 1024 per CTA (small scenes and windows of records still fill the GPU); the
// views of a batch, which fill it together, 4096.
uint32_t bin_rows(uint64_t n, int num_sms, uint32_t per_cta = 4096);
// (b) binning into per-tile buckets and (c) the per-tile depth sorts, over
// all views of the table: count matrix, tile totals, ranges, mid/long lists.
struct BinLaunch {
  uint32_t n_views;
  uint32_t bin_ctas;      // total CTAs of the count and scatter launches
  uint32_t col_ctas;      // total CTAs of the column-scan launch
  uint32_t n_tiles;       // global tiles (views' tile ranges, padded)
  uint32_t max_tiles;     // largest view's tile count
  bool counts_zeroed;     // counts must be zeroed when a row does not fit shared memory
  uint32_t* counts_all;   // all count matrices (for the zeroing)
  size_t counts_bytes;
};
// tile_sorts: launch the sorts of tiles of at most kMidSortCap pairs (false
// when the blend sorts them itself, blend_sorts_tiles).
cudaError_t launch_binning(const ViewTask* table, const BinLaunch& bl, uint32_t* totals, uint2* ranges,
                           uint32_t* order, uint64_t* pairs, uint64_t* pairs_alt,
                           uint64_t cap, const FrameCounters& fc, int num_sms, size_t max_smem, cudaStream_t stream,
                           uint32_t* launches, bool tile_sorts = true);
// (d) blend + downsample over the depth-sorted buckets of every view.
// host_rows: the views' frames are mapped pinned host memory (see k_blend).
cudaError_t launch_blend(const ViewTask* table, uint32_t n_views, uint32_t n_tiles, uint64_t* pairs,
                         const uint2* ranges, const uint32_t* order, bool exact, const BlendConfig& cfg, DevState* st,
                         int num_sms, cudaStream_t stream, uint32_t* launches, bool host_rows = false,
                         bool count = false);
// Splat-sharded frames (shard.cu). Row windows of a frame, [bound[k],
// bound[k + 1]) for k < n, at most kMaxShardWindows of them.
constexpr uint32_t kMaxShardWindows = 64;
struct ShardWindows {
  uint32_t n;
  uint32_t bound[kMaxShardWindows + 1];
};
// Device scratch of the record selection of n splats over w.n windows.
size_t shard_scratch_bytes(uint64_t n, uint32_t windows);
// The sender side: counts, for every window, the projected splats (rec and
// bin of a whole-frame projection of n splats) whose pixel bbox meets its
// rows, into totals[0 .. w.n) (device memory), keeping in `scratch` the
// offsets the scatter uses.
cudaError_t launch_shard_count(const Record* rec, const BinInfo* bin, uint64_t n, const ShardWindows& w,
                               void* scratch, unsigned long long* totals, cudaStream_t stream, uint32_t* launches);
// ... then writes each such splat's record to every window its rows meet:
// window k's records from send + (totals of the windows before k) on, in
// scene order; positions at or past cap are not written.
cudaError_t launch_shard_scatter(const Record* rec, const BinInfo* bin, uint64_t n, const ShardWindows& w,
                                 const void* scratch, const unsigned long long* totals, Record* send, uint64_t cap,
                                 cudaStream_t stream, uint32_t* launches);
// The receiver side: the binning input of t.s.n records (t.rec, received in
// scene order) for the view's window, in place of the projection; CTA 0
// also stores t as table[0].
cudaError_t launch_records_bin(const ViewTask& t, ViewTask* table, const FrameCounters& fc, cudaStream_t stream,
                               uint32_t* launches);

// Half-block terminal cells (SPLAT_CELLS_*) of a frame of width w.
cudaError_t launch_cells(const uint8_t* frame, uint32_t w, uint32_t cols, uint32_t rows, uint32_t mode, uint8_t* cells,
                         cudaStream_t stream, uint32_t* launches);
// term::downsample of one view's full-resolution scratch frame.
cudaError_t launch_downsample(const FrameParams& fp, const uint8_t* full, uint8_t* out, cudaStream_t stream,
                              uint32_t* launches);

}  // namespace splat
