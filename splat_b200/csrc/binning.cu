// Kernel (b): binning of (splat, tile) pairs into per-tile buckets, and the
// sort of tiles too long to sort inside the blend CTA.
//
// Every visible splat duplicates into one pair per tile of its pixel bbox
// (src/render/cpu.rs:251-277) that its alpha = 1/255 ellipse reaches (every
// bbox tile with kFrameBboxPairs; the projection marks the tiles in the
// splat's BinInfo / BinSkip). The reference buckets pairs with a counting
// sort by tile (cpu.rs:149-199): per-group tile histograms, a prefix over
// (tile, group), then a scatter. The same scheme here, with CTAs as groups:
//
//  k_bin_count    each CTA counts the pairs of its slice of splats per tile
//                 in shared memory and writes its row of the count matrix;
//  k_bin_colscan  per tile, an exclusive scan of the counts down the rows;
//                 tile totals, and their sums per chunk of kScanChunk tiles;
//  k_tile_ranges  per chunk, an exclusive scan of the tile totals offset by
//                 the preceding chunks: the tile ranges ([begin, end); [0, 0)
//                 for an empty tile) and the tiles' class lists (tile_class:
//                 the long sort's, the mid sort's and the blend's order);
//  k_bin_scatter  each CTA writes its pairs at its row's offsets, positions
//                 handed out by shared-memory atomics.
//
// Every launch covers all views of the view table: the tiles of the views
// are concatenated (each view's first tile aligned to kTileAlign) into one
// global tile space, so the ranges, the pair buffer and the sorts are shared
// by the views; a CTA of the count, column-scan and scatter launches finds
// its view by binary search over the views' first CTA.
//
// A pair is the word depth bits << 32 | splat index. Order inside a bucket is
// whatever the atomics produced; the per-tile depth sort that follows (in the
// blend CTA, or k_sort_long for long tiles) restores the reference's order.
#include <algorithm>
#include <atomic>
#include <cstddef>

#include "common.cuh"
#include "tilesort.cuh"

namespace splat {
namespace {

constexpr int kBinThreads = 512;

// Calls fw(tile, splat, depth bits) for every pair of the splats at
// positions [s0, s1) of the binning order (SceneDev::order; null: scene
// order). A splat whose rectangle holds at most kMaskTiles tiles is expanded
// by its own lane from its bit mask; a larger one by the whole warp, row by
// row of its spans (row_span).
template <class FW>
__device__ __forceinline__ void for_each_pair(const BinInfo* __restrict__ bin, const BinSkip* __restrict__ skip,
                                              const uint32_t* __restrict__ order, uint64_t s0, uint64_t s1,
                                              uint32_t tiles_x, FW&& fw) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr uint64_t kStride = (uint64_t)kBinThreads;
  // The lane's splat of the warp's next group of 32 is loaded while the
  // current group's pairs are expanded.
  const BinInfo culled{kCulled, 0u, 0u, 0u};
  auto splat_at = [&](uint64_t k) -> uint32_t { return order ? __ldg(order + k) : (uint32_t)k; };
  uint64_t wb = s0 + (uint64_t)warp * 32;
  uint32_t ni = wb + lane < s1 ? splat_at(wb + lane) : 0u;
  BinInfo nb = wb + lane < s1 ? bin[ni] : culled;
  for (; wb < s1; wb += kStride) {
    const uint64_t k = wb + lane;
    const BinInfo b = nb;
    const uint32_t i = ni;
    if (k + kStride < s1) {
      ni = splat_at(k + kStride);
      nb = bin[ni];
    } else {
      nb = culled;
    }
    const uint32_t tx0 = b.rect_lo & 0xFFFFu, ty0 = b.rect_lo >> 16, tx1 = b.rect_hi & 0xFFFFu;
    const uint32_t wdt0 = tx1 - tx0, rows = (b.rect_hi >> 16) - ty0;
    const bool small = b.rect_lo != kCulled && wdt0 * rows <= kMaskTiles;
    const uint32_t cnt = b.rect_lo == kCulled ? 0u : (small ? (uint32_t)__popc(b.cm) : b.cm);
    if (small) {
      // The rectangle's kept tiles, one bit each (row-major): the common
      // case, one code path whether tiles are skipped or not. kb / wdt0 for
      // kb < 32 as a multiply and shift: inv = floor(65536 / wdt0) + 1 from
      // the hardware reciprocal (exact for powers of two; otherwise
      // 65536 / wdt0 lies at least 1/32 from an integer, far beyond its error).
      const uint32_t inv = (uint32_t)(rcp_hw((float)max(wdt0, 1u)) * 65536.0f) + 1u;
      uint32_t m = b.cm;
      while (m) {
        const uint32_t kb = (uint32_t)__ffs(m) - 1u;
        m &= m - 1u;
        const uint32_t row = (kb * inv) >> 16;
        fw((ty0 + row) * tiles_x + tx0 + (kb - row * wdt0), i, b.depth_bits);
      }
    }
    // Larger rectangles (at most 32 pairs or not) go through the whole warp,
    // so that no lane runs a long per-row loop while the others wait.
    uint32_t big = __ballot_sync(0xffffffffu, !small && cnt > 0);
    while (big) {
      const int L = __ffs(big) - 1;
      big &= big - 1u;
      const uint32_t b_lo = __shfl_sync(0xffffffffu, b.rect_lo, L), b_hi = __shfl_sync(0xffffffffu, b.rect_hi, L);
      const uint32_t b_d = __shfl_sync(0xffffffffu, b.depth_bits, L), b_i = __shfl_sync(0xffffffffu, i, L);
      const uint32_t b_cnt = __shfl_sync(0xffffffffu, cnt, L);
      const BinSkip w = skip[b_i];  // the same words for every lane
      const uint32_t btx0 = b_lo & 0xFFFFu, bty0 = b_lo >> 16;
      const uint32_t btx1 = b_hi & 0xFFFFu, brows = (b_hi >> 16) - bty0, wdt = btx1 - btx0;
      if (!has_skips(w)) {
        for (uint32_t q = lane; q < b_cnt; q += 32) {
          const uint32_t row = q / wdt;
          fw((bty0 + row) * tiles_x + btx0 + (q - row * wdt), b_i, b_d);
        }
        continue;
      }
      // Lane r < kSkipRows holds row r's span and the pairs up to its end;
      // rows past kSkipRows are whole.
      uint32_t ra = 0, re = 0;
      if ((uint32_t)lane < min(brows, kSkipRows)) row_span(w, (uint32_t)lane, btx0, btx1, ra, re);
      const uint32_t wr = re - ra;
      uint32_t incl = wr;
#pragma unroll
      for (int o = 1; o < (int)kSkipRows; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      const uint32_t head = __shfl_sync(0xffffffffu, incl, kSkipRows - 1);
      // The warp's lanes take 32 consecutive pairs at a time: a pair among
      // the first rows finds its row by binary search over those lanes.
      for (uint32_t q0 = 0; q0 < b_cnt; q0 += 32) {
        const uint32_t q = q0 + (uint32_t)lane;
        uint32_t lo = 0;
#pragma unroll
        for (uint32_t step = kSkipRows / 2; step >= 1; step >>= 1) {
          if (__shfl_sync(0xffffffffu, incl, lo + step - 1) <= q) lo += step;
        }
        const uint32_t a_r = __shfl_sync(0xffffffffu, ra, lo), ex = __shfl_sync(0xffffffffu, incl - wr, lo);
        uint32_t row, col;
        if (q < head) {
          row = lo;
          col = a_r + (q - ex);
        } else {
          const uint32_t q2 = q - head;
          row = kSkipRows + q2 / wdt;
          col = btx0 + q2 % wdt;
        }
        if (q < b_cnt) fw((bty0 + row) * tiles_x + col, b_i, b_d);
      }
    }
  }
}

// The per-view fields the count and scatter CTAs need.
struct BinView {
  const BinInfo* bin;
  const BinSkip* skip;
  const uint32_t* order;  // the binning order (null: scene order)
  uint32_t* row;  // this CTA's row of the view's count matrix
  uint64_t s0, s1;
  uint32_t tiles_x, tiles, tile0;
};

__device__ __forceinline__ BinView bin_view(const ViewTask* __restrict__ table, uint32_t n_views) {
  const uint32_t v = find_view(table, n_views, blockIdx.x, offsetof(ViewTask, bin_cta0));
  const ViewTask* t = table + v;
  BinView b;
  b.bin = t->bin;
  b.skip = t->skip;
  b.order = t->s.order;
  b.tiles_x = t->fp.tiles_x;
  b.tiles = t->fp.tiles_x * t->fp.tiles_y;
  b.tile0 = t->tile0;
  const uint32_t r = blockIdx.x - t->bin_cta0, rows = t->rows;
  const uint64_t n = t->s.n, per_cta = n ? (n + rows - 1) / rows : 1;
  b.row = t->counts + (uint64_t)r * b.tiles;
  b.s0 = min(n, (uint64_t)r * per_cta);
  b.s1 = min(n, b.s0 + per_cta);
  return b;
}

// SMEM: the CTA's row lives in shared memory (tiles * 4 bytes); otherwise the
// CTA counts straight into its global row (zeroed beforehand).
template <bool SMEM>
__global__ void __launch_bounds__(kBinThreads) k_bin_count(const ViewTask* __restrict__ table, uint32_t n_views) {
  extern __shared__ uint32_t s_row[];
  const BinView b = bin_view(table, n_views);
  if (SMEM) {
    for (uint32_t t = threadIdx.x; t < b.tiles; t += kBinThreads) s_row[t] = 0u;
    __syncthreads();
  }
  uint32_t* const cnt = SMEM ? s_row : b.row;
  for_each_pair(b.bin, b.skip, b.order, b.s0, b.s1, b.tiles_x, [&](uint32_t t, uint32_t, uint32_t) { atomicAdd(&cnt[t], 1u); });
  if (SMEM) {
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < b.tiles; t += kBinThreads) b.row[t] = s_row[t];
  }
}

// Per tile: exclusive scan of the counts down the rows; the tile's total.
// A CTA takes 32 tiles of one view; its 8 warps each scan a contiguous eighth
// of the rows (a warp reads 32 adjacent tiles of a row: coalesced), then the
// segment sums are combined and the rows rewritten with exclusive offsets.
// The CTA's pair total goes to its scan chunk and to its view.
__global__ void __launch_bounds__(256) k_bin_colscan(const ViewTask* __restrict__ table, uint32_t n_views,
                                                     uint32_t* __restrict__ totals, FrameCounters fc) {
  __shared__ uint32_t s_seg[8][32];
  const uint32_t v = find_view(table, n_views, blockIdx.x, offsetof(ViewTask, col_cta0));
  const ViewTask* tv = table + v;
  uint32_t* counts = tv->counts;
  const uint32_t rows = tv->rows, tiles = tv->fp.tiles_x * tv->fp.tiles_y;
  const uint32_t first = (blockIdx.x - tv->col_cta0) * 32, tile0 = tv->tile0;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t t = first + lane;
  const uint32_t per = (rows + 7) / 8;
  const uint32_t r0 = min(rows, warp * per), r1 = min(rows, r0 + per);
  // Rows are independent loads: unrolled so that several are in flight.
  uint32_t sum = 0;
  if (t < tiles) {
#pragma unroll 8
    for (uint32_t r = r0; r < r1; r++) sum += counts[(uint64_t)r * tiles + t];
  }
  s_seg[warp][lane] = sum;
  __syncthreads();
  uint32_t run = 0, total = 0;
  for (uint32_t w = 0; w < 8; w++) {
    if (w < warp) run += s_seg[w][lane];
    total += s_seg[w][lane];
  }
  if (t < tiles) {
#pragma unroll 8
    for (uint32_t r = r0; r < r1; r++) {
      const uint32_t c = counts[(uint64_t)r * tiles + t];
      counts[(uint64_t)r * tiles + t] = run;
      run += c;
    }
    if (warp == 0) totals[tile0 + t] = total;
  }
  if (warp == 0) {
    unsigned long long cta = t < tiles ? total : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cta += __shfl_xor_sync(0xffffffffu, cta, o);
    if (lane == 0 && cta) {
      // tile0 and first are multiples of 32, so the CTA's tiles share a chunk.
      atomicAdd(&fc.chunk_sum[(tile0 + first) / kScanChunk], cta);
      atomicAdd(&fc.view_pairs[v], cta);
    }
  }
}

// One CTA per chunk of kScanChunk global tiles: exclusive scan of the tile
// totals offset by the sum of the preceding chunks -> ranges, the lists of
// tiles sorted by a whole CTA (mid) or in chunks (long), and (last chunk)
// the total pair count.
constexpr int kRangeThreads = 512;
static_assert(kScanChunk == kRangeThreads * 4, "four tiles per thread");

__global__ void __launch_bounds__(kRangeThreads) k_tile_ranges(const uint32_t* __restrict__ totals, uint32_t n_tiles,
                                                               uint64_t cap, uint2* __restrict__ ranges,
                                                               uint32_t* __restrict__ order, FrameCounters fc) {
  __shared__ unsigned long long s_warp[kRangeThreads / 32];
  __shared__ unsigned long long s_base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t chunk = blockIdx.x;
  // Sum of the preceding chunks.
  unsigned long long pre = 0;
  for (uint32_t c = tid; c < chunk; c += kRangeThreads) pre += fc.chunk_sum[c];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pre += __shfl_xor_sync(0xffffffffu, pre, o);
  if (lane == 0) s_warp[warp] = pre;
  __syncthreads();
  if (tid == 0) {
    unsigned long long b = 0;
    for (int w = 0; w < kRangeThreads / 32; w++) b += s_warp[w];
    s_base = b;
  }
  __syncthreads();
  const unsigned long long base = s_base;
  uint32_t c[4];
  unsigned long long sum = 0;
  const uint32_t t0 = chunk * kScanChunk + tid * 4;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    c[k] = t0 + k < n_tiles ? totals[t0 + k] : 0u;
    sum += c[k];
  }
  unsigned long long x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();  // s_warp is reused
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  unsigned long long before = 0, chunk_total = 0;
  for (int w = 0; w < kRangeThreads / 32; w++) {
    if (w < warp) before += s_warp[w];
    chunk_total += s_warp[w];
  }
  unsigned long long start = base + before + x - sum;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t t = t0 + k;
    uint32_t cls = kTileClasses;
    if (t < n_tiles) {
      // Ranges are clamped to the pair capacity: past it the frame is
      // incomplete and rendered again with larger buffers, and nothing
      // reads beyond the buffers meanwhile.
      const uint32_t s = (uint32_t)min(start, (unsigned long long)cap);
      const uint32_t e = (uint32_t)min(start + c[k], (unsigned long long)cap);
      ranges[t] = e > s ? make_uint2(s, e) : make_uint2(0u, 0u);
      cls = tile_class(e > s ? e - s : 0u);
    }
    // The tile joins its class's list: one atomic per class in the warp.
    const uint32_t same = __match_any_sync(0xffffffffu, cls);
    const int leader = __ffs(same) - 1;
    uint32_t at = 0;
    if (lane == leader && cls < kTileClasses) at = atomicAdd(&fc.st->cls[cls], (uint32_t)__popc(same));
    at = __shfl_sync(0xffffffffu, at, leader) + __popc(same & ((1u << lane) - 1u));
    if (cls < kTileClasses) order[(size_t)cls * n_tiles + at] = t;
    start += c[k];
  }
  if (chunk == gridDim.x - 1 && tid == 0) fc.st->total_pairs = base + chunk_total;
}

template <bool SMEM>
__global__ void __launch_bounds__(kBinThreads) k_bin_scatter(const ViewTask* __restrict__ table, uint32_t n_views,
                                                             const uint2* __restrict__ ranges,
                                                             uint64_t* __restrict__ pairs, uint64_t cap) {
  extern __shared__ uint32_t s_row[];
  const BinView b = bin_view(table, n_views);
  const uint2* vr = ranges + b.tile0;
  if (SMEM) {
#pragma unroll 4
    for (uint32_t t = threadIdx.x; t < b.tiles; t += kBinThreads) s_row[t] = vr[t].x + b.row[t];
    __syncthreads();
  }
  for_each_pair(b.bin, b.skip, b.order, b.s0, b.s1, b.tiles_x, [&](uint32_t t, uint32_t i, uint32_t depth_bits) {
    const uint64_t pos = SMEM ? atomicAdd(&s_row[t], 1u) : (uint64_t)vr[t].x + atomicAdd(&b.row[t], 1u);
    if (pos < cap) pairs[pos] = ((uint64_t)depth_bits << 32) | i;
  });
}

// Tiles of at most kWarpSortCap pairs (classes 4 and 5, the heavier class
// first): one warp per tile, persistent warps striding over the two lists.
__global__ void __launch_bounds__(256, 3) k_sort_small(const uint2* __restrict__ ranges,
                                                    const uint32_t* __restrict__ order, uint32_t n_tiles,
                                                    uint64_t* __restrict__ pairs, const DevState* st) {
  __shared__ uint64_t s_scratch[8][kWarpSortCap];
  __shared__ uint32_t s_counts[8][256];
  const uint32_t warp = threadIdx.x >> 5;
  const uint32_t n4 = st->cls[4], n5 = st->cls[5];
  for (uint32_t li = blockIdx.x * 8 + warp; li < n4 + n5; li += gridDim.x * 8) {
    const uint32_t tile = li < n4 ? order[4 * (size_t)n_tiles + li] : order[5 * (size_t)n_tiles + (li - n4)];
    const uint2 r = ranges[tile];
    const uint32_t n = r.y - r.x;
    if (n >= 2) warp_sort_tile(pairs + r.x, n, s_scratch[warp], s_counts[warp]);
  }
}

// Tiles of (kWarpSortCap, kMidSortCap] pairs: one CTA per tile, in shared
// memory (smem_count_sort).
struct MidSmem {
  uint64_t words[kMidSortCap];
  uint32_t hist[kCountBuckets / 2];
  uint16_t slot[kMidSortCap];
  CountSortSmem t;
};

// Tiles of classes 1-3, heaviest class first, taken one at a time from a
// shared counter (the tiles differ in length up to 8x).
__global__ void __launch_bounds__(kTileThreads) k_sort_mid(const uint2* __restrict__ ranges,
                                                           const uint32_t* __restrict__ order, uint32_t n_tiles,
                                                           uint64_t* __restrict__ pairs, DevState* st) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  MidSmem& sm = *reinterpret_cast<MidSmem*>(s_raw);
  __shared__ uint32_t s_tile;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t n1 = st->cls[1], n2 = st->cls[2], n3 = st->cls[3];
  for (;;) {
    if (tid == 0) {
      const uint32_t li = atomicAdd(&st->mid_next, 1u);
      s_tile = li < n1             ? order[(size_t)n_tiles + li]
               : li < n1 + n2      ? order[2 * (size_t)n_tiles + (li - n1)]
               : li < n1 + n2 + n3 ? order[3 * (size_t)n_tiles + (li - n1 - n2)]
                                   : 0xFFFFFFFFu;
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile == 0xFFFFFFFFu) break;
    const uint2 r = ranges[tile];
    const uint32_t n = r.y - r.x;
    uint32_t mn = 0xFFFFFFFFu, mx = 0u;
    for (uint32_t e = tid; e < n; e += kTileThreads) {
      const uint64_t w = pairs[r.x + e];
      sm.words[e] = w;
      mn = min(mn, (uint32_t)(w >> 32));
      mx = max(mx, (uint32_t)(w >> 32));
    }
    for (uint32_t b = tid; b < kCountBuckets / 2; b += kTileThreads) sm.hist[b] = 0u;
    // block min / max of the depth bits (positive floats order like their bits)
#pragma unroll
    for (int s2 = 16; s2 > 0; s2 >>= 1) {
      mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, s2));
      mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, s2));
    }
    if (lane == 0) {
      sm.t.red[0][warp] = mn;
      sm.t.red[1][warp] = mx;
    }
    __syncthreads();
#pragma unroll
    for (int w = 0; w < kTileWarps; w++) {
      mn = min(mn, sm.t.red[0][w]);
      mx = max(mx, sm.t.red[1][w]);
    }
    smem_count_sort(sm.words, n, mn, mx, sm.hist, sm.slot, sm.t);
    for (uint32_t e = tid; e < n; e += kTileThreads) pairs[r.x + e] = sm.words[sm.slot[e]];
    __syncthreads();
  }
}

// Sorts the pairs of each tile longer than kMidSortCap in global memory (the
// pair buffer, the second pair buffer as ping-pong), one CTA per tile
// (long_tile_sort: chunked LSD passes, ties ordered by splat index).
__global__ void __launch_bounds__(kTileThreads) k_sort_long(const uint2* __restrict__ ranges,
                                                            const uint32_t* __restrict__ long_list,
                                                            uint64_t* __restrict__ w0, uint64_t* __restrict__ w1,
                                                            uint64_t cap, const DevState* st) {  // class 0
  __shared__ ChunkSortSmem sm;
  const uint32_t nlong = st->cls[0];
  for (uint32_t li = blockIdx.x; li < nlong; li += gridDim.x) {
    const uint2 r = ranges[long_list[li]];  // within the capacity (k_tile_ranges)
    long_tile_sort(w0 + r.x, w1 + r.x, r.y - r.x, sm);
  }
}

}  // namespace

uint32_t bin_rows(uint64_t n, int num_sms, uint32_t per_cta) {
  // About per_cta splats per CTA, at most two CTAs per SM.
  const uint64_t r = (n + per_cta - 1) / per_cta;
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(r, 2ull * (uint64_t)num_sms));
}

cudaError_t launch_binning(const ViewTask* table, const BinLaunch& bl, uint32_t* totals, uint2* ranges,
                           uint32_t* order, uint64_t* pairs, uint64_t* pairs_alt,
                           uint64_t cap, const FrameCounters& fc, int num_sms, size_t max_smem, cudaStream_t stream,
                           uint32_t* launches, bool tile_sorts) {
  if (bl.n_tiles == 0) return cudaSuccess;
  const size_t smem = (size_t)bl.max_tiles * sizeof(uint32_t);
  const bool use_smem = smem <= max_smem;
  cudaError_t e = cudaSuccess;
  // Shared-memory limits are raised to the device's opt-in maximum outside
  // stream capture (the first frame or batch always runs uncaptured).
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if ((e = cudaStreamIsCapturing(stream, &cs))) return e;
  if (cs == cudaStreamCaptureStatusNone) {
    const int big = (int)max_smem;
    if ((e = cudaFuncSetAttribute(k_bin_count<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(k_bin_scatter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(k_sort_mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MidSmem))))
      return e;
  }
  if (use_smem) {
    k_bin_count<true><<<bl.bin_ctas, kBinThreads, smem, stream>>>(table, bl.n_views);
  } else {
    if ((e = cudaMemsetAsync(bl.counts_all, 0, bl.counts_bytes, stream))) return e;
    k_bin_count<false><<<bl.bin_ctas, kBinThreads, 0, stream>>>(table, bl.n_views);
  }
  k_bin_colscan<<<bl.col_ctas, 256, 0, stream>>>(table, bl.n_views, totals, fc);
  const uint32_t chunks = (bl.n_tiles + kScanChunk - 1) / kScanChunk;
  k_tile_ranges<<<chunks, kRangeThreads, 0, stream>>>(totals, bl.n_tiles, cap, ranges, order, fc);
  if (use_smem) {
    k_bin_scatter<true><<<bl.bin_ctas, kBinThreads, smem, stream>>>(table, bl.n_views, ranges, pairs, cap);
  } else {
    k_bin_scatter<false><<<bl.bin_ctas, kBinThreads, 0, stream>>>(table, bl.n_views, ranges, pairs, cap);
  }
  // The sorts loop over their tile lists: as many CTAs as fit on the device
  // at once (looked up once).
  static std::atomic<int> occ_small{0}, occ_mid{0}, occ_long{0};
  if (occ_mid.load(std::memory_order_relaxed) == 0 && cs == cudaStreamCaptureStatusNone) {
    int os = 0, om = 0, ol = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&os, k_sort_small, 256, 0))) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&om, k_sort_mid, kTileThreads, sizeof(MidSmem)))) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ol, k_sort_long, kTileThreads, 0))) return e;
    occ_small.store(std::max(os, 1), std::memory_order_relaxed);
    occ_long.store(std::max(ol, 1), std::memory_order_relaxed);
    occ_mid.store(std::max(om, 1), std::memory_order_relaxed);
  }
  const int os = std::max(occ_small.load(std::memory_order_relaxed), 1);
  const int om = std::max(occ_mid.load(std::memory_order_relaxed), 1);
  const int ol = std::max(occ_long.load(std::memory_order_relaxed), 1);
  if (tile_sorts) {
    k_sort_small<<<num_sms * os, 256, 0, stream>>>(ranges, order, bl.n_tiles, pairs, fc.st);
    k_sort_mid<<<num_sms * om, kTileThreads, sizeof(MidSmem), stream>>>(ranges, order, bl.n_tiles, pairs, fc.st);
    *launches += 2;
  }
  k_sort_long<<<num_sms * ol, kTileThreads, 0, stream>>>(ranges, order, pairs, pairs_alt, cap, fc.st);
  *launches += 5;
  return cudaGetLastError();
}

}  // namespace splat
