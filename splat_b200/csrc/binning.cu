// Kernel (b): device-wide exclusive scan of the per-splat pair counts with
// warp shuffles and a decoupled look-back, fused with the pair emission.
//
// The scan runs over the visible splats in depth order (the first `visible`
// words of the depth sort's output: depth bits << 32 | splat index, ties in
// splat-index order). Each visible splat duplicates into one pair per tile of
// its pixel bbox, row-major (ty, then tx) as the reference's `emit` does
// (src/render/cpu.rs:251-277); a pair is the 64-bit word tile << 32 | splat.
// Pairs are therefore laid out in (depth, splat index) order, and the stable
// tile sort that follows yields the reference's per-tile blending order:
// by depth, ties by scene index (src/render/naive.rs:306-308,
// src/render/cpu.rs:396-414). The reference's sort key of a pair,
// tile << 32 | depth bits, is recovered exactly from the pair's tile and its
// splat's depth bits.
//
// A CTA scans 1024 splats (4 rounds of 32 per warp, their gathers in flight
// together). A lane expands its own splat when it has at most 32 pairs; a
// larger splat is expanded by its whole warp, so one large splat does not
// serialise its warp. Pairs are staged in shared memory at their offset in
// the CTA's contiguous output range and then written out coalesced, and the
// tile sort's digit histograms are counted from the staged pairs (pairs past
// the staging buffer go straight to global memory and are counted there).
#include "common.cuh"
#include "lookback.cuh"

namespace splat {
namespace {

constexpr int kWarps = kScanThreads / 32;
constexpr int kRounds = 4;
constexpr int kEmitPart = kScanThreads * kRounds;

constexpr uint32_t kStage = 4096;  // staged pairs per CTA (32 KB)

__device__ __forceinline__ void count_digits(uint32_t (*hist)[256], uint32_t tile, int digits) {
  for (int d = 0; d < digits; d++) atomicAdd(&hist[d][(tile >> (8 * d)) & 255u], 1u);
}

__global__ void __launch_bounds__(kScanThreads) k_emit(uint32_t tiles_x, int tile_digits,
                                                       const BinInfo* __restrict__ bin, unsigned long long* desc,
                                                       const uint64_t* dw0, const uint64_t* dw1,
                                                       uint64_t* __restrict__ pairs, uint64_t cap, DevState* st) {
  __shared__ uint32_t s_part;
  __shared__ uint32_t s_warp[kWarps];
  __shared__ unsigned long long s_base;
  __shared__ uint32_t s_total;
  __shared__ uint32_t s_hist[kMaxPasses][256];
  __shared__ uint64_t s_stage[kStage];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t V = *(const volatile unsigned long long*)&st->visible;
  const uint64_t nparts = (V + kEmitPart - 1) / kEmitPart;
  if (tid == 0) s_part = atomicAdd(&st->emit_ticket, 1u);
  for (int t = tid; t < kMaxPasses * 256; t += kScanThreads) (&s_hist[0][0])[t] = 0u;
  __syncthreads();
  const uint32_t part = s_part;
  if (part >= nparts) return;  // uniform across the block
  const uint64_t* __restrict__ dsorted = st->depth.final_sel ? dw1 : dw0;
  const uint64_t wbase = (uint64_t)part * kEmitPart + (uint64_t)warp * (32 * kRounds);
  uint32_t idx[kRounds], cnt[kRounds], lo[kRounds], hi[kRounds], incl[kRounds];
#pragma unroll
  for (int r = 0; r < kRounds; r++) {
    const uint64_t q = wbase + (uint64_t)r * 32 + lane;
    idx[r] = q < V ? (uint32_t)dsorted[q] : 0xFFFFFFFFu;
  }
#pragma unroll
  for (int r = 0; r < kRounds; r++) {
    cnt[r] = 0u;
    lo[r] = hi[r] = 0u;
    if (idx[r] != 0xFFFFFFFFu) {
      const BinInfo b = bin[idx[r]];
      cnt[r] = b.count;
      lo[r] = b.rect_lo;
      hi[r] = b.rect_hi;
    }
  }
  uint32_t warp_total = 0;
#pragma unroll
  for (int r = 0; r < kRounds; r++) {
    uint32_t x = cnt[r];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    incl[r] = x;
    warp_total += __shfl_sync(0xffffffffu, x, 31);
  }
  if (lane == 0) s_warp[warp] = warp_total;
  __syncthreads();
  if (warp == 0) {
    const uint32_t c = lane < kWarps ? s_warp[lane] : 0u;
    uint32_t w = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, w, 31);
    if (lane < kWarps) s_warp[lane] = w - c;  // exclusive per warp
    const unsigned long long base = lookback_exclusive(desc, part, total, st, kErrEmitTimeout);
    if (lane == 0) {
      s_base = base;
      s_total = total;
      if ((uint64_t)part == nparts - 1) st->total_pairs = base + total;
    }
  }
  __syncthreads();

  // Expansion into the staging buffer: local offset = offset in this CTA's range.
  const uint64_t cta_base = s_base;
  auto put = [&](uint32_t local, uint32_t tile, uint32_t splat) {
    const uint64_t word = ((uint64_t)tile << 32) | splat;
    if (local < kStage) {
      s_stage[local] = word;
    } else if (cta_base + local < cap) {
      pairs[cta_base + local] = word;
      count_digits(s_hist, tile, tile_digits);
    }
  };
  constexpr uint32_t kLanePairs = 32;
  uint32_t round_local = s_warp[warp];
#pragma unroll
  for (int r = 0; r < kRounds; r++) {
    const uint32_t x = incl[r];
    const uint32_t round_total = __shfl_sync(0xffffffffu, x, 31);
    const uint32_t my_excl = x - cnt[r];
    if (cnt[r] <= kLanePairs) {
      const uint32_t tx0 = lo[r] & 0xFFFFu, ty0 = lo[r] >> 16, tx1 = hi[r] & 0xFFFFu;
      uint32_t local = round_local + my_excl;
      uint32_t tx = tx0, ty = ty0;
      for (uint32_t p = 0; p < cnt[r]; p++, local++) {
        put(local, ty * tiles_x + tx, idx[r]);
        if (++tx == tx1) {
          tx = tx0;
          ty++;
        }
      }
    }
    uint32_t big = __ballot_sync(0xffffffffu, cnt[r] > kLanePairs);
    while (big) {
      const int L = __ffs(big) - 1;
      big &= big - 1u;
      const uint32_t b_lo = __shfl_sync(0xffffffffu, lo[r], L), b_hi = __shfl_sync(0xffffffffu, hi[r], L);
      const uint32_t b_cnt = __shfl_sync(0xffffffffu, cnt[r], L), b_ex = __shfl_sync(0xffffffffu, my_excl, L);
      const uint32_t b_id = __shfl_sync(0xffffffffu, idx[r], L);
      const uint32_t btx0 = b_lo & 0xFFFFu, bty0 = b_lo >> 16, wdt = (b_hi & 0xFFFFu) - btx0;
      for (uint32_t k = lane; k < b_cnt; k += 32) {
        const uint32_t row = k / wdt;
        put(round_local + b_ex + k, (bty0 + row) * tiles_x + btx0 + (k - row * wdt), b_id);
      }
    }
    round_local += round_total;
  }
  __syncthreads();
  // Coalesced write-out of the staged pairs, counting their tile digits.
  const uint32_t staged = min(s_total, kStage);
  for (uint32_t l = tid; l < staged; l += kScanThreads) {
    if (cta_base + l < cap) {
      const uint64_t word = s_stage[l];
      pairs[cta_base + l] = word;
      count_digits(s_hist, (uint32_t)(word >> 32), tile_digits);
    }
  }
  __syncthreads();
  for (int t = tid; t < tile_digits * 256; t += kScanThreads) {
    const uint32_t v = (&s_hist[0][0])[t];
    if (v) atomicAdd(&(&st->tile.hist[0][0])[t], v);
  }
}

}  // namespace

cudaError_t launch_emit(const FrameParams& fp, int tile_digits, const BinInfo* bin, uint64_t n,
                        unsigned long long* scan_desc, uint64_t* const* depth_words, uint64_t* pairs, uint64_t cap,
                        DevState* st, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  // Enough CTAs for every splat being visible; CTAs past the visible count return at once.
  const unsigned grid = (unsigned)((n + kEmitPart - 1) / kEmitPart);
  k_emit<<<grid, kScanThreads, 0, stream>>>(fp.tiles_x, tile_digits, bin, scan_desc, depth_words[0], depth_words[1],
                                            pairs, cap, st);
  return cudaGetLastError();
}

}  // namespace splat
