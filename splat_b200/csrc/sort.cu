// Kernel (c): onesweep LSD radix sort plus the tile-range kernel.
//
// The reference sorts each tile's bucket stably by depth (radix::sort_hi32,
// src/render/radix.rs:13-57, after a counting sort by tile, cpu.rs:149-199)
// and breaks depth ties by scene index (fix_ties, cpu.rs:396-414). Here two
// stable LSD sorts of 64-bit words produce the same order: the visible splats
// by depth (words depth bits << 32 | splat, built in splat-index order, so
// ties keep index order), then, after emission in that order, the pairs by
// tile (words tile << 32 | splat). Only the upper 32 bits are digits: 8-bit
// digits, one histogram kernel counts every digit of a sort up front, and a
// digit shared by all words is skipped (as sort_hi32 does, radix.rs:389-393).
// Each remaining digit is one onesweep pass: a CTA ranks its 4096-word
// partition stably with warp match-any, publishes its per-digit counts,
// resolves its global offsets by a decoupled look-back over the earlier
// partitions (bounded spin) and scatters.
// Tile ranges ([begin, end) per tile) come from neighbour compares over the
// sorted pairs, as the reference's `ranges_main` does (tiles.wgsl:83-101).
#include "common.cuh"

namespace splat {
namespace {

constexpr int kWarps = kSortThreads / 32;
constexpr uint32_t kLbAgg = 1u << 30;
constexpr uint32_t kLbInc = 2u << 30;
constexpr uint32_t kLbMask = (1u << 30) - 1;

__device__ __forceinline__ uint64_t sort_count(const unsigned long long* count, uint64_t cap) {
  const unsigned long long t = *(const volatile unsigned long long*)count;
  return t < cap ? t : cap;
}

// Histograms of `digits` 8-bit digits (from bit 32 + 8 * first_digit) of the
// words, with warp-aggregated shared-memory atomics (peers found by match-any).
__global__ void __launch_bounds__(256) k_hist(const uint64_t* __restrict__ words, const unsigned long long* count,
                                              uint64_t cap, int first_digit, int digits, SortState* ss) {
  __shared__ uint32_t h[kMaxPasses][256];
  for (int t = threadIdx.x; t < kMaxPasses * 256; t += blockDim.x) (&h[0][0])[t] = 0u;
  __syncthreads();
  const uint64_t n = sort_count(count, cap);
  const int lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  // Whole warps iterate together so match-any sees every lane.
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
    const uint64_t i = base + lane;
    const bool valid = i < n;
    const uint32_t hi = valid ? (uint32_t)(words[i] >> 32) : 0u;
    for (int d = 0; d < digits; d++) {
      const uint32_t dig = valid ? (hi >> (8 * (first_digit + d))) & 255u : 256u;
      const uint32_t peers = __match_any_sync(0xffffffffu, dig);
      if (valid && lane == 31 - __clz(peers)) atomicAdd(&h[d][dig], (uint32_t)__popc(peers));
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < digits * 256; t += blockDim.x) {
    const uint32_t v = (&h[0][0])[t];
    if (v) atomicAdd(&(&ss->hist[0][0])[t], v);
  }
}

// One CTA: exclusive scans of the digit histograms and the pass schedule.
__global__ void __launch_bounds__(256) k_hist_scan(SortState* ss, const unsigned long long* count, uint64_t cap,
                                                   int digits) {
  __shared__ uint32_t s_warp[8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t n = sort_count(count, cap);
  int parity = 0;
  for (int d = 0; d < digits; d++) {
    const uint32_t v = ss->hist[d][tid];
    const int trivial = __syncthreads_or((uint64_t)v == n);
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t base = 0;
    for (int w = 0; w < warp; w++) base += s_warp[w];
    ss->hist[d][tid] = base + x - v;
    __syncthreads();
    if (tid == 0) ss->pass_src[d] = trivial ? -1 : parity;
    if (!trivial) parity ^= 1;
  }
  if (tid == 0) {
    for (int d = digits; d < kMaxPasses; d++) ss->pass_src[d] = -1;
    ss->final_sel = parity;
  }
}

__global__ void __launch_bounds__(kSortThreads, 3) k_onesweep(SortState* ss, const unsigned long long* count,
                                                              uint64_t cap, int pass, int shift, uint64_t* w0,
                                                              uint64_t* w1, uint32_t* lb, DevState* st) {
  __shared__ uint32_t s_whist[kWarps][256];
  __shared__ uint32_t s_gbase[256];
  __shared__ uint32_t s_part;
  const int src = ss->pass_src[pass];
  if (src < 0) return;
  const uint64_t* __restrict__ in = src ? w1 : w0;
  uint64_t* __restrict__ out = src ? w0 : w1;
  const uint64_t n = sort_count(count, cap);
  const uint32_t nparts = (uint32_t)((n + kSortPart - 1) / kSortPart);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;

  for (;;) {
    if (tid == 0) s_part = atomicAdd(&ss->ticket[pass], 1u);
#pragma unroll
    for (int w = 0; w < kWarps; w++) s_whist[w][tid] = 0u;
    __syncthreads();
    const uint32_t part = s_part;
    if (part >= nparts) break;

    // This warp's 16 x 32 words (warp-striped, coalesced), ranked stably per
    // digit: item (j, lane) is word base + 32 j + lane.
    const uint64_t base = (uint64_t)part * kSortPart + (uint64_t)warp * (kSortItems * 32);
    uint64_t key[kSortItems];
    uint32_t dr[kSortItems];  // rank << 8 | digit, or 0xFFFFFFFF past the end
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
      const uint64_t idx = base + (uint64_t)j * 32 + lane;
      const bool valid = idx < n;
      key[j] = valid ? in[idx] : 0ull;
      dr[j] = valid ? (uint32_t)((key[j] >> shift) & 255u) : 0xFFFFFFFFu;
    }
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
      const bool valid = dr[j] != 0xFFFFFFFFu;
      const uint32_t dig = valid ? dr[j] : 256u;
      const uint32_t peers = __match_any_sync(0xffffffffu, dig);
      const int leader = 31 - __clz(peers);
      uint32_t cnt = 0;
      if (valid) cnt = s_whist[warp][dig];
      __syncwarp();
      if (valid) {
        dr[j] = ((cnt + __popc(peers & lt_mask)) << 8) | dig;
        if (lane == leader) s_whist[warp][dig] = cnt + __popc(peers);
      }
      __syncwarp();
    }
    __syncthreads();

    // Thread `tid` owns digit tid: warp offsets, block count, look-back.
    uint32_t running = 0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) {
      const uint32_t t = s_whist[w][tid];
      s_whist[w][tid] = running;
      running += t;
    }
    uint32_t* my = lb + (uint64_t)part * 256 + tid;
    uint32_t prefix = 0;
    if (part == 0) {
      *(volatile uint32_t*)my = kLbInc | running;
    } else {
      *(volatile uint32_t*)my = kLbAgg | running;
      long long j = (long long)part - 1;
      while (j >= 0) {
        const uint32_t* q = lb + (uint64_t)j * 256 + tid;
        uint32_t v = *(const volatile uint32_t*)q;
        uint32_t spins = 0;
        while ((v >> 30) == 0u) {
          // Give up at the bound, or at once after another wait gave up.
          if (++spins > kSpinLimit || ((spins & 1023u) == 0u && (*(volatile uint32_t*)&st->error & kErrSortTimeout))) {
            atomicOr(&st->error, kErrSortTimeout);
            v = kLbInc;
            break;
          }
          __nanosleep(20);
          v = *(const volatile uint32_t*)q;
        }
        prefix += v & kLbMask;
        if ((v >> 30) == 2u) break;
        j--;
      }
      *(volatile uint32_t*)my = kLbInc | (prefix + running);
    }
    s_gbase[tid] = ss->hist[pass][tid] + prefix;
    __syncthreads();

#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
      if (dr[j] != 0xFFFFFFFFu) {
        const uint32_t dig = dr[j] & 255u;
        const uint64_t pos = (uint64_t)s_gbase[dig] + s_whist[warp][dig] + (dr[j] >> 8);
        if (pos < n)
          out[pos] = key[j];
        else
          atomicOr(&st->error, kErrSortRange);
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_ranges(uint64_t cap, const uint64_t* p0, const uint64_t* p1,
                                                uint2* __restrict__ ranges, uint32_t tiles, const DevState* st) {
  const uint64_t* __restrict__ pairs = st->tile.final_sel ? p1 : p0;
  const uint64_t n = sort_count(&st->total_pairs, cap);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t t = (uint32_t)(pairs[i] >> 32);
    if (t >= tiles) continue;
    if (i == 0 || (uint32_t)(pairs[i - 1] >> 32) != t) ranges[t].x = (uint32_t)i;
    if (i + 1 == n || (uint32_t)(pairs[i + 1] >> 32) != t) ranges[t].y = (uint32_t)(i + 1);
  }
}

}  // namespace

cudaError_t launch_sort(SortState* ss, const unsigned long long* count, uint64_t cap, int first_digit, int digits,
                        uint64_t* words0, uint64_t* words1, uint32_t* lookback, uint64_t lookback_parts,
                        DevState* st, int num_sms, cudaStream_t stream) {
  if (digits <= 0) return cudaSuccess;
  k_hist<<<num_sms * 4, 256, 0, stream>>>(words0, count, cap, first_digit, digits, ss);
  k_hist_scan<<<1, 256, 0, stream>>>(ss, count, cap, digits);
  for (int d = 0; d < digits; d++) {
    k_onesweep<<<num_sms * 3, kSortThreads, 0, stream>>>(ss, count, cap, d, 32 + 8 * (first_digit + d), words0,
                                                        words1, lookback + (uint64_t)d * lookback_parts * 256, st);
  }
  return cudaGetLastError();
}

cudaError_t launch_ranges(uint64_t cap, uint64_t* const* pairs, uint2* ranges, uint32_t tiles, DevState* st,
                          int num_sms, cudaStream_t stream) {
  k_ranges<<<num_sms * 4, 256, 0, stream>>>(cap, pairs[0], pairs[1], ranges, tiles, st);
  return cudaGetLastError();
}

}  // namespace splat
