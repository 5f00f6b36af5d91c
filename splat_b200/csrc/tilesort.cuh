// Per-tile depth sort: the reference's per-tile radix::sort_hi32 followed by
// fix_ties (src/render/cpu.rs:208-210, radix.rs:13-57, cpu.rs:396-414),
// run by one CTA of kTileThreads threads.
//
// A tile's pairs arrive in arbitrary order (they are bucketed with shared-
// memory atomics). Each pair is the word depth bits << 32 | splat index; the
// key is the depth bits (a positive float's bit pattern orders like the
// float). A stable LSD radix sort over the 8-bit digits that are not shared by
// every key of the tile orders the pairs by depth; runs of equal depth are
// then ordered by splat index, which makes the result independent of the
// bucketing order: exactly the reference's (depth, scene index) order.
//
// Ranking is stable per pass: each warp ranks a contiguous segment of the
// elements 32 at a time (lanes with equal digits found by ballots over the
// digit bits), per-warp digit counts are prefix-summed over the warps, and
// the digit starts come from a block scan of the counts.
#pragma once

#include "common.cuh"

namespace splat {

constexpr int kTileThreads = 256;
constexpr int kTileWarps = kTileThreads / 32;

struct TileSortSmem {
  uint32_t wh[kTileWarps][256];  // per-warp digit counts, then exclusive offsets
  uint32_t dstart[256];          // digit starts in the block
  uint32_t wsum[kTileWarps];
  uint32_t red[2][kTileWarps];
};

// AND and OR of all keys of the tile (bits that vary = and ^ or).
__device__ __forceinline__ void block_and_or(uint32_t a, uint32_t o, TileSortSmem& sm, uint32_t& and_all,
                                             uint32_t& or_all) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    a &= __shfl_xor_sync(0xffffffffu, a, s);
    o |= __shfl_xor_sync(0xffffffffu, o, s);
  }
  if (lane == 0) {
    sm.red[0][warp] = a;
    sm.red[1][warp] = o;
  }
  __syncthreads();
  and_all = 0xFFFFFFFFu;
  or_all = 0u;
#pragma unroll
  for (int w = 0; w < kTileWarps; w++) {
    and_all &= sm.red[0][w];
    or_all |= sm.red[1][w];
  }
  __syncthreads();
}

// Stable ranks of up to 32 * kChunks elements per warp (a contiguous segment
// [seg0, seg1) of key[]), digit at `shift`. Fills sm.wh with per-warp counts,
// returns per-chunk (rank << 8 | digit) in dr[] (0xFFFFFFFF past the end).
template <int kChunks>
__device__ __forceinline__ void warp_rank(const uint32_t* key, uint32_t seg0, uint32_t seg1, int shift,
                                          TileSortSmem& sm, uint32_t (&k)[kChunks], uint32_t (&dr)[kChunks]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int c = 0; c < kChunks; c++) {
    const uint32_t e = seg0 + (uint32_t)c * 32 + lane;
    const bool valid = e < seg1;
    k[c] = valid ? key[e] : 0u;
    const uint32_t dig = (k[c] >> shift) & 255u;
    uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int b = 0; b < 8; b++) {
      const bool bit = (dig >> b) & 1u;
      const uint32_t bal = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? bal : ~bal;
    }
    uint32_t cnt = 0;
    if (valid) cnt = sm.wh[warp][dig];
    __syncwarp();
    dr[c] = 0xFFFFFFFFu;
    if (valid) {
      dr[c] = ((cnt + __popc(peers & lt)) << 8) | dig;
      if (lane == 31 - __clz(peers)) sm.wh[warp][dig] = cnt + __popc(peers);
    }
    __syncwarp();
  }
}

// Thread t owns digit t: exclusive per-warp offsets and the digit start.
__device__ __forceinline__ void digit_offsets(TileSortSmem& sm) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t running = 0;
#pragma unroll
  for (int w = 0; w < kTileWarps; w++) {
    const uint32_t t = sm.wh[w][tid];
    sm.wh[w][tid] = running;
    running += t;
  }
  uint32_t x = running;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm.wsum[warp] = x;
  __syncthreads();
  uint32_t wb = 0;
  for (int w = 0; w < warp; w++) wb += sm.wsum[w];
  sm.dstart[tid] = wb + x - running;
  __syncthreads();
}

__device__ __forceinline__ void clear_counts(TileSortSmem& sm) {
#pragma unroll
  for (int w = 0; w < kTileWarps; w++) sm.wh[w][threadIdx.x] = 0u;
}

// In-shared-memory sort of n <= kCap (key, value) pairs held in key[0]/val[0];
// returns the buffer index (0/1) holding the result.
template <int kCap>
__device__ int smem_sort(uint32_t (*key)[kCap], uint32_t (*val)[kCap], uint32_t n, TileSortSmem& sm) {
  constexpr int kChunks = kCap / (32 * kTileWarps);
  uint32_t a = 0xFFFFFFFFu, o = 0u;
  for (uint32_t e = threadIdx.x; e < n; e += kTileThreads) {
    a &= key[0][e];
    o |= key[0][e];
  }
  uint32_t and_all, or_all;
  block_and_or(a, o, sm, and_all, or_all);
  const uint32_t vary = and_all ^ or_all;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t seg = (n + kTileWarps - 1) / kTileWarps;
  const uint32_t seg0 = min(n, (uint32_t)warp * seg), seg1 = min(n, seg0 + seg);
  int cur = 0;
  for (int d = 0; d < 4; d++) {
    const int shift = 8 * d;
    if (((vary >> shift) & 255u) == 0u) continue;
    clear_counts(sm);
    __syncthreads();
    uint32_t k[kChunks], dr[kChunks];
    warp_rank<kChunks>(key[cur], seg0, seg1, shift, sm, k, dr);
    __syncthreads();
    digit_offsets(sm);
#pragma unroll
    for (int c = 0; c < kChunks; c++) {
      if (dr[c] != 0xFFFFFFFFu) {
        const uint32_t dig = dr[c] & 255u;
        const uint32_t pos = sm.dstart[dig] + sm.wh[warp][dig] + (dr[c] >> 8);
        key[cur ^ 1][pos] = k[c];
        val[cur ^ 1][pos] = val[cur][seg0 + (uint32_t)c * 32 + lane];
      }
    }
    __syncthreads();
    cur ^= 1;
  }
  // fix_ties: within runs of equal depth, order by splat index.
  for (uint32_t e = threadIdx.x + 1; e < n; e += kTileThreads) {
    const uint32_t kk = key[cur][e];
    if (kk == key[cur][e - 1] && (e == 1 || key[cur][e - 2] != kk)) {
      uint32_t r1 = e + 1;
      while (r1 < n && key[cur][r1] == kk) r1++;
      uint32_t* v = val[cur];
      for (uint32_t i = e; i < r1; i++) {  // insertion sort of v[e-1, r1)
        const uint32_t x = v[i];
        uint32_t j = i;
        while (j > e - 1 && v[j - 1] > x) {
          v[j] = v[j - 1];
          j--;
        }
        v[j] = x;
      }
    }
  }
  __syncthreads();
  return cur;
}

// Warp-level sort of one tile's n <= kWarpSortCap words (depth bits << 32 |
// splat index) in place in global memory: the elements live in registers,
// warp-striped (element j*32 + lane), each pass ranks them stably with
// ballots, places them in `scratch` (kWarpSortCap words of shared memory) and
// reads them back striped; fix_ties runs on the final scratch copy.
__device__ __forceinline__ void warp_sort_tile(uint64_t* __restrict__ words, uint32_t n, uint64_t* scratch,
                                               uint32_t* counts) {
  constexpr int kM = kWarpSortCap / 32;
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  uint64_t w[kM];
  uint32_t a = 0xFFFFFFFFu, o = 0u;
#pragma unroll
  for (int j = 0; j < kM; j++) {
    const uint32_t e = (uint32_t)j * 32 + lane;
    w[j] = e < n ? words[e] : ~0ull;
    if (e < n) {
      a &= (uint32_t)(w[j] >> 32);
      o |= (uint32_t)(w[j] >> 32);
    }
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    a &= __shfl_xor_sync(0xffffffffu, a, s);
    o |= __shfl_xor_sync(0xffffffffu, o, s);
  }
  const uint32_t vary = a ^ o;
  const int m = (int)((n + 31) / 32);
  for (int d = 0; d < 4; d++) {
    const int shift = 32 + 8 * d;
    if (((vary >> (8 * d)) & 255u) == 0u) continue;
#pragma unroll
    for (int b = 0; b < 8; b++) counts[b * 32 + lane] = 0u;
    __syncwarp();
    uint32_t dr[kM];
#pragma unroll
    for (int j = 0; j < kM; j++) {
      if (j < m) {
        const uint32_t e = (uint32_t)j * 32 + lane;
        const bool valid = e < n;
        const uint32_t dig = (uint32_t)(w[j] >> shift) & 255u;
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < 8; b++) {
          const bool bit = (dig >> b) & 1u;
          const uint32_t bal = __ballot_sync(0xffffffffu, bit);
          peers &= bit ? bal : ~bal;
        }
        const uint32_t cnt = valid ? counts[dig] : 0u;
        __syncwarp();
        dr[j] = 0xFFFFFFFFu;
        if (valid) {
          dr[j] = ((cnt + __popc(peers & lt)) << 8) | dig;
          if (lane == 31 - __clz(peers)) counts[dig] = cnt + __popc(peers);
        }
        __syncwarp();
      }
    }
    // Exclusive scan of the 256 digit counts (8 per lane, then across lanes).
    uint32_t c[8], sum = 0;
#pragma unroll
    for (int b = 0; b < 8; b++) {
      c[b] = counts[lane * 8 + b];
      sum += c[b];
    }
    uint32_t x = sum;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, s);
      if (lane >= s) x += y;
    }
    uint32_t run = x - sum;
    __syncwarp();
#pragma unroll
    for (int b = 0; b < 8; b++) {
      counts[lane * 8 + b] = run;
      run += c[b];
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kM; j++)
      if (j < m && dr[j] != 0xFFFFFFFFu) scratch[counts[dr[j] & 255u] + (dr[j] >> 8)] = w[j];
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kM; j++) {
      const uint32_t e = (uint32_t)j * 32 + lane;
      if (e < n) w[j] = scratch[e];
    }
    __syncwarp();
  }
#pragma unroll
  for (int j = 0; j < kM; j++) {
    const uint32_t e = (uint32_t)j * 32 + lane;
    if (e < n) scratch[e] = w[j];
  }
  __syncwarp();
  // fix_ties: runs of equal depth ordered by splat index.
  for (uint32_t e = lane + 1; e < n; e += 32) {
    const uint32_t kk = (uint32_t)(scratch[e] >> 32);
    if (kk == (uint32_t)(scratch[e - 1] >> 32) && (e == 1 || (uint32_t)(scratch[e - 2] >> 32) != kk)) {
      uint32_t r1 = e + 1;
      while (r1 < n && (uint32_t)(scratch[r1] >> 32) == kk) r1++;
      for (uint32_t i = e; i < r1; i++) {
        const uint64_t v = scratch[i];
        uint32_t j = i;
        while (j > e - 1 && (uint32_t)scratch[j - 1] > (uint32_t)v) {
          scratch[j] = scratch[j - 1];
          j--;
        }
        scratch[j] = v;
      }
    }
  }
  __syncwarp();
  for (uint32_t e = lane; e < n; e += 32) words[e] = scratch[e];
  __syncwarp();
}

}  // namespace splat
