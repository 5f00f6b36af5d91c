// Kernel (c): onesweep LSD radix sort plus the tile ranges.
//
// The reference sorts each tile's bucket stably by depth (radix::sort_hi32,
// src/render/radix.rs:13-57, after a counting sort by tile, cpu.rs:149-199)
// and breaks depth ties by scene index (fix_ties, cpu.rs:396-414). Here two
// stable LSD sorts of 64-bit words produce the same order: all splats by
// depth (words depth bits << 32 | splat, built in splat-index order, so ties
// keep index order; culled splats carry 0xFFFFFFFF and sort last), then,
// after emission in that order, the pairs by tile (words tile << 32 | splat).
// Only the upper 32 bits are digits, 8 bits each. Their histograms come from
// the producers (the projection counts depth digits; the per-tile pair counts
// of the emission give the tile digits), and a digit shared by all words is
// skipped (as sort_hi32 does, radix.rs:389-393). Each remaining digit is one
// onesweep pass: a CTA ranks its 4096-word partition stably (peers by warp
// ballots over the digit bits), publishes its per-digit counts, resolves its
// global offsets by a decoupled look-back over the earlier partitions
// (bounded spin), stages the words in shared memory in partition order and
// writes each digit's run out contiguously.
// Tile ranges ([begin, end) per tile) are the exclusive scan of the per-tile
// pair counts, equal to the reference's neighbour compares over the sorted
// pairs (tiles.wgsl:83-101).
#include "common.cuh"

namespace splat {
namespace {

constexpr int kWarps = kSortThreads / 32;
constexpr uint32_t kLbAgg = 1u << 30;
constexpr uint32_t kLbInc = 2u << 30;
constexpr uint32_t kLbMask = (1u << 30) - 1;

// Words to sort: *count capped at cap, or cap itself when count is null.
__device__ __forceinline__ uint64_t sort_count(const unsigned long long* count, uint64_t cap) {
  if (!count) return cap;
  const unsigned long long t = *(const volatile unsigned long long*)count;
  return t < cap ? t : cap;
}

// Exclusive scans of the digit histograms and the pass schedule (one CTA of
// 256 threads, thread t owning digit value t).
__device__ void schedule_passes(SortState* ss, uint64_t n, int digits) {
  __shared__ uint32_t s_warp[8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
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

__global__ void __launch_bounds__(256) k_hist_scan(SortState* ss, const unsigned long long* count, uint64_t cap,
                                                   int digits) {
  schedule_passes(ss, sort_count(count, cap), digits);
}

// Per-tile [begin, end) from neighbour compares over the tile-sorted pairs
// (tiles.wgsl:83-101); empty tiles keep the zeroed [0, 0).
__global__ void __launch_bounds__(256) k_ranges(uint64_t cap, const uint64_t* p0, const uint64_t* p1,
                                                uint2* __restrict__ ranges, uint32_t tiles, const DevState* st) {
  const uint64_t* __restrict__ pairs = st->tile.final_sel ? p1 : p0;
  const uint64_t n = sort_count(&st->total_pairs, cap);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t t = (uint32_t)(pairs[i] >> 32);
    const uint32_t tn = i + 1 < n ? (uint32_t)(pairs[i + 1] >> 32) : 0xFFFFFFFFu;
    if (i == 0 && t < tiles) ranges[t].x = 0u;
    if (tn != t) {
      if (t < tiles) ranges[t].y = (uint32_t)(i + 1);
      if (tn < tiles) ranges[tn].x = (uint32_t)(i + 1);
    }
  }
}

__global__ void __launch_bounds__(kSortThreads, 3) k_onesweep(SortState* ss, const unsigned long long* count,
                                                              uint64_t cap, int pass, int shift, uint64_t* w0,
                                                              uint64_t* w1, uint32_t* lb, DevState* st) {
  __shared__ uint32_t s_whist[kWarps][256];
  __shared__ uint32_t s_gbase[256];  // global start of digit v's run from this partition
  __shared__ uint32_t s_lbase[256];  // start of digit v's run inside the partition
  __shared__ uint64_t s_keys[kSortPart];
  __shared__ uint32_t s_part;
  __shared__ uint32_t s_wsum[kWarps];
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
    const uint64_t pbase = (uint64_t)part * kSortPart;
    const uint32_t pcount = (uint32_t)min((uint64_t)kSortPart, n - pbase);

    // This warp's 16 x 32 words (warp-striped, coalesced), ranked stably per
    // digit: item (j, lane) is word base + 32 j + lane. Lanes holding the same
    // digit are found with eight ballots over its bits.
    const uint64_t base = pbase + (uint64_t)warp * (kSortItems * 32);
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
      const uint32_t dig = dr[j] & 255u;
      uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
      for (int b = 0; b < 8; b++) {
        const bool bit = (dig >> b) & 1u;
        const uint32_t bal = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? bal : ~bal;
      }
      uint32_t cnt = 0;
      if (valid) cnt = s_whist[warp][dig];
      __syncwarp();
      if (valid) {
        dr[j] = ((cnt + __popc(peers & lt_mask)) << 8) | dig;
        if (lane == 31 - __clz(peers)) s_whist[warp][dig] = cnt + __popc(peers);
      }
      __syncwarp();
    }
    __syncthreads();

    // Thread `tid` owns digit tid: warp offsets, the block count (published
    // at once as this partition's aggregate) and the digit's run start inside
    // the partition (a block scan of the counts).
    uint32_t running = 0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) {
      const uint32_t t = s_whist[w][tid];
      s_whist[w][tid] = running;
      running += t;
    }
    uint32_t* my = lb + (uint64_t)part * 256 + tid;
    *(volatile uint32_t*)my = (part == 0 ? kLbInc : kLbAgg) | running;
    uint32_t x = running;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_wsum[warp] = x;
    __syncthreads();
    uint32_t wb = 0;
    for (int w = 0; w < warp; w++) wb += s_wsum[w];
    s_lbase[tid] = wb + x - running;
    __syncthreads();

    // Place the words in shared memory in partition order (this needs only
    // the partition's own counts), freeing their registers for the look-back.
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
      if (dr[j] != 0xFFFFFFFFu) {
        const uint32_t dig = dr[j] & 255u;
        s_keys[s_lbase[dig] + s_whist[warp][dig] + (dr[j] >> 8)] = key[j];
      }
    }

    // Look back kLookAhead predecessors per step (independent loads), summing
    // aggregates up to and including the nearest inclusive prefix. When a
    // whole wave of partitions starts together, partition p resolves after
    // about p / (2 kLookAhead) load round trips.
    uint32_t prefix = 0;
    if (part != 0) {
      constexpr int kLookAhead = 32;
      long long j = (long long)part - 1;
      bool found = false;
      while (!found && j >= 0) {
        uint32_t v[kLookAhead];
#pragma unroll
        for (int k = 0; k < kLookAhead; k++)
          v[k] = (j - k >= 0) ? *(const volatile uint32_t*)(lb + (uint64_t)(j - k) * 256 + tid) : kLbInc;
#pragma unroll
        for (int k = 0; k < kLookAhead; k++) {
          if (!found) {
            uint32_t spins = 0;
            while ((v[k] >> 30) == 0u) {
              // Give up at the bound, or at once after another wait gave up.
              if (++spins > kSpinLimit ||
                  ((spins & 1023u) == 0u && (*(volatile uint32_t*)&st->error & kErrSortTimeout))) {
                atomicOr(&st->error, kErrSortTimeout);
                v[k] = kLbInc;
                break;
              }
              __nanosleep(20);
              v[k] = *(const volatile uint32_t*)(lb + (uint64_t)(j - k) * 256 + tid);
            }
            prefix += v[k] & kLbMask;
            if ((v[k] >> 30) == 2u) found = true;
          }
        }
        j -= kLookAhead;
      }
      *(volatile uint32_t*)my = kLbInc | (prefix + running);
    }
    s_gbase[tid] = ss->hist[pass][tid] + prefix;
    __syncthreads();
    for (uint32_t l = tid; l < pcount; l += kSortThreads) {
      const uint64_t k = s_keys[l];
      const uint32_t dig = (uint32_t)(k >> shift) & 255u;
      const uint64_t pos = (uint64_t)s_gbase[dig] + (l - s_lbase[dig]);
      if (pos < n)
        out[pos] = k;
      else
        atomicOr(&st->error, kErrSortRange);
    }
    __syncthreads();
  }
}

}  // namespace

cudaError_t launch_sort(SortState* ss, const unsigned long long* count, uint64_t cap, int digits, uint64_t* words0,
                        uint64_t* words1, uint32_t* lookback, uint64_t lookback_parts, DevState* st, int num_sms,
                        cudaStream_t stream) {
  if (digits <= 0) return cudaSuccess;
  for (int d = 0; d < digits; d++) {
    k_onesweep<<<num_sms * 3, kSortThreads, 0, stream>>>(ss, count, cap, d, 32 + 8 * d, words0, words1,
                                                        lookback + (uint64_t)d * lookback_parts * 256, st);
  }
  return cudaGetLastError();
}

cudaError_t launch_depth_schedule(DevState* st, uint64_t n, cudaStream_t stream) {
  k_hist_scan<<<1, 256, 0, stream>>>(&st->depth, nullptr, n, kMaxPasses);  // all n depth words
  return cudaGetLastError();
}

cudaError_t launch_tile_schedule(DevState* st, uint64_t cap, int digits, cudaStream_t stream) {
  k_hist_scan<<<1, 256, 0, stream>>>(&st->tile, &st->total_pairs, cap, digits);
  return cudaGetLastError();
}

cudaError_t launch_ranges(uint64_t cap, uint64_t* const* pairs, uint2* ranges, uint32_t tiles, DevState* st,
                          int num_sms, cudaStream_t stream) {
  k_ranges<<<num_sms * 8, 256, 0, stream>>>(cap, pairs[0], pairs[1], ranges, tiles, st);
  return cudaGetLastError();
}

}  // namespace splat
