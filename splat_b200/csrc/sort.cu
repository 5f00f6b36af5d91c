// Kernel (c): onesweep LSD radix sort of the (tile << 32 | depth bits) keys
// with their splat-index values, plus the tile-range kernel.
//
// The reference sorts each tile's bucket stably by depth (radix::sort_hi32,
// src/render/radix.rs:13-57, after a counting sort by tile, cpu.rs:149-199)
// and breaks depth ties by scene index (fix_ties, cpu.rs:396-414). Here one
// stable LSD sort over the whole key does both: pairs arrive in splat-index
// order, so equal keys keep index order. Digits are 8 bits; one histogram
// pass counts every digit up front, a digit shared by all keys is skipped
// (as sort_hi32 does, radix.rs:389-393), and each remaining digit is one
// onesweep pass: a CTA ranks its 4096-key partition stably with warp
// match-any, publishes per-digit counts, resolves its global offsets by a
// decoupled look-back over earlier partitions (bounded spin), and scatters.
// Tile ranges ([begin, end) per tile) come from neighbour compares over the
// sorted keys, as the reference's `ranges_main` does (tiles.wgsl:83-101).
#include "common.cuh"

namespace splat {
namespace {

constexpr int kWarps = kSortThreads / 32;
constexpr uint32_t kLbAgg = 1u << 30;
constexpr uint32_t kLbInc = 2u << 30;
constexpr uint32_t kLbMask = (1u << 30) - 1;

__device__ __forceinline__ uint64_t pair_count(const DevState* st, uint64_t cap) {
  const unsigned long long t = *(const volatile unsigned long long*)&st->total_pairs;
  return t < cap ? t : cap;
}

__global__ void __launch_bounds__(256) k_hist(const uint64_t* __restrict__ keys, uint64_t cap, int digits,
                                              DevState* st) {
  __shared__ uint32_t h[kMaxDigits][256];
  for (int t = threadIdx.x; t < kMaxDigits * 256; t += blockDim.x) (&h[0][0])[t] = 0u;
  __syncthreads();
  const uint64_t P = pair_count(st, cap);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    for (int d = 0; d < digits; d++) atomicAdd(&h[d][(k >> (8 * d)) & 255u], 1u);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < digits * 256; t += blockDim.x) {
    const uint32_t v = (&h[0][0])[t];
    if (v) atomicAdd(&(&st->hist[0][0])[t], v);
  }
}

// One CTA: exclusive scans of the digit histograms and the pass schedule.
__global__ void __launch_bounds__(256) k_hist_scan(uint64_t cap, int digits, DevState* st) {
  __shared__ uint32_t s_warp[8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t P = pair_count(st, cap);
  int parity = 0;
  for (int d = 0; d < digits; d++) {
    const uint32_t v = st->hist[d][tid];
    const int trivial = __syncthreads_or((uint64_t)v == P);
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
    st->hist[d][tid] = base + x - v;
    __syncthreads();
    if (tid == 0) st->pass_src[d] = trivial ? -1 : parity;
    if (!trivial) parity ^= 1;
  }
  if (tid == 0) {
    for (int d = digits; d < kMaxDigits; d++) st->pass_src[d] = -1;
    st->final_sel = parity;
  }
}

__global__ void __launch_bounds__(kSortThreads, 2) k_onesweep(int d, uint64_t cap, uint64_t* k0, uint32_t* v0,
                                                              uint64_t* k1, uint32_t* v1, uint32_t* lb, DevState* st) {
  __shared__ uint32_t s_whist[kWarps][256];
  __shared__ uint32_t s_gbase[256];
  __shared__ uint32_t s_part;
  const int src = st->pass_src[d];
  if (src < 0) return;
  const uint64_t* __restrict__ kin = src ? k1 : k0;
  const uint32_t* __restrict__ vin = src ? v1 : v0;
  uint64_t* __restrict__ kout = src ? k0 : k1;
  uint32_t* __restrict__ vout = src ? v0 : v1;
  const uint64_t P = pair_count(st, cap);
  const uint32_t nparts = (uint32_t)((P + kSortPart - 1) / kSortPart);
  const int shift = 8 * d;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;

  for (;;) {
    if (tid == 0) s_part = atomicAdd(&st->sort_ticket[d], 1u);
#pragma unroll
    for (int w = 0; w < kWarps; w++) s_whist[w][tid] = 0u;
    __syncthreads();
    const uint32_t part = s_part;
    if (part >= nparts) break;

    // Load this warp's 16 x 32 keys (warp-striped, coalesced) and rank them
    // stably per digit: item (j, lane) is key base + 32 j + lane.
    const uint64_t base = (uint64_t)part * kSortPart + (uint64_t)warp * (kSortItems * 32);
    uint64_t key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t dr[kSortItems];  // rank << 8 | digit, or 0xFFFFFFFF when past the end
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
      const uint64_t idx = base + (uint64_t)j * 32 + lane;
      const bool valid = idx < P;
      key[j] = valid ? kin[idx] : 0ull;
      val[j] = valid ? vin[idx] : 0u;
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
    s_gbase[tid] = st->hist[d][tid] + prefix;
    __syncthreads();

#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
      if (dr[j] != 0xFFFFFFFFu) {
        const uint32_t dig = dr[j] & 255u;
        const uint64_t pos = (uint64_t)s_gbase[dig] + s_whist[warp][dig] + (dr[j] >> 8);
        if (pos < P) {
          kout[pos] = key[j];
          vout[pos] = val[j];
        } else {
          atomicOr(&st->error, kErrSortRange);
        }
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_ranges(uint64_t cap, const uint64_t* k0, const uint64_t* k1,
                                                uint2* __restrict__ ranges, uint32_t tiles, const DevState* st) {
  const uint64_t* __restrict__ keys = st->final_sel ? k1 : k0;
  const uint64_t P = pair_count(st, cap);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t t = (uint32_t)(keys[i] >> 32);
    if (t >= tiles) continue;
    if (i == 0 || (uint32_t)(keys[i - 1] >> 32) != t) ranges[t].x = (uint32_t)i;
    if (i + 1 == P || (uint32_t)(keys[i + 1] >> 32) != t) ranges[t].y = (uint32_t)(i + 1);
  }
}

}  // namespace

cudaError_t launch_sort(uint32_t key_bits, uint64_t cap, uint64_t* keys0, uint32_t* vals0, uint64_t* keys1,
                        uint32_t* vals1, uint32_t* lookback, uint64_t lookback_parts, DevState* st, int num_sms,
                        cudaStream_t stream) {
  const int digits = (int)((key_bits + 7) / 8);
  k_hist<<<num_sms * 4, 256, 0, stream>>>(keys0, cap, digits, st);
  k_hist_scan<<<1, 256, 0, stream>>>(cap, digits, st);
  for (int d = 0; d < digits; d++) {
    k_onesweep<<<num_sms * 2, kSortThreads, 0, stream>>>(d, cap, keys0, vals0, keys1, vals1,
                                                        lookback + (uint64_t)d * lookback_parts * 256, st);
  }
  return cudaGetLastError();
}

cudaError_t launch_ranges(uint64_t cap, uint64_t* const* keys, uint2* ranges, uint32_t tiles, DevState* st,
                          int num_sms, cudaStream_t stream) {
  k_ranges<<<num_sms * 4, 256, 0, stream>>>(cap, keys[0], keys[1], ranges, tiles, st);
  return cudaGetLastError();
}

}  // namespace splat
