// Splat-sharded frames: one frame drawn by several devices, each holding a
// share of the splats, with one exchange of projected splats between them
// (tile ownership by row windows).
//
// Sender (one device, its shard): the projection runs over the whole frame;
// every visible splat whose pixel bbox holds a pixel then goes, as its
// 48-byte Record, to each row window its bbox rows meet. Per window the
// records keep scene order, so a receiver that concatenates the senders'
// records in shard order holds them in global scene order, and the pair
// words it forms from record positions (depth << 32 | position) sort exactly
// as the global (depth, splat index) keys of the whole-frame render do.
//
// Receiver (the window's owner): the records' tile rectangles for its
// window take the projection's place (k_records_bin); binning, sorts and
// blend are the single-device pipeline's. Every pixel of the window sees
// the splats whose bbox holds it, in the same order, so the window is the
// whole-frame render's rows bit for bit.
//
// The reference has no multi-device path; the pipeline it splits is
// Renderer::render (src/render/mod.rs:89-96, src/render/cpu.rs:109-222).
#include <algorithm>

#include "common.cuh"

namespace splat {
namespace {

constexpr uint32_t kShardThreads = 256;
constexpr uint32_t kShardPerCta = 4096;  // splats per CTA of the count and scatter launches

uint32_t shard_ctas(uint64_t n) { return (uint32_t)std::max<uint64_t>(1, (n + kShardPerCta - 1) / kShardPerCta); }

// The pixel rows [y0, y1) of splat i's bbox, if it is visible and its bbox
// holds a pixel of the frame (the projection ran over the whole frame).
__device__ __forceinline__ bool splat_rows(const Record* __restrict__ rec, const BinInfo* __restrict__ bin, uint64_t i,
                                           uint32_t& y0, uint32_t& y1) {
  const BinInfo b = bin[i];
  if (b.rect_lo == kCulled || b.count == 0u) return false;
  const uint32_t yb = __float_as_uint(rec[i].r2.z);
  y0 = yb & 0xFFFFu;
  y1 = yb >> 16;
  return true;
}

__device__ __forceinline__ bool meets(const ShardWindows& w, uint32_t k, uint32_t y0, uint32_t y1) {
  return w.bound[k] < y1 && w.bound[k + 1] > y0;
}

// Records per (CTA, window): cnt[cta * w.n + k].
__global__ void __launch_bounds__(kShardThreads) k_shard_count(const Record* __restrict__ rec,
                                                               const BinInfo* __restrict__ bin, uint64_t n,
                                                               const ShardWindows w, uint32_t* __restrict__ cnt) {
  __shared__ uint32_t c[kMaxShardWindows];
  const uint32_t tid = threadIdx.x, lane = tid & 31;
  for (uint32_t k = tid; k < w.n; k += kShardThreads) c[k] = 0u;
  __syncthreads();
  const uint64_t s0 = (uint64_t)blockIdx.x * kShardPerCta, s1 = n < s0 + kShardPerCta ? n : s0 + kShardPerCta;
  // Whole warps walk the range (s1 - s0 rounded up), so every ballot is full.
  for (uint64_t i = s0 + tid; i < s0 + ((s1 - s0 + 31) & ~31ull); i += kShardThreads) {
    uint32_t y0 = 0, y1 = 0;
    const bool v = i < s1 && splat_rows(rec, bin, i, y0, y1);
    for (uint32_t k = 0; k < w.n; k++) {
      const uint32_t m = __ballot_sync(0xffffffffu, v && meets(w, k, y0, y1));
      if (lane == 0 && m) atomicAdd(&c[k], (uint32_t)__popc(m));
    }
  }
  __syncthreads();
  for (uint32_t k = tid; k < w.n; k += kShardThreads) cnt[(uint64_t)blockIdx.x * w.n + k] = c[k];
}

// One CTA: per window, the exclusive scan of the CTAs' counts, offset by the
// totals of the windows before it, into off[cta * w.n + k]; totals[k].
__global__ void __launch_bounds__(1024) k_shard_scan(const uint32_t* __restrict__ cnt, uint32_t ctas,
                                                     const ShardWindows w, unsigned long long* __restrict__ off,
                                                     unsigned long long* __restrict__ totals) {
  __shared__ unsigned long long wsum[32];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned long long base = 0;  // records of the windows before k
  for (uint32_t k = 0; k < w.n; k++) {
    unsigned long long carry = base;
    for (uint32_t c0 = 0; c0 < ctas; c0 += 1024) {
      const uint32_t c = c0 + tid;
      const unsigned long long v = c < ctas ? cnt[(uint64_t)c * w.n + k] : 0ull;
      unsigned long long x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
      }
      if (lane == 31) wsum[warp] = x;
      __syncthreads();
      unsigned long long before = 0, all = 0;
      for (uint32_t q = 0; q < 32; q++) {
        if (q < warp) before += wsum[q];
        all += wsum[q];
      }
      if (c < ctas) off[(uint64_t)c * w.n + k] = carry + before + x - v;
      carry += all;
      __syncthreads();  // wsum is rewritten by the next chunk
    }
    if (tid == 0) totals[k] = carry - base;
    base = carry;
  }
}

// Writes the records: each CTA walks its splats in rounds of 256, in scene
// order, and places the round's records of window k after those of the
// earlier rounds (a block-wide ballot scan per window).
__global__ void __launch_bounds__(kShardThreads) k_shard_scatter(const Record* __restrict__ rec,
                                                                 const BinInfo* __restrict__ bin, uint64_t n,
                                                                 const ShardWindows w,
                                                                 const unsigned long long* __restrict__ off,
                                                                 Record* __restrict__ send, uint64_t cap) {
  __shared__ unsigned long long cur[kMaxShardWindows];
  __shared__ uint32_t wcnt[kShardThreads / 32];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (uint32_t k = tid; k < w.n; k += kShardThreads) cur[k] = off[(uint64_t)blockIdx.x * w.n + k];
  __syncthreads();
  const uint64_t s0 = (uint64_t)blockIdx.x * kShardPerCta, s1 = n < s0 + kShardPerCta ? n : s0 + kShardPerCta;
  for (uint64_t r0 = s0; r0 < s1; r0 += kShardThreads) {
    const uint64_t i = r0 + tid;
    uint32_t y0 = 0, y1 = 0;
    const bool v = i < s1 && splat_rows(rec, bin, i, y0, y1);
    Record r{};
    if (v) r = rec[i];
    for (uint32_t k = 0; k < w.n; k++) {
      const bool hit = v && meets(w, k, y0, y1);
      if (!__syncthreads_or(hit)) continue;  // uniform: no record of this round goes to k
      const uint32_t m = __ballot_sync(0xffffffffu, hit);
      if (lane == 0) wcnt[warp] = (uint32_t)__popc(m);
      __syncthreads();
      uint32_t before = 0, all = 0;
#pragma unroll
      for (uint32_t q = 0; q < kShardThreads / 32; q++) {
        if (q < warp) before += wcnt[q];
        all += wcnt[q];
      }
      const unsigned long long pos = cur[k] + before + (uint32_t)__popc(m & ((1u << lane) - 1u));
      if (hit && pos < cap) send[pos] = r;
      __syncthreads();  // every thread has read cur[k] and wcnt
      if (tid == 0) cur[k] += all;
      // cur[k] is read again only after the next round's __syncthreads_or.
    }
  }
}

__global__ void __launch_bounds__(256) k_records_bin(const ViewTask t, ViewTask* table, FrameCounters fc) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *table = t;
  const uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
  const bool v = i < t.s.n;
  if (v) {
    const float4 r2 = t.rec[i].r2;
    const uint32_t xb = __float_as_uint(r2.y), yb = __float_as_uint(r2.z);
    BinInfo b;
    b.depth_bits = __float_as_uint(r2.w);
    window_rect(t.fp, xb & 0xFFFFu, xb >> 16, yb & 0xFFFFu, yb >> 16, b);
    t.bin[i] = b;
  }
  const uint32_t c = (uint32_t)__syncthreads_count(v);
  if (threadIdx.x == 0 && c) {
    atomicAdd(&fc.st->visible, (unsigned long long)c);
    atomicAdd(&fc.view_visible[0], (unsigned long long)c);
  }
}

// Scratch layout: offsets (u64, ctas x windows), then counts (u32, same).
struct ShardScratch {
  unsigned long long* off;
  uint32_t* cnt;
};
ShardScratch shard_scratch_at(void* p, uint64_t n, uint32_t windows) {
  const size_t cells = (size_t)shard_ctas(n) * windows;
  ShardScratch s;
  s.off = static_cast<unsigned long long*>(p);
  s.cnt = reinterpret_cast<uint32_t*>(s.off + cells);
  return s;
}

}  // namespace

size_t shard_scratch_bytes(uint64_t n, uint32_t windows) {
  return (size_t)shard_ctas(n) * windows * (sizeof(unsigned long long) + sizeof(uint32_t));
}

cudaError_t launch_shard_count(const Record* rec, const BinInfo* bin, uint64_t n, const ShardWindows& w,
                               void* scratch, unsigned long long* totals, cudaStream_t stream, uint32_t* launches) {
  const uint32_t ctas = shard_ctas(n);
  const ShardScratch s = shard_scratch_at(scratch, n, w.n);
  k_shard_count<<<ctas, kShardThreads, 0, stream>>>(rec, bin, n, w, s.cnt);
  k_shard_scan<<<1, 1024, 0, stream>>>(s.cnt, ctas, w, s.off, totals);
  *launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_shard_scatter(const Record* rec, const BinInfo* bin, uint64_t n, const ShardWindows& w,
                                 const void* scratch, Record* send, uint64_t cap, cudaStream_t stream,
                                 uint32_t* launches) {
  const ShardScratch s = shard_scratch_at(const_cast<void*>(scratch), n, w.n);
  k_shard_scatter<<<shard_ctas(n), kShardThreads, 0, stream>>>(rec, bin, n, w, s.off, send, cap);
  *launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_records_bin(const ViewTask& t, ViewTask* table, const FrameCounters& fc, cudaStream_t stream,
                               uint32_t* launches) {
  const unsigned grid = t.s.n ? (unsigned)((t.s.n + 255) / 256) : 1u;
  k_records_bin<<<grid, 256, 0, stream>>>(t, table, fc);
  *launches += 1;
  return cudaGetLastError();
}

}  // namespace splat
