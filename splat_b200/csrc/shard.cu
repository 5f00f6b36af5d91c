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
constexpr uint32_t kShardWarps = kShardThreads / 32;
// Each warp of the count and scatter launches walks one chunk of kShardChunk
// consecutive splats, 32 at a time, in scene order: the scatter orders each
// window's records within a chunk by ballots alone (no block barrier), and
// the chunks' counts, scanned in chunk order, place the chunks.
constexpr uint32_t kShardChunk = 256;

__host__ __device__ __forceinline__ uint64_t shard_chunks(uint64_t n) {
  return n ? (n + kShardChunk - 1) / kShardChunk : 1;
}
uint32_t shard_ctas(uint64_t n) { return (uint32_t)((shard_chunks(n) + kShardWarps - 1) / kShardWarps); }

// The pixel rows [y0, y1) of splat i's bbox, if it is visible and its bbox
// holds a pixel of the frame (the projection ran over the whole frame).
__device__ __forceinline__ bool splat_rows(const Record* __restrict__ rec, const BinInfo* __restrict__ bin, uint64_t i,
                                           uint32_t& y0, uint32_t& y1) {
  if (bin_count(bin[i]) == 0u) return false;
  const uint32_t yb = __float_as_uint(rec[i].r2.z);
  y0 = yb & 0xFFFFu;
  y1 = yb >> 16;
  return true;
}

__device__ __forceinline__ bool meets(const ShardWindows& w, uint32_t k, uint32_t y0, uint32_t y1) {
  return w.bound[k] < y1 && w.bound[k + 1] > y0;
}

// Records per (window, chunk): cnt[k * chunks + chunk].
__global__ void __launch_bounds__(kShardThreads) k_shard_count(const Record* __restrict__ rec,
                                                               const BinInfo* __restrict__ bin, uint64_t n,
                                                               const ShardWindows w, uint32_t* __restrict__ cnt) {
  __shared__ uint32_t c[kShardWarps][kMaxShardWindows];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t chunk = (uint64_t)blockIdx.x * kShardWarps + warp;
  if (chunk >= shard_chunks(n)) return;  // whole warps: no block barrier follows
  for (uint32_t k = lane; k < w.n; k += 32) c[warp][k] = 0u;
  __syncwarp();
  const uint64_t s0 = chunk * kShardChunk, s1 = n < s0 + kShardChunk ? n : s0 + kShardChunk;
  for (uint64_t b0 = s0; b0 < s1; b0 += 32) {
    const uint64_t i = b0 + lane;
    uint32_t y0 = 0, y1 = 0;
    const bool v = i < s1 && splat_rows(rec, bin, i, y0, y1);
    for (uint32_t k = 0; k < w.n; k++) {
      const uint32_t m = __ballot_sync(0xffffffffu, v && meets(w, k, y0, y1));
      if (lane == 0) c[warp][k] += (uint32_t)__popc(m);
    }
  }
  __syncwarp();
  const uint64_t chunks = shard_chunks(n);
  for (uint32_t k = lane; k < w.n; k += 32) cnt[k * chunks + chunk] = c[warp][k];
}

// CTA k: the exclusive scan of window k's chunk counts into off[k * chunks +
// chunk] and their sum into totals[k] (the windows are scanned side by side;
// the scatter adds the earlier windows' totals).
__global__ void __launch_bounds__(1024) k_shard_scan(const uint32_t* __restrict__ cnt, uint32_t chunks,
                                                     unsigned long long* __restrict__ off,
                                                     unsigned long long* __restrict__ totals) {
  __shared__ unsigned long long wsum[32];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, k = blockIdx.x;
  const uint32_t* src = cnt + (uint64_t)k * chunks;
  unsigned long long* dst = off + (uint64_t)k * chunks;
  unsigned long long carry = 0;
  for (uint32_t c0 = 0; c0 < chunks; c0 += 1024) {
    const uint32_t c = c0 + tid;
    const unsigned long long v = c < chunks ? src[c] : 0ull;
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
    if (c < chunks) dst[c] = carry + before + x - v;
    carry += all;
    __syncthreads();  // wsum is rewritten by the next block of chunks
  }
  if (tid == 0) totals[k] = carry;
}

// Writes the records: each warp walks its chunk 32 splats at a time, in
// scene order, and places each window's records of the 32 after those
// already written (a ballot prefix; the window cursors live in the warp's
// shared-memory row).
__global__ void __launch_bounds__(kShardThreads) k_shard_scatter(const Record* __restrict__ rec,
                                                                 const BinInfo* __restrict__ bin, uint64_t n,
                                                                 const ShardWindows w,
                                                                 const unsigned long long* __restrict__ off,
                                                                 const unsigned long long* __restrict__ totals,
                                                                 Record* __restrict__ send, uint64_t cap) {
  __shared__ unsigned long long cur[kShardWarps][kMaxShardWindows];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t chunk = (uint64_t)blockIdx.x * kShardWarps + warp, chunks = shard_chunks(n);
  if (chunk >= chunks) return;
  for (uint32_t k = lane; k < w.n; k += 32) {
    unsigned long long base = 0;  // the records of the windows before k
    for (uint32_t j = 0; j < k; j++) base += totals[j];
    cur[warp][k] = base + off[k * chunks + chunk];
  }
  __syncwarp();
  const uint64_t s0 = chunk * kShardChunk, s1 = n < s0 + kShardChunk ? n : s0 + kShardChunk;
  const uint32_t below = (1u << lane) - 1u;
  for (uint64_t b0 = s0; b0 < s1; b0 += 32) {
    const uint64_t i = b0 + lane;
    uint32_t y0 = 0, y1 = 0;
    const bool v = i < s1 && splat_rows(rec, bin, i, y0, y1);
    Record r{};
    if (v) r = rec[i];
    for (uint32_t k = 0; k < w.n; k++) {
      const bool hit = v && meets(w, k, y0, y1);
      const uint32_t m = __ballot_sync(0xffffffffu, hit);
      if (m == 0u) continue;  // uniform over the warp
      const unsigned long long pos = cur[warp][k] + (uint32_t)__popc(m & below);
      if (hit && pos < cap) send[pos] = r;
      __syncwarp();  // every lane has read cur[warp][k]
      if (lane == 0) cur[warp][k] += (uint32_t)__popc(m);
      __syncwarp();
    }
  }
}

__global__ void __launch_bounds__(256) k_records_bin(const ViewTask t, ViewTask* table, FrameCounters fc) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *table = t;
  const uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
  const bool v = i < t.s.n;
  if (v) {
    const Record r = t.rec[i];
    const uint32_t xb = __float_as_uint(r.r2.y), yb = __float_as_uint(r.r2.z);
    BinInfo b;
    BinSkip k;
    b.depth_bits = __float_as_uint(r.r2.w);
    if (window_rect(t.fp, xb & 0xFFFFu, xb >> 16, yb & 0xFFFFu, yb >> 16, r, b, k)) t.skip[i] = k;
    t.bin[i] = b;
  }
  const uint32_t c = (uint32_t)__syncthreads_count(v);
  if (threadIdx.x == 0 && c) {
    atomicAdd(&fc.st->visible, (unsigned long long)c);
    atomicAdd(&fc.view_visible[0], (unsigned long long)c);
  }
}

// Scratch layout: offsets (u64, chunks x windows), then counts (u32, same).
struct ShardScratch {
  unsigned long long* off;
  uint32_t* cnt;
};
ShardScratch shard_scratch_at(void* p, uint64_t n, uint32_t windows) {
  const size_t cells = (size_t)shard_chunks(n) * windows;
  ShardScratch s;
  s.off = static_cast<unsigned long long*>(p);
  s.cnt = reinterpret_cast<uint32_t*>(s.off + cells);
  return s;
}

}  // namespace

size_t shard_scratch_bytes(uint64_t n, uint32_t windows) {
  return (size_t)shard_chunks(n) * windows * (sizeof(unsigned long long) + sizeof(uint32_t));
}

cudaError_t launch_shard_count(const Record* rec, const BinInfo* bin, uint64_t n, const ShardWindows& w,
                               void* scratch, unsigned long long* totals, cudaStream_t stream, uint32_t* launches) {
  const ShardScratch s = shard_scratch_at(scratch, n, w.n);
  k_shard_count<<<shard_ctas(n), kShardThreads, 0, stream>>>(rec, bin, n, w, s.cnt);
  k_shard_scan<<<w.n, 1024, 0, stream>>>(s.cnt, (uint32_t)shard_chunks(n), s.off, totals);
  *launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_shard_scatter(const Record* rec, const BinInfo* bin, uint64_t n, const ShardWindows& w,
                                 const void* scratch, const unsigned long long* totals, Record* send, uint64_t cap,
                                 cudaStream_t stream, uint32_t* launches) {
  const ShardScratch s = shard_scratch_at(const_cast<void*>(scratch), n, w.n);
  k_shard_scatter<<<shard_ctas(n), kShardThreads, 0, stream>>>(rec, bin, n, w, s.off, totals, send, cap);
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
