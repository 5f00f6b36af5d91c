// Per-tile depth sort: the reference's per-tile radix::sort_hi32 followed by
// fix_ties (src/render/cpu.rs:208-210, radix.rs:13-57, cpu.rs:396-414), by
// one warp (short tiles: the LSD scheme below), one CTA of kTileThreads
// threads (mid tiles: one counting pass, smem_count_sort) or one CTA over
// chunks in global memory (long tiles, binning.cu: the LSD scheme).
//
// A tile's pairs arrive in arbitrary order (they are bucketed with shared-
// memory atomics). Each pair is the word depth bits << 32 | splat index. A
// stable LSD radix sort on a 16-bit monotone quantisation of the depth (two
// 8-bit passes) orders the pairs up to runs of equal quantised depth; each
// run is then ordered by the full word, i.e. by depth and, within equal
// depth, by splat index. The result is independent of the bucketing order:
// exactly the reference's (depth, scene index) order.
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

// Sort key of a pair: its depth quantised to 16 bits over the tile's depth
// range, q = min(65535, (d - dmin) * (65535 / (dmax - dmin))), truncated.
// Every step is monotone (IEEE subtraction, multiplication by a positive
// factor, truncation), so d1 <= d2 implies q1 <= q2: a stable sort on q
// followed by ordering each run of equal q by the full word (depth bits,
// splat index) gives exactly the (depth, scene index) order.
struct DepthQuant {
  float dmin, scale;
  __device__ __forceinline__ uint32_t operator()(uint64_t word) const {
    const float d = __uint_as_float((uint32_t)(word >> 32));
    const float q = (d - dmin) * scale;
    return q >= 65535.0f ? 65535u : (uint32_t)q;  // d >= dmin, so q >= 0
  }
};

__device__ __forceinline__ DepthQuant make_quant(uint32_t min_bits, uint32_t max_bits) {
  const float dmin = __uint_as_float(min_bits), dmax = __uint_as_float(max_bits);
  const float range = dmax - dmin;
  return DepthQuant{dmin, range > 0.0f ? 65535.0f / range : 0.0f};
}

// Runs of equal quantised key up to this length are ordered by one thread
// (insertion sort: at most kMaxInsertRun^2 / 2 steps); a tile holding a
// longer run is sorted again as a whole by bitonic_sort (degenerate depth
// distributions: a plane seen head-on gives every pair of a tile one depth).
constexpr uint32_t kMaxInsertRun = 32;

// Orders each run of at most kMaxInsertRun items with equal quantised key by
// their full word, the run's first thread sorting it. q(item) gives the
// quantised key, w(item) the 64-bit word (depth bits, splat index) the run is
// ordered by. Returns true in a thread that found a longer run, which it
// leaves as it is (the caller then sorts the whole tile with bitonic_sort).
template <class Item, class Q, class W>
__device__ __forceinline__ bool sort_short_runs(Item* items, uint32_t n, uint32_t tid, uint32_t nthreads, Q&& q,
                                                W&& w) {
  bool long_run = false;
  for (uint32_t e = tid + 1; e < n; e += nthreads) {
    const uint32_t qq = q(items[e]);
    if (qq == q(items[e - 1]) && (e == 1 || q(items[e - 2]) != qq)) {
      uint32_t r1 = e + 1;
      while (r1 < n && r1 - (e - 1) <= kMaxInsertRun && q(items[r1]) == qq) r1++;
      if (r1 - (e - 1) > kMaxInsertRun) {
        long_run = true;
        continue;
      }
      for (uint32_t i = e; i < r1; i++) {
        const Item x = items[i];
        const uint64_t wx = w(x);
        uint32_t j = i;
        while (j > e - 1 && w(items[j - 1]) > wx) {
          items[j] = items[j - 1];
          j--;
        }
        items[j] = x;
      }
    }
  }
  return long_run;
}

// Bitonic sort of words[0, n) (n <= cap, cap a power of two, the array
// holding cap words) by the full word, ascending, by `nthreads` threads
// (thread tid) with sync() between the steps: words[n, m) are padded with
// ~0 up to the power of two m >= n. A tile holds each splat at most once, so
// its words are distinct and the order is exactly (depth, splat index).
template <class Sync>
__device__ __forceinline__ void bitonic_sort(uint64_t* words, uint32_t n, uint32_t tid, uint32_t nthreads,
                                             Sync&& sync) {
  uint32_t m = 1;
  while (m < n) m <<= 1;
  for (uint32_t e = n + tid; e < m; e += nthreads) words[e] = ~0ull;
  sync();
  for (uint32_t k = 2; k <= m; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = tid; i < m / 2; i += nthreads) {
        const uint32_t lo = 2 * i - (i & (j - 1)), hi = lo + j;
        const uint64_t a = words[lo], b = words[hi];
        if ((a > b) == ((lo & k) == 0)) {
          words[lo] = b;
          words[hi] = a;
        }
      }
      sync();
    }
  }
}

// Stable ranks of the elements key[seg0, seg1) of one warp, 32 at a time,
// digit at `shift` (lanes holding the same digit found by ballots over its
// bits). Fills sm.wh[warp] with the warp's digit counts and returns per chunk
// (rank << 8 | digit) in dr[] (0xFFFFFFFF past the end); only the chunks that
// hold elements are ranked.
template <int kChunks>
__device__ __forceinline__ void warp_rank(const uint32_t* key, uint32_t seg0, uint32_t seg1, int shift,
                                          TileSortSmem& sm, uint32_t (&k)[kChunks], uint32_t (&dr)[kChunks]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t nch = (seg1 - seg0 + 31) / 32;
#pragma unroll
  for (int c = 0; c < kChunks; c++) {
    dr[c] = 0xFFFFFFFFu;
    k[c] = 0u;
    if ((uint32_t)c < nch) {
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
      if (valid) {
        dr[c] = ((cnt + __popc(peers & lt)) << 8) | dig;
        if (lane == 31 - __clz(peers)) sm.wh[warp][dig] = cnt + __popc(peers);
      }
      __syncwarp();
    }
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

// Long tiles (more pairs than shared memory holds): stable LSD passes in
// global memory, each over chunks of kSortChunk words staged through shared
// memory, digit starts carried across chunks, ping-pong between the tile's
// words and a scratch range of the same length.
constexpr int kSortChunk = 4096;

struct ChunkSortSmem {
  TileSortSmem t;
  uint32_t run[256];  // running start of each digit across chunks
  uint32_t key[kSortChunk];
};

// Stable LSD passes over the bytes of the 64-bit words whose bit is set in
// `bytes` (bit b: byte b, least significant first; byte 4 is the low byte of
// the depth bits), from src into dst and back. Returns the buffer holding
// the result. One CTA of kTileThreads threads.
__device__ __forceinline__ uint64_t* chunked_lsd(uint64_t* src, uint64_t* dst, uint32_t n, uint32_t bytes,
                                                 ChunkSortSmem& sm) {
  constexpr int kChunks = kSortChunk / (32 * kTileWarps);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int byte = 0; byte < 8; byte++) {
    if (!((bytes >> byte) & 1u)) continue;
    const int shift = 8 * byte, half = byte >> 2, dshift = 8 * (byte & 3);
    // Digit starts over the whole tile.
    clear_counts(sm.t);
    __syncthreads();
    for (uint32_t e = tid; e < n; e += kTileThreads) atomicAdd(&sm.t.wh[warp][(src[e] >> shift) & 255u], 1u);
    __syncthreads();
    digit_offsets(sm.t);
    sm.run[tid] = sm.t.dstart[tid];
    __syncthreads();
    // Stable scatter, chunk by chunk in order.
    for (uint32_t c0 = 0; c0 < n; c0 += kSortChunk) {
      const uint32_t cn = min((uint32_t)kSortChunk, n - c0);
      for (uint32_t e = tid; e < cn; e += kTileThreads) sm.key[e] = (uint32_t)(src[c0 + e] >> (32 * half));
      clear_counts(sm.t);
      __syncthreads();
      const uint32_t seg = (cn + kTileWarps - 1) / kTileWarps;
      const uint32_t seg0 = min(cn, (uint32_t)warp * seg), seg1 = min(cn, seg0 + seg);
      uint32_t k[kChunks], dr[kChunks];
      warp_rank<kChunks>(sm.key, seg0, seg1, dshift, sm.t, k, dr);
      __syncthreads();
      // Exclusive per-warp offsets per digit; the chunk's count per digit.
      uint32_t running = 0;
#pragma unroll
      for (int w = 0; w < kTileWarps; w++) {
        const uint32_t t = sm.t.wh[w][tid];
        sm.t.wh[w][tid] = running;
        running += t;
      }
      __syncthreads();
#pragma unroll
      for (int c = 0; c < kChunks; c++) {
        if (dr[c] != 0xFFFFFFFFu) {
          const uint32_t dig = dr[c] & 255u;
          dst[sm.run[dig] + sm.t.wh[warp][dig] + (dr[c] >> 8)] = src[c0 + seg0 + (uint32_t)c * 32 + lane];
        }
      }
      __syncthreads();
      sm.run[tid] += running;
      __syncthreads();
    }
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

// Sorts words[0, n) in place by the full word (depth bits, then splat
// index: the reference's sort_hi32 + fix_ties order), scratch[0, n) as the
// ping-pong range. The depth bytes that vary over the tile are sorted first;
// runs of equal depth that this leaves (a few equal floats among thousands
// of depths are common) are then ordered by splat index by their first
// thread when at most kMaxInsertRun long; if any run is longer, the tile is
// sorted again over the varying bytes of the splat index and then of the
// depth (LSD over the whole word), so ties never cost more than linear
// passes.
__device__ __forceinline__ void long_tile_sort(uint64_t* words, uint64_t* scratch, uint32_t n, ChunkSortSmem& sm) {
  const int tid = threadIdx.x;
  uint32_t ah = 0xFFFFFFFFu, oh = 0u, al = 0xFFFFFFFFu, ol = 0u;
  for (uint32_t e = tid; e < n; e += kTileThreads) {
    const uint64_t w = words[e];
    ah &= (uint32_t)(w >> 32);
    oh |= (uint32_t)(w >> 32);
    al &= (uint32_t)w;
    ol |= (uint32_t)w;
  }
  uint32_t and_hi, or_hi, and_lo, or_lo;
  block_and_or(ah, oh, sm.t, and_hi, or_hi);
  block_and_or(al, ol, sm.t, and_lo, or_lo);
  const uint32_t vary_hi = and_hi ^ or_hi, vary_lo = and_lo ^ or_lo;
  uint32_t depth_bytes = 0, index_bytes = 0;
  for (int b = 0; b < 4; b++) {
    if ((vary_hi >> (8 * b)) & 255u) depth_bytes |= 1u << (4 + b);
    if ((vary_lo >> (8 * b)) & 255u) index_bytes |= 1u << b;
  }
  uint64_t* res = chunked_lsd(words, scratch, n, depth_bytes, sm);
  const bool long_run = sort_short_runs(
      res, n, (uint32_t)tid, kTileThreads, [](uint64_t x) { return (uint32_t)(x >> 32); },
      [](uint64_t x) { return x; });
  if (__syncthreads_or(long_run))
    res = chunked_lsd(res, res == words ? scratch : words, n, index_bytes | depth_bytes, sm);
  if (res != words)
    for (uint32_t e = tid; e < n; e += kTileThreads) words[e] = res[e];
  __syncthreads();
}

// CTA sort of one tile's n <= kMidSortCap words (already in shared memory,
// their depth-bit range [mn, mx] known): one counting pass on the depth
// quantised to 12 bits over that range, q = min(4095, (d - dmin) * 4095 /
// (dmax - dmin)) (monotone, as DepthQuant), positions handed out by
// shared-memory atomics, then every run of equal q ordered by the full word.
// The order the atomics produce within a run does not matter, so the result
// is exactly the (depth, scene index) order. slot[i] receives the index into
// words[] of the i-th word of the order. The 4096 counters are 16-bit, two
// per word of hist (counts and offsets never exceed n <= 4096).
constexpr int kCountBits = 12;
constexpr uint32_t kCountBuckets = 1u << kCountBits;

struct CountSortSmem {
  uint32_t red[2][kTileWarps];
  uint32_t wsum[kTileWarps];
};

__device__ __forceinline__ void smem_count_sort(uint64_t* words, uint32_t n, uint32_t mn, uint32_t mx,
                                                uint32_t* hist /* kCountBuckets / 2 words */, uint16_t* slot,
                                                CountSortSmem& sm) {
  static_assert(kCountBuckets == 16 * kTileThreads, "16 counters per thread");
  static_assert(kMidSortCap < 65536, "16-bit counters");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float dmin = __uint_as_float(mn), range = __uint_as_float(mx) - dmin;
  const float scale = range > 0.0f ? (float)(kCountBuckets - 1) / range : 0.0f;
  auto quant = [&](uint64_t w) -> uint32_t {
    const float q = (__uint_as_float((uint32_t)(w >> 32)) - dmin) * scale;
    return q >= (float)(kCountBuckets - 1) ? kCountBuckets - 1 : (uint32_t)q;
  };
  // hist was zeroed by the caller before its last barrier.
  for (uint32_t e = tid; e < n; e += kTileThreads) {
    const uint32_t q = quant(words[e]);
    atomicAdd(&hist[q >> 1], 1u << (16 * (q & 1u)));
  }
  __syncthreads();
  // Exclusive scan of the counters, 16 per thread (8 words).
  uint32_t c[16], sum = 0;
  uint4* h4 = reinterpret_cast<uint4*>(hist + 8 * tid);
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
  __syncthreads();
  uint32_t run = x - sum;
  for (int w = 0; w < warp; w++) run += sm.wsum[w];
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
  __syncthreads();
  for (uint32_t e = tid; e < n; e += kTileThreads) {
    const uint32_t q = quant(words[e]), sh = 16 * (q & 1u);
    slot[(atomicAdd(&hist[q >> 1], 1u << sh) >> sh) & 0xFFFFu] = (uint16_t)e;
  }
  __syncthreads();
  const bool long_run = sort_short_runs(
      slot, n, tid, kTileThreads, [&](uint16_t i) { return quant(words[i]); }, [&](uint16_t i) { return words[i]; });
  if (__syncthreads_or(long_run)) {
    bitonic_sort(words, n, tid, kTileThreads, [] { __syncthreads(); });
    for (uint32_t e = tid; e < n; e += kTileThreads) slot[e] = (uint16_t)e;
  }
  __syncthreads();
}

// Warp sort of one tile's n <= kWarpSortCap words in place in global memory.
// The words live in registers, warp-striped (element j*32 + lane); each of
// the two passes on the quantised depth ranks them stably with ballots,
// places them in `scratch` (kWarpSortCap words of shared memory) and reads
// them back striped; runs of equal quantised depth are then ordered by word.
__device__ __forceinline__ void warp_sort_tile(uint64_t* __restrict__ words, uint32_t n, uint64_t* scratch,
                                               uint32_t* counts) {
  constexpr int kM = kWarpSortCap / 32;
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const int m = (int)((n + 31) / 32);
  uint64_t w[kM];
  uint32_t mn = 0xFFFFFFFFu, mx = 0u;
#pragma unroll
  for (int j = 0; j < kM; j++) {
    const uint32_t e = (uint32_t)j * 32 + lane;
    w[j] = 0ull;
    if (j < m && e < n) {
      w[j] = words[e];
      mn = min(mn, (uint32_t)(w[j] >> 32));
      mx = max(mx, (uint32_t)(w[j] >> 32));
    }
  }
#pragma unroll
  for (int s2 = 16; s2 > 0; s2 >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, s2));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, s2));
  }
  const DepthQuant quant = make_quant(mn, mx);
  uint32_t a = 0xFFFFFFFFu, o = 0u;
#pragma unroll
  for (int j = 0; j < kM; j++) {
    const uint32_t e = (uint32_t)j * 32 + lane;
    if (j < m && e < n) {
      const uint32_t q = quant(w[j]);
      a &= q;
      o |= q;
    }
  }
#pragma unroll
  for (int s2 = 16; s2 > 0; s2 >>= 1) {
    a &= __shfl_xor_sync(0xffffffffu, a, s2);
    o |= __shfl_xor_sync(0xffffffffu, o, s2);
  }
  const uint32_t vary = a ^ o;
  for (int d = 0; d < 2; d++) {
    const int shift = 8 * d;
    if (((vary >> shift) & 255u) == 0u) continue;
#pragma unroll
    for (int b = 0; b < 8; b++) counts[b * 32 + lane] = 0u;
    __syncwarp();
    uint32_t dr[kM];
#pragma unroll
    for (int j = 0; j < kM; j++) {
      dr[j] = 0xFFFFFFFFu;
      if (j < m) {
        const uint32_t e = (uint32_t)j * 32 + lane;
        const bool valid = e < n;
        const uint32_t dig = (quant(w[j]) >> shift) & 255u;
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < 8; b++) {
          const bool bit = (dig >> b) & 1u;
          const uint32_t bal = __ballot_sync(0xffffffffu, bit);
          peers &= bit ? bal : ~bal;
        }
        const uint32_t cnt = valid ? counts[dig] : 0u;
        __syncwarp();
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
    for (int s2 = 1; s2 < 32; s2 <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, s2);
      if (lane >= s2) x += y;
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
      if (dr[j] != 0xFFFFFFFFu) scratch[counts[dr[j] & 255u] + (dr[j] >> 8)] = w[j];
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kM; j++) {
      const uint32_t e = (uint32_t)j * 32 + lane;
      if (j < m && e < n) w[j] = scratch[e];
    }
    __syncwarp();
  }
#pragma unroll
  for (int j = 0; j < kM; j++) {
    const uint32_t e = (uint32_t)j * 32 + lane;
    if (j < m && e < n) scratch[e] = w[j];
  }
  __syncwarp();
  const bool long_run = sort_short_runs(
      scratch, n, lane, 32, [&](uint64_t x) { return quant(x); }, [](uint64_t x) { return x; });
  if (__any_sync(0xffffffffu, long_run)) bitonic_sort(scratch, n, lane, 32, [] { __syncwarp(); });
  __syncwarp();
  for (uint32_t e = lane; e < n; e += 32) words[e] = scratch[e];
  __syncwarp();
}

}  // namespace splat
