// Kernel (b): device-wide exclusive scan of the per-splat pair counts with
// warp shuffles and a decoupled look-back (single pass; each CTA takes its
// partition from a ticket so every predecessor is already resident), fused
// with the pair emission: each visible splat writes one 64-bit key
// (tile << 32 | depth bits) and its splat index per tile of its pixel bbox,
// row-major (ty, then tx) as the reference's `emit` does
// (src/render/cpu.rs:251-277). Offsets come from the scan in splat-index
// order, so pairs are laid out in index order and a stable sort by key gives
// the reference's (tile, depth, scene index) order (src/render/naive.rs:
// 306-308, src/render/cpu.rs:396-414).
#include "common.cuh"

namespace splat {
namespace {

constexpr int kEmitThreads = 512;
constexpr int kEmitWarps = kEmitThreads / 32;

__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}
__device__ __forceinline__ void st_volatile(unsigned long long* p, unsigned long long v) {
  *(volatile unsigned long long*)p = v;
}

__global__ void __launch_bounds__(kEmitThreads) k_emit(uint32_t tiles_x, const BinInfo* __restrict__ bin, uint64_t n,
                                                       unsigned long long* desc, uint64_t* __restrict__ keys,
                                                       uint32_t* __restrict__ vals, uint64_t cap, DevState* st) {
  __shared__ uint32_t s_part;
  __shared__ uint32_t s_warp[kEmitWarps];
  __shared__ unsigned long long s_excl;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_part = atomicAdd(&st->emit_ticket, 1u);
  __syncthreads();
  const uint32_t part = s_part;
  const uint64_t nparts = (n + kEmitThreads - 1) / kEmitThreads;
  const uint64_t i = (uint64_t)part * kEmitThreads + tid;
  BinInfo b{kCulled, 0u, 0u, 0u};
  if (i < n) b = bin[i];
  const uint32_t cnt = (b.rect_lo != kCulled) ? b.count : 0u;

  // Block-wide exclusive scan of the counts.
  uint32_t x = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kEmitWarps ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kEmitWarps) s_warp[lane] = w;  // inclusive per warp
  }
  __syncthreads();
  const uint32_t warp_excl = warp ? s_warp[warp - 1] : 0u;
  const uint32_t local_excl = warp_excl + x - cnt;
  const unsigned long long block_total = s_warp[kEmitWarps - 1];

  // Decoupled look-back over the partition descriptors (warp 0).
  if (warp == 0) {
    unsigned long long excl = 0;
    if (part == 0) {
      if (lane == 0) st_volatile(&desc[0], kFlagInc | block_total);
    } else {
      if (lane == 0) st_volatile(&desc[part], kFlagAgg | block_total);
      long long j = (long long)part - 1;
      bool done = false;
      while (!done) {
        const long long idx = j - lane;
        unsigned long long d = kFlagInc;  // before partition 0: an inclusive zero
        if (idx >= 0) {
          uint32_t spins = 0;
          d = ld_volatile(&desc[idx]);
          while ((d >> 62) == 0ull) {
            if (++spins > kSpinLimit || ((spins & 1023u) == 0u && (*(volatile uint32_t*)&st->error & kErrEmitTimeout))) {
              atomicOr(&st->error, kErrEmitTimeout);
              d = kFlagInc;
              break;
            }
            __nanosleep(20);
            d = ld_volatile(&desc[idx]);
          }
        }
        const unsigned inc = __ballot_sync(0xffffffffu, (d >> 62) == 2ull);
        unsigned long long v = d & kValMask;
        if (inc) {
          const int first = __ffs(inc) - 1;
          if (lane > first) v = 0;
          done = true;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        j -= 32;
      }
      if (lane == 0) st_volatile(&desc[part], kFlagInc | (excl + block_total));
    }
    if (lane == 0) {
      s_excl = excl;
      if ((uint64_t)part == nparts - 1) st->total_pairs = excl + block_total;
    }
  }
  __syncthreads();

  if (cnt) {
    uint64_t off = s_excl + local_excl;
    const uint32_t tx0 = b.rect_lo & 0xFFFFu, ty0 = b.rect_lo >> 16;
    const uint32_t tx1 = b.rect_hi & 0xFFFFu, ty1 = b.rect_hi >> 16;
    const uint64_t lo = b.depth_bits;
    for (uint32_t ty = ty0; ty < ty1 && off < cap; ty++) {
      for (uint32_t tx = tx0; tx < tx1; tx++, off++) {
        if (off >= cap) break;
        keys[off] = ((uint64_t)(ty * tiles_x + tx) << 32) | lo;
        vals[off] = (uint32_t)i;
      }
    }
  }
}

}  // namespace

cudaError_t launch_emit(const FrameParams& fp, const BinInfo* bin, uint64_t n, unsigned long long* emit_desc,
                        uint64_t* keys, uint32_t* vals, uint64_t cap, DevState* st, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const unsigned grid = (unsigned)((n + kEmitThreads - 1) / kEmitThreads);
  k_emit<<<grid, kEmitThreads, 0, stream>>>(fp.tiles_x, bin, n, emit_desc, keys, vals, cap, st);
  return cudaGetLastError();
}

}  // namespace splat
