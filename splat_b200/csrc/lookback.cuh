// Decoupled look-back of a single-pass exclusive scan over ticketed
// partitions (Merrill & Garland, "Single-pass Parallel Prefix Scan with
// Decoupled Look-back", 2016), one 64-bit descriptor per partition:
// flag (aggregate / inclusive prefix) in the top two bits, value below.
#pragma once

#include "common.cuh"

namespace splat {

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}
__device__ __forceinline__ void st_volatile_u64(unsigned long long* p, unsigned long long v) {
  *(volatile unsigned long long*)p = v;
}

// Called by all 32 lanes of one warp. Publishes this partition's aggregate,
// walks back over its predecessors 32 descriptors at a time until one carries
// an inclusive prefix, publishes this partition's inclusive prefix and returns
// the exclusive prefix (in every lane). Each wait is bounded: on running out
// it sets `err_bit` in st->error and treats the descriptor as zero.
__device__ __forceinline__ unsigned long long lookback_exclusive(unsigned long long* desc, uint32_t part,
                                                                 unsigned long long aggregate, DevState* st,
                                                                 uint32_t err_bit) {
  const int lane = threadIdx.x & 31;
  if (part == 0) {
    if (lane == 0) st_volatile_u64(&desc[0], kFlagInc | aggregate);
    return 0ull;
  }
  if (lane == 0) st_volatile_u64(&desc[part], kFlagAgg | aggregate);
  unsigned long long excl = 0;
  long long j = (long long)part - 1;
  for (;;) {
    const long long idx = j - lane;
    unsigned long long d = kFlagInc;  // before partition 0: an inclusive zero
    if (idx >= 0) {
      uint32_t spins = 0;
      d = ld_volatile_u64(&desc[idx]);
      while ((d >> 62) == 0ull) {
        if (++spins > kSpinLimit || ((spins & 1023u) == 0u && (*(volatile uint32_t*)&st->error & err_bit))) {
          atomicOr(&st->error, err_bit);
          d = kFlagInc;
          break;
        }
        __nanosleep(20);
        d = ld_volatile_u64(&desc[idx]);
      }
    }
    const unsigned inc = __ballot_sync(0xffffffffu, (d >> 62) == 2ull);
    unsigned long long v = d & kValMask;
    if (inc) {
      const int first = __ffs(inc) - 1;
      if (lane > first) v = 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    excl += v;
    if (inc) break;
    j -= 32;
  }
  if (lane == 0) st_volatile_u64(&desc[part], kFlagInc | (excl + aggregate));
  return excl;
}

}  // namespace splat
