// sm_100a tensor-core primitives (tcgen05 + TMEM) for the learned-colour MLP.
//
// One elected thread issues tcgen05.mma on operands in shared memory,
// described by 64-bit matrix descriptors in the canonical no-swizzle
// ("interleave") layout; the FP32 accumulators live in tensor memory (TMEM)
// and are read back with tcgen05.ld by the warps that own the TMEM lanes.
// Completion is tracked with tcgen05.commit on an mbarrier; every wait is
// bounded by a time limit, after which the caller gives up and reports an
// error instead of hanging.
//
// Operand layout used throughout (fp16, "feature-chunked"): element (row r,
// column c) of a tile with `rows` rows lives at byte
//     (c / 8) * rows * 16 + r * 16 + (c % 8) * 2
// i.e. chunks of 8 columns, each chunk a column of 16-byte row segments. Read
// with the rows as M (or N) and the columns as K, this is the K-major
// canonical layout with SBO = 128 B (next 8 rows) and LBO = rows * 16 B (next
// 8 columns). Read with the columns as M (or N) and the rows as K, the same
// bytes are the MN-major canonical layout with SBO = rows * 16 B and
// LBO = 128 B: so one buffer serves as the A operand of a forward GEMM (rows =
// samples) and as an operand of a weight-gradient GEMM (K = samples) without
// a transpose.
#pragma once

#include <cstdint>

namespace splat {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, c) in a feature-chunked tile of `rows` rows.
__host__ __device__ constexpr uint32_t chunked_offset(uint32_t r, uint32_t c, uint32_t rows) {
  return (c >> 3) * rows * 16u + r * 16u + (c & 7u) * 2u;
}

// Shared-memory matrix descriptor, no swizzle: start address, leading and
// stride byte offsets (all multiples of 16), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// K-major operand: `rows` rows (M or N) of a feature-chunked tile, starting
// at column chunk `chunk` (K advances by 16 per instruction = 2 chunks).
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t tile_saddr, uint32_t rows, uint32_t chunk) {
  return desc(tile_saddr + chunk * rows * 16u, rows * 16u, 128u);
}
// MN-major operand: the columns starting at chunk `chunk` are M (or N), the
// rows are K; `k0` is the first row (a multiple of 8).
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t tile_saddr, uint32_t rows, uint32_t chunk, uint32_t k0) {
  return desc(tile_saddr + chunk * rows * 16u + k0 * 16u, 128u, rows * 16u);
}

// Instruction descriptor, kind::f16: A and B fp16, D fp32, dense.
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t m, uint32_t n, bool a_mn_major, bool b_mn_major) {
  return (1u << 4)                           // D format: F32
         | (0u << 7) | (0u << 10)            // A, B format: F16
         | ((a_mn_major ? 1u : 0u) << 15)    // A major
         | ((b_mn_major ? 1u : 0u) << 16)    // B major
         | ((n >> 3) << 17)                  // N / 8
         | ((m >> 4) << 24);                 // M / 16
}

// D[tmem] (+)= A * B, one instruction (K = 16). Issued by one thread.
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// The mbarrier at `mbar` completes a phase when every tcgen05.mma this thread
// issued before has finished.
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits until the mbarrier's phase with this parity has completed, at most
// `limit_ns` nanoseconds. Returns false when it gave up. Each try_wait may
// suspend the thread for up to 0.1 ms (the hardware resumes it as soon as
// the phase completes), so waiting threads do not spin on the barrier.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint64_t limit_ns = 1000000000ull) {
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity), "r"(100000u)
        : "memory");
    if (done) return true;
    if (it == 0) t0 = globaltimer_ns();
    else if ((it & 63u) == 0 && globaltimer_ns() - t0 > limit_ns) return false;
  }
}

// Orders generic-proxy shared-memory writes before tensor-core reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation by one full warp; the base address goes to *slot (shared).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// Reads 16 consecutive fp32 columns of this thread's TMEM lane (warp w owns
// lanes 32*(w%4) .. +31; `taddr` carries the warp's lane base in bits 16+)
// and waits for the load, in one statement so no use can move above it.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// As tmem_ld16, 32 columns.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// TMEM address of column `col` in the lanes of the calling warp.
__device__ __forceinline__ uint32_t tmem_warp_addr(uint32_t base, uint32_t col) {
  return base + ((((threadIdx.x >> 5) & 3u) * 32u) << 16) + col;
}

}  // namespace umma
}  // namespace splat
