// The learned-colour MLP shared by its training kernels (mlp.cu) and the
// fused projection (project.cu): parameter layout, shared-memory tiles,
// tensor-core GEMM issue and the per-row epilogues.
//
// Network: x = [latent (16, fp16) | unit view direction (3) | 1 | 0 x 12]
// -> z1 = W1 x (64; b1 is W1's column 19) -> h1 = relu(z1)
// -> z2 = W2 h1 + b2 (64) -> h2 = relu(z2)
// -> z3 = W3 h2 + b3 (3 of 16) -> rgb = sigmoid(z3).
// Weights are fp16 (tensor-core operands), accumulation is fp32 in TMEM,
// h1 and h2 are rounded to fp16 as the next layer's operand. One CTA tile is
// 128 samples (the M = 128 tcgen05 shape; TMEM lane = sample).
#pragma once

#include <cuda_fp16.h>

#include <cstdint>

#include "umma.cuh"

namespace splat {
namespace mlp {

constexpr uint32_t kLatent = 16;
constexpr uint32_t kIn = 32;      // padded input width
constexpr uint32_t kBiasCol = 19;  // the constant-1 input
constexpr uint32_t kHidden = 64;
constexpr uint32_t kOut = 16;      // padded output width (3 used)
constexpr uint32_t kRows = 128;    // samples per tile

// Flat parameter vector (floats for the masters, halves for the operands):
// row-major W1 64x32, W2 64x64, b2, W3 16x64, b3 (16).
constexpr uint32_t kW1 = 0;
constexpr uint32_t kW2 = kW1 + kHidden * kIn;
constexpr uint32_t kB2 = kW2 + kHidden * kHidden;
constexpr uint32_t kW3 = kB2 + kHidden;
constexpr uint32_t kB3 = kW3 + kOut * kHidden;
constexpr uint32_t kParams = kB3 + kOut;  // 7248

// Instruction descriptors (M = 128 samples).
constexpr uint32_t kIdN64 = umma::idesc_f16(128, 64, false, false);
constexpr uint32_t kIdN16 = umma::idesc_f16(128, 16, false, false);
// Weight gradients: both operands MN-major (K = samples).
constexpr uint32_t kIdWgN96 = umma::idesc_f16(128, 96, true, true);
constexpr uint32_t kIdWgN16 = umma::idesc_f16(128, 16, true, true);

// Inference tiles of one CTA (feature-chunked, 128 rows).
//   act: chunks 0-3 = x; then chunks 0-7 = h1 once layer 1 is done; then h2
//   w1f: W1 as B (n = out 64, k = in 32); w2f: W2 (64 x 64); w3f: W3 (16 x 64)
struct ForwardTiles {
  alignas(128) uint16_t act[kRows * kHidden];
  alignas(128) uint16_t w1f[kHidden * kIn];
  alignas(128) uint16_t w2f[kHidden * kHidden];
  alignas(128) uint16_t w3f[kOut * kHidden];
  alignas(16) float b2[kHidden];
  float b3[4];
};

__device__ __forceinline__ uint32_t pack_half2(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// Copies a row-major fp16 matrix (rows x cols, cols % 8 == 0) from global
// memory into a feature-chunked tile (rows as M/N, cols as K).
__device__ __forceinline__ void load_rows(uint16_t* tile, const uint16_t* __restrict__ g, uint32_t rows, uint32_t cols) {
  const uint32_t groups = rows * cols / 8;
  for (uint32_t q = threadIdx.x; q < groups; q += blockDim.x) {
    const uint32_t r = q / (cols / 8), c = (q % (cols / 8)) * 8;
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(g + (size_t)r * cols + c));
    *reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(tile) + umma::chunked_offset(r, c, rows)) = v;
  }
}
// The transpose: tile row n = source column n, tile column k = source row k,
// for source rows [0, src_rows) and columns [0, out_rows).
__device__ __forceinline__ void load_cols(uint16_t* tile, const uint16_t* __restrict__ g, uint32_t src_rows,
                                          uint32_t src_cols, uint32_t out_rows) {
  const uint32_t groups = out_rows * src_rows / 8;
  for (uint32_t q = threadIdx.x; q < groups; q += blockDim.x) {
    const uint32_t n = q % out_rows, k = (q / out_rows) * 8;
    uint16_t v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = __ldg(g + (size_t)(k + j) * src_cols + n);
    uint4 u;
    u.x = v[0] | ((uint32_t)v[1] << 16);
    u.y = v[2] | ((uint32_t)v[3] << 16);
    u.z = v[4] | ((uint32_t)v[5] << 16);
    u.w = v[6] | ((uint32_t)v[7] << 16);
    *reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(tile) + umma::chunked_offset(n, k, out_rows)) = u;
  }
}

// Stores 8 consecutive features (chunk `chunk`) of row r.
__device__ __forceinline__ void store_chunk(uint16_t* tile, uint32_t r, uint32_t chunk, const float (&v)[8]) {
  uint4 u;
  u.x = pack_half2(v[0], v[1]);
  u.y = pack_half2(v[2], v[3]);
  u.z = pack_half2(v[4], v[5]);
  u.w = pack_half2(v[6], v[7]);
  *reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(tile) + chunk * kRows * 16u + r * 16u) = u;
}
__device__ __forceinline__ void store_chunk_raw(uint16_t* tile, uint32_t r, uint32_t chunk, uint4 u) {
  *reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(tile) + chunk * kRows * 16u + r * 16u) = u;
}

__device__ __forceinline__ void load_forward_weights(ForwardTiles& S, const uint16_t* __restrict__ p) {
  load_rows(S.w1f, p + kW1, kHidden, kIn);
  load_rows(S.w2f, p + kW2, kHidden, kHidden);
  load_rows(S.w3f, p + kW3, kOut, kHidden);
  for (uint32_t i = threadIdx.x; i < kHidden; i += blockDim.x) S.b2[i] = __half2float(__ushort_as_half(p[kB2 + i]));
  for (uint32_t i = threadIdx.x; i < 4; i += blockDim.x)
    S.b3[i] = i < 3 ? __half2float(__ushort_as_half(p[kB3 + i])) : 0.0f;
}

// Inference epilogue of layer 1 or 2 for this thread's row: h = fp16(relu(z
// (+ bias))) from TMEM columns [col, col + 64) into chunks 0-7 of `act`,
// converted and clamped two values at a time (relu after the rounding gives
// the same values: rounding is monotonic and keeps 0).
__device__ __forceinline__ void relu_epilogue(uint32_t tmem_base, uint32_t col, const float* bias, uint16_t* act,
                                              uint32_t r) {
  const __half2 zero = __float2half2_rn(0.0f);
#pragma unroll
  for (uint32_t q = 0; q < 2; q++) {
    float v[32];
    umma::tmem_ld32(umma::tmem_warp_addr(tmem_base, col + 32 * q), v);
    uint32_t h[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
      float a = v[2 * j], b = v[2 * j + 1];
      if (bias) {
        a += bias[32 * q + 2 * j];
        b += bias[32 * q + 2 * j + 1];
      }
      const __half2 x = __hmax2(__floats2half2_rn(a, b), zero);
      h[j] = *reinterpret_cast<const uint32_t*>(&x);
    }
#pragma unroll
    for (int c = 0; c < 4; c++) store_chunk_raw(act, r, 4 * q + c, make_uint4(h[4 * c], h[4 * c + 1], h[4 * c + 2], h[4 * c + 3]));
  }
}

// Writes the input row r: 16 latent halves (two uint4), direction, 1, zeros.
__device__ __forceinline__ void store_input(uint16_t* tile, uint32_t first_chunk, uint32_t r, uint4 lat0, uint4 lat1,
                                            float dx, float dy, float dz) {
  store_chunk_raw(tile, r, first_chunk, lat0);
  store_chunk_raw(tile, r, first_chunk + 1, lat1);
  uint4 u;
  u.x = pack_half2(dx, dy);
  u.y = pack_half2(dz, 1.0f);
  u.z = 0u;
  u.w = 0u;
  store_chunk_raw(tile, r, first_chunk + 2, u);
  store_chunk_raw(tile, r, first_chunk + 3, make_uint4(0u, 0u, 0u, 0u));
}

// D = A * B over k_steps of 16, A K-major (chunks from a_chunk), B K-major.
__device__ __forceinline__ void gemm_k(uint32_t tmem_d, uint32_t a_tile, uint32_t a_chunk, uint32_t b_tile,
                                       uint32_t b_rows, uint32_t k_steps, uint32_t idesc) {
  for (uint32_t s = 0; s < k_steps; s++)
    umma::mma(tmem_d, umma::desc_kmajor(a_tile, kRows, a_chunk + 2 * s), umma::desc_kmajor(b_tile, b_rows, 2 * s),
              idesc, s > 0 ? 1u : 0u);
}

__device__ __forceinline__ float sigmoidf(float z) { return 1.0f / (1.0f + __expf(-z)); }

// Epilogue of layer 1 or 2 for this thread's row: 64 fp32 accumulators from
// TMEM columns [col, col + 64), plus bias, relu, to fp16 chunks 0-7 of `act`.
// Returns the relu mask (bit j: output j > 0 after rounding).
__device__ __forceinline__ uint64_t hidden_epilogue(uint32_t tmem_base, uint32_t col, const float* bias,
                                                    uint16_t* act, uint32_t r) {
  uint64_t mask = 0;
#pragma unroll
  for (uint32_t q = 0; q < 4; q++) {
    float v[16];
    umma::tmem_ld16(umma::tmem_warp_addr(tmem_base, col + 16 * q), v);
#pragma unroll
    for (int j = 0; j < 16; j++) {
      float z = v[j] + (bias ? bias[16 * q + j] : 0.0f);
      z = fmaxf(z, 0.0f);
      // fp16 rounding decides the mask, so backward masks what forward used
      const __half hz = __float2half_rn(z);
      v[j] = __half2float(hz);
      if (v[j] > 0.0f) mask |= 1ull << (16 * q + j);
    }
    float a[8], b[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      a[j] = v[j];
      b[j] = v[8 + j];
    }
    store_chunk(act, r, 2 * q, a);
    store_chunk(act, r, 2 * q + 1, b);
  }
  return mask;
}

// Bijective shuffle of [0, m) (m <= 2^bits): an invertible xorshift-multiply
// hash of `bits`-bit integers, cycle-walked back into range.
__host__ __device__ __forceinline__ uint64_t shuffle_hash(uint64_t x, uint64_t key, uint32_t bits) {
  const uint64_t mask = (bits >= 64) ? ~0ull : ((1ull << bits) - 1);
  const uint32_t s = bits / 2 + 1;
  x = (x ^ key) & mask;
  x ^= x >> s;
  x = (x * 0x9E3779B97F4A7C15ull) & mask;
  x ^= x >> s;
  x = (x * 0xC2B2AE3D27D4EB4Full) & mask;
  x ^= x >> s;
  x = (x * 0x165667B19E3779F9ull) & mask;
  x ^= x >> s;
  return x;
}
__host__ __device__ __forceinline__ uint64_t shuffle_index(uint64_t i, uint64_t m, uint64_t key, uint32_t bits) {
  uint64_t x = shuffle_hash(i, key, bits);
  for (int walk = 0; x >= m && walk < 4096; walk++) x = shuffle_hash(x, key, bits);
  return x < m ? x : i;
}

}  // namespace mlp
}  // namespace splat
