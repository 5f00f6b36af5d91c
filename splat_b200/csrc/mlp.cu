// Learned colour: training of the per-splat latents and the shared MLP
// (mlp.cuh) on the exact SH colours of a scene, with hand-written tcgen05
// kernels, plus the C ABI of the learner (include/splat_cuda.h).
//
// No counterpart in the reference, which evaluates degree-3 SH per splat
// (src/sh.rs:39-64, src/render/mod.rs:250-257). The targets are that exact
// evaluation, clamped to [0, 1] (a sigmoid head cannot exceed 1; the
// reference clamps only at 0), at `n_dirs` Fibonacci-sphere directions per
// splat: sample s of an epoch is (splat, direction) = divmod(perm(s), n_dirs)
// for a bijective shuffle `perm` of [0, n * n_dirs) keyed by the epoch.
//
// One step over `batch` samples is two launches:
//   k_train<SRC>     forward + backward, 128 samples per tile, persistent CTAs;
//                    weight gradients accumulate in TMEM over a CTA's tiles and
//                    are added to one fp32 vector; latent gradients are added
//                    to per-splat rows
//   k_adam           Adam on the fp32 master parameters (fp16 operand copy
//                    refreshed) and lazy Adam on the latent rows the step
//                    sampled (found again from the epoch's shuffle)
// Loss: mean over active samples and channels of (rgb - target)^2.
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "handle.h"
#include "mlp.cuh"
#include "sh.cuh"

#define SPLAT_API extern "C" __attribute__((visibility("default")))

using namespace splat;

static_assert(mlp::kW1 == SPLAT_MLP_W1 && mlp::kW2 == SPLAT_MLP_W2 && mlp::kB2 == SPLAT_MLP_B2 &&
                  mlp::kW3 == SPLAT_MLP_W3 && mlp::kB3 == SPLAT_MLP_B3 && mlp::kParams == SPLAT_MLP_PARAMS &&
                  mlp::kLatent == SPLAT_MLP_LATENT,
              "parameter layout of the C ABI");

namespace {

constexpr uint32_t kTrainThreads = 128;
constexpr uint32_t kTrainTmemCols = 256;
// TMEM columns of the training kernel.
constexpr uint32_t kTW = 0;     // [dz2 | dz1]^T [h1 | x]: 128 x 96 (dW2, db2, dW1)
constexpr uint32_t kTW3 = 96;   // [h2 | dz2]^T dz3: 128 x 16 (dW3^T)
constexpr uint32_t kTS = 128;   // z1, z2, dh2, dh1 (64)
constexpr uint32_t kTZ = 192;   // z3, dx (16)
// dz3 is scaled by this before its fp16 rounding (keeps the backward
// operands in fp16's normal range); the Adam kernels divide it out.
constexpr float kLossScale = 128.0f;

struct TrainSmem {
  alignas(128) uint16_t R[mlp::kRows * 96];   // chunks 0-7 h1, 8-11 x
  alignas(128) uint16_t Q[mlp::kRows * 192];  // chunks 0-7 h2, 8-15 dz2, 16-23 dz1
  alignas(128) uint16_t D3[mlp::kRows * 16];  // chunks 0-1 dz3
  alignas(128) uint16_t w1f[64 * 32];         // B: n = out, k = in
  alignas(128) uint16_t w2f[64 * 64];
  alignas(128) uint16_t w2b[64 * 64];         // B: n = in, k = out (W2^T)
  alignas(128) uint16_t w1b[16 * 64];         // W1^T, latent inputs only
  float w3[3][64];  // layer 3 on the CUDA cores: the fp16 values of W3's rows 0-2
  float b2[64];
  float b3[16];
  float db3[16];
  uint64_t mbar;
  uint64_t lost;  // never arrived on: the injected lost completion (StepState::lost_wait_us)
  uint32_t tmem;
};

// Device step state of a learner.
struct StepState {
  unsigned long long step;  // completed steps
  double loss_step;         // sum of squared errors of the running step
  double loss_sum;          // sum of per-step mean losses since the last reset
  unsigned long long loss_steps;
  float last_loss;
  unsigned int adam_done;     // CTAs of k_adam finished with the step
  unsigned int error;         // a bounded wait gave up (the step is dropped)
  unsigned int lost_wait_us;  // fault injection: see SceneDev::lost_wait_us
};

enum class Src { kExplicit, kScene };

struct TrainArgs {
  const uint16_t* p16;  // fp16 operand copy of the parameters
  float* grad;          // kParams fp32 gradient sums (zeroed by k_adam)
  StepState* st;
  // explicit samples (gradient checks)
  const uint4* ex_lat;  // count x 16 halves
  const float* ex_dir;  // count x 3
  const float* ex_tgt;  // count x 3
  float* ex_glat;       // count x 16: d loss_sum / d latent (scaled by kLossScale)
  float* ex_out;        // count x 3
  double* ex_loss;      // sum of squared errors
  uint32_t ex_count;
  // scene samples
  const float* color;   // FP32 scene: 3 planes of n
  const float* sh;      // FP32 scene: rest*3 planes of n
  const uint16_t* sh16; // FP16 scene: (rest+1)*3 planes of n halves
  const float4* shs;    // the same coefficients splat-major: base colour, then
                        // the rest (RGB innermost), padded to sh_row4 float4
  uint32_t sh_row4;
  uint64_t n;
  const float4* dirs;
  uint32_t n_dirs;
  const uint4* lat16;   // n x 16 halves
  float* lat_grad;      // n x 16
  uint64_t samples;     // n * n_dirs
  uint64_t seed;
  uint32_t bits;
  uint32_t batch;
  uint32_t steps_per_epoch;
  uint32_t tiles;       // tiles per step
};

__device__ __forceinline__ uint64_t epoch_key(uint64_t seed, uint64_t epoch) {
  return seed * 0x9E3779B97F4A7C15ull + epoch * 0xD1B54A32D192ED03ull + 1;
}

// Float4s per splat-major coefficient row of SH degree DEG.
template <int DEG>
__host__ __device__ constexpr uint32_t sh_row4() {
  return ((DEG + 1) * (DEG + 1) * 3 + 3) / 4;
}

// Exact SH colour of a splat whose coefficient row is `row` (base colour,
// then the rest coefficients, RGB innermost) at unit direction d, clamped
// to [0, 1].
template <int DEG>
__device__ __forceinline__ void sh_target(const float* row, float dx, float dy, float dz, float c[3]) {
  c[0] = row[0];
  c[1] = row[1];
  c[2] = row[2];
  sh::eval_sh<DEG>([&](int coef, int ch) { return row[3 + 3 * coef + ch]; }, dx, dy, dz, c);
  for (int ch = 0; ch < 3; ch++) c[ch] = fminf(fmaxf(c[ch], 0.0f), 1.0f);
}

// The splat-major coefficient rows from the scene's planes.
__global__ void k_pack_sh(const float* __restrict__ color, const float* __restrict__ sh,
                          const uint16_t* __restrict__ sh16, uint64_t n, uint32_t coefs, uint32_t row4,
                          float* __restrict__ out) {
  for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n * row4 * 4;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s = q / (row4 * 4);
    const uint32_t c = (uint32_t)(q % (row4 * 4));
    float v = 0.0f;
    if (c < coefs) {
      if (sh16)
        v = __half2float(__ushort_as_half(sh16[(uint64_t)c * n + s]));
      else
        v = c < 3 ? color[(uint64_t)c * n + s] : sh[(uint64_t)(c - 3) * n + s];
    }
    out[q] = v;
  }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

// Stores 64 values (TMEM columns [col, col + 64) of this row, times a 0/1
// mask) as fp16 into chunks [chunk0, chunk0 + 8) of tile `t`.
__device__ __forceinline__ void masked_epilogue(uint32_t tmem, uint32_t col, uint64_t mask, uint16_t* t,
                                                uint32_t chunk0, uint32_t r) {
#pragma unroll
  for (uint32_t q = 0; q < 4; q++) {
    float v[16];
    umma::tmem_ld16(umma::tmem_warp_addr(tmem, col + 16 * q), v);
    float a[8], b[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      a[j] = ((mask >> (16 * q + j)) & 1ull) ? v[j] : 0.0f;
      b[j] = ((mask >> (16 * q + 8 + j)) & 1ull) ? v[8 + j] : 0.0f;
    }
    mlp::store_chunk(t, r, chunk0 + 2 * q, a);
    mlp::store_chunk(t, r, chunk0 + 2 * q + 1, b);
  }
}

// dst (out_rows x k_count, feature-chunked) = the transpose of the first
// out_rows columns of src (src_rows x >= out_rows, feature-chunked), both
// in shared memory: dst row n, column k = src row k, column n.
__device__ __forceinline__ void transpose_tile(uint16_t* dst, const uint16_t* src, uint32_t src_rows,
                                               uint32_t out_rows, uint32_t k_count) {
  const uint8_t* sb = reinterpret_cast<const uint8_t*>(src);
  for (uint32_t q = threadIdx.x; q < out_rows * k_count / 8; q += blockDim.x) {
    const uint32_t n = q % out_rows, k = (q / out_rows) * 8;
    uint16_t v[8];
#pragma unroll
    for (int j = 0; j < 8; j++)
      v[j] = *reinterpret_cast<const uint16_t*>(sb + umma::chunked_offset(k + j, n, src_rows));
    uint4 u;
    u.x = v[0] | ((uint32_t)v[1] << 16);
    u.y = v[2] | ((uint32_t)v[3] << 16);
    u.z = v[4] | ((uint32_t)v[5] << 16);
    u.w = v[6] | ((uint32_t)v[7] << 16);
    *reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(dst) + umma::chunked_offset(n, k, out_rows)) = u;
  }
}

template <Src SRC, int DEG>
__global__ void __launch_bounds__(kTrainThreads) k_train(TrainArgs a) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
  const uint32_t tid = threadIdx.x;

  // Parameters into the operand tiles (forward and transposed copies).
  mlp::load_rows(S.w1f, a.p16 + mlp::kW1, 64, 32);
  mlp::load_rows(S.w2f, a.p16 + mlp::kW2, 64, 64);
  for (uint32_t i = tid; i < 3 * 64; i += kTrainThreads)
    S.w3[i / 64][i % 64] = __half2float(__ushort_as_half(a.p16[mlp::kW3 + i]));
  __syncthreads();
  // The transposed operands of the backward pass, from the forward tiles.
  transpose_tile(S.w2b, S.w2f, 64, 64, 64);
  transpose_tile(S.w1b, S.w1f, 64, 16, 64);
  if (tid < 64) S.b2[tid] = __half2float(__ushort_as_half(a.p16[mlp::kB2 + tid]));
  if (tid < 16) {
    S.b3[tid] = __half2float(__ushort_as_half(a.p16[mlp::kB3 + tid]));
    S.db3[tid] = 0.0f;
  }
  if (tid == 0) {
    umma::mbar_init(umma::smem_u32(&S.mbar), 1);
    umma::mbar_init(umma::smem_u32(&S.lost), 1);
  }
  if (tid < 32) umma::tmem_alloc(&S.tmem, kTrainTmemCols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = S.tmem;
  const uint32_t mbar = umma::smem_u32(&S.mbar);
  const uint32_t sR = umma::smem_u32(S.R), sQ = umma::smem_u32(S.Q), sD3 = umma::smem_u32(S.D3);

  // Step bookkeeping (scene samples).
  uint64_t step = 0, base = 0, key = 0;
  if (SRC == Src::kScene) {
    step = *reinterpret_cast<volatile unsigned long long*>(&a.st->step);
    const uint64_t k = step % a.steps_per_epoch;
    base = k * a.batch;
    key = epoch_key(a.seed, step / a.steps_per_epoch);
  }

  uint32_t phase = 0;
  bool timed_out = false, aborted = false, inflight = false;
  float loss = 0.0f;
  // Fault injection (tests of the timeout path): the first wait also waits
  // for a completion that never arrives, for at most lost_wait_us.
  uint64_t lost_ns = 1000ull * *reinterpret_cast<volatile unsigned int*>(&a.st->lost_wait_us);
  // Waits for the MMAs committed to `mbar`; after a wait that gave up, the
  // phase stays the one still in flight, which the exit path waits for.
  auto wait_mma = [&]() {
    if (umma::mbar_wait(mbar, phase)) {
      phase ^= 1u;
      inflight = false;
    } else {
      timed_out = true;
    }
    if (lost_ns) {
      if (!umma::mbar_wait(umma::smem_u32(&S.lost), 0, lost_ns)) timed_out = true;
      lost_ns = 0;
    }
    umma::fence_after_sync();
  };
  auto sync_or_abort = [&]() -> bool {
    umma::fence_async_smem();
    umma::fence_before_sync();
    return __syncthreads_or(timed_out) != 0;
  };

  bool first = true;
  for (uint32_t tile = blockIdx.x; tile < a.tiles; tile += gridDim.x) {
    // ---- inputs of row tid -------------------------------------------------
    const uint64_t j = (uint64_t)tile * mlp::kRows + tid;
    bool active;
    uint64_t splat = 0;
    uint4 l0 = make_uint4(0, 0, 0, 0), l1 = l0;
    float d[3] = {0.f, 0.f, 0.f}, tgt[3] = {0.f, 0.f, 0.f};
    constexpr uint32_t R4 = sh_row4<DEG>();
    float4 row4[R4];  // the splat's coefficients: loads in flight during the forward pass
    if (SRC == Src::kExplicit) {
      active = j < a.ex_count;
      if (active) {
        l0 = __ldg(a.ex_lat + 2 * j);
        l1 = __ldg(a.ex_lat + 2 * j + 1);
        for (int c = 0; c < 3; c++) {
          d[c] = __ldg(a.ex_dir + 3 * j + c);
          tgt[c] = __ldg(a.ex_tgt + 3 * j + c);
        }
      }
    } else {
      active = j < a.batch && base + j < a.samples;
      if (active) {
        const uint64_t p = mlp::shuffle_index(base + j, a.samples, key, a.bits);
        splat = p / a.n_dirs;
        const float4 dv = __ldg(a.dirs + (p % a.n_dirs));
        d[0] = dv.x;
        d[1] = dv.y;
        d[2] = dv.z;
        l0 = __ldg(a.lat16 + 2 * splat);
        l1 = __ldg(a.lat16 + 2 * splat + 1);
        const float4* src = a.shs + splat * R4;
#pragma unroll
        for (uint32_t q = 0; q < R4; q++) row4[q] = __ldg(src + q);
      }
    }
    mlp::store_input(S.R, 8, tid, l0, l1, d[0], d[1], d[2]);
    if (sync_or_abort()) { aborted = true; break; }

    // ---- forward -------------------------------------------------------------
    if (tid == 0) {
      umma::fence_after_sync();
      mlp::gemm_k(tmem + kTS, sR, 8, umma::smem_u32(S.w1f), 64, 2, mlp::kIdN64);
      umma::commit(mbar);
    }
    inflight = true;
    wait_mma();
    const uint64_t mask1 = mlp::hidden_epilogue(tmem, kTS, nullptr, S.R, tid);
    if (sync_or_abort()) { aborted = true; break; }
    if (tid == 0) {
      umma::fence_after_sync();
      mlp::gemm_k(tmem + kTS, sR, 0, umma::smem_u32(S.w2f), 64, 4, mlp::kIdN64);
      umma::commit(mbar);
    }
    inflight = true;
    wait_mma();
    // Layer 2's epilogue with layer 3 and its backward on the CUDA cores:
    // h2 = fp16(relu(z2 + b2)) to Q chunks 0-7, z3 = W3 h2 + b3, rgb, loss,
    // dz3 (fp16) to D3, dh2 = W3^T dz3, dz2 = dh2 masked by h2 > 0 to Q 8-15.
    if (SRC == Src::kScene && active) sh_target<DEG>(reinterpret_cast<const float*>(row4), d[0], d[1], d[2], tgt);
    {
      uint64_t mask2 = 0;
      float z3[3] = {S.b3[0], S.b3[1], S.b3[2]};
#pragma unroll
      for (uint32_t q = 0; q < 4; q++) {
        float v[16];
        umma::tmem_ld16(umma::tmem_warp_addr(tmem, kTS + 16 * q), v);
#pragma unroll
        for (int k = 0; k < 16; k++) {
          const uint32_t c = 16 * q + k;
          v[k] = __half2float(__float2half_rn(fmaxf(v[k] + S.b2[c], 0.0f)));
          if (v[k] > 0.0f) mask2 |= 1ull << c;
          z3[0] = fmaf(S.w3[0][c], v[k], z3[0]);
          z3[1] = fmaf(S.w3[1][c], v[k], z3[1]);
          z3[2] = fmaf(S.w3[2][c], v[k], z3[2]);
        }
        float lo[8], hi[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
          lo[k] = v[k];
          hi[k] = v[8 + k];
        }
        mlp::store_chunk(S.Q, tid, 2 * q, lo);
        mlp::store_chunk(S.Q, tid, 2 * q + 1, hi);
      }
      float dz[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      float y[3];
      for (int c = 0; c < 3; c++) {
        y[c] = mlp::sigmoidf(z3[c]);
        if (active) {
          const float e = y[c] - tgt[c];
          loss += e * e;
          dz[c] = kLossScale * (2.0f / 3.0f) * e * (y[c] * (1.0f - y[c]));
        }
      }
      if (SRC == Src::kExplicit && active)
        for (int c = 0; c < 3; c++) a.ex_out[3 * j + c] = y[c];
      // The GEMMs and the bias gradient use the fp16-rounded dz3.
      for (int c = 0; c < 3; c++) {
        dz[c] = __half2float(__float2half_rn(dz[c]));
        const float s3 = warp_sum(dz[c]);
        if ((tid & 31) == 0) atomicAdd(&S.db3[c], s3);
      }
      mlp::store_chunk(S.D3, tid, 0, dz);
      const float zero[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      mlp::store_chunk(S.D3, tid, 1, zero);
#pragma unroll
      for (uint32_t q = 0; q < 8; q++) {
        float g8[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const uint32_t c = 8 * q + k;
          const float dh = fmaf(dz[2], S.w3[2][c], fmaf(dz[1], S.w3[1][c], dz[0] * S.w3[0][c]));
          g8[k] = ((mask2 >> c) & 1ull) ? dh : 0.0f;
        }
        mlp::store_chunk(S.Q, tid, 8 + q, g8);
      }
    }
    if (sync_or_abort()) { aborted = true; break; }
    if (tid == 0) {
      umma::fence_after_sync();
      mlp::gemm_k(tmem + kTS, sQ, 8, umma::smem_u32(S.w2b), 64, 4, mlp::kIdN64);  // dh1 = dz2 W2
      for (uint32_t s = 0; s < 8; s++)  // [h2 | dz2]^T dz3 over the tile's samples
        umma::mma(tmem + kTW3, umma::desc_mnmajor(sQ, mlp::kRows, 0, 16 * s),
                  umma::desc_mnmajor(sD3, mlp::kRows, 0, 16 * s), mlp::kIdWgN16, (first && s == 0) ? 0u : 1u);
      umma::commit(mbar);
    }
    inflight = true;
    wait_mma();
    masked_epilogue(tmem, kTS, mask1, S.Q, 16, tid);  // dz1
    if (sync_or_abort()) { aborted = true; break; }
    if (tid == 0) {
      umma::fence_after_sync();
      mlp::gemm_k(tmem + kTZ, sQ, 16, umma::smem_u32(S.w1b), 16, 4, mlp::kIdN16);  // dx = dz1 W1 (latent part)
      for (uint32_t s = 0; s < 8; s++)  // [dz2 | dz1]^T [h1 | x]
        umma::mma(tmem + kTW, umma::desc_mnmajor(sQ, mlp::kRows, 8, 16 * s),
                  umma::desc_mnmajor(sR, mlp::kRows, 0, 16 * s), mlp::kIdWgN96, (first && s == 0) ? 0u : 1u);
      umma::commit(mbar);
    }
    inflight = true;
    wait_mma();
    {
      float g[16];
      umma::tmem_ld16(umma::tmem_warp_addr(tmem, kTZ), g);
      if (active) {
        if (SRC == Src::kExplicit) {
          float4* o = reinterpret_cast<float4*>(a.ex_glat + 16 * j);
          for (int q = 0; q < 4; q++) o[q] = make_float4(g[4 * q], g[4 * q + 1], g[4 * q + 2], g[4 * q + 3]);
        } else {
          float4* o = reinterpret_cast<float4*>(a.lat_grad + 16 * splat);
          for (int q = 0; q < 4; q++) atomicAdd(o + q, make_float4(g[4 * q], g[4 * q + 1], g[4 * q + 2], g[4 * q + 3]));
        }
      }
    }
    first = false;
  }
  if (!aborted && __syncthreads_or(timed_out)) aborted = true;

  // ---- this CTA's weight gradients -------------------------------------------
  if (!aborted && !first) {
    umma::fence_after_sync();
    const uint32_t w = tid >> 5;
    float v[16];
    if (w < 2) {  // rows 0-63 of kTW: dW2[o = tid], db2 (column 64 + 19 = 83)
      float* gw2 = a.grad + mlp::kW2 + 64 * tid;
      for (uint32_t q = 0; q < 4; q++) {
        umma::tmem_ld16(umma::tmem_warp_addr(tmem, kTW + 16 * q), v);
        for (int c = 0; c < 4; c++)
          atomicAdd(reinterpret_cast<float4*>(gw2 + 16 * q + 4 * c),
                    make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]));
      }
      umma::tmem_ld16(umma::tmem_warp_addr(tmem, kTW + 80), v);
      atomicAdd(a.grad + mlp::kB2 + tid, v[3]);
      umma::tmem_ld16(umma::tmem_warp_addr(tmem, kTW3), v);  // dW3^T[i = tid][o]
      for (int o = 0; o < 3; o++) atomicAdd(a.grad + mlp::kW3 + 64 * o + tid, v[o]);
    } else {  // rows 64-127: dW1[o = tid - 64], columns 64-95
      float* gw1 = a.grad + mlp::kW1 + 32 * (tid - 64);
      for (uint32_t q = 0; q < 2; q++) {
        umma::tmem_ld16(umma::tmem_warp_addr(tmem, kTW + 64 + 16 * q), v);
        for (int c = 0; c < 4; c++)
          atomicAdd(reinterpret_cast<float4*>(gw1 + 16 * q + 4 * c),
                    make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]));
      }
    }
    if (tid < 3) atomicAdd(a.grad + mlp::kB3 + tid, S.db3[tid]);
    const float ls = warp_sum(loss);
    if ((tid & 31) == 0 && ls != 0.0f) atomicAdd(SRC == Src::kExplicit ? a.ex_loss : &a.st->loss_step, (double)ls);
  }
  if (aborted) {
    if (tid == 0) atomicExch(&a.st->error, 1u);
    if (inflight) umma::mbar_wait(mbar, phase, 100000000ull);  // the MMAs still in flight
  }
  umma::fence_before_sync();
  __syncthreads();
  if (tid < 32) {
    umma::fence_after_sync();
    umma::tmem_free(tmem, kTrainTmemCols);
  }
}

struct AdamArgs {
  float lr, b1, b2, eps;
  uint32_t batch, steps_per_epoch;
  uint64_t samples;
  // the step's sample order (for the latent rows it touched)
  uint64_t seed;
  uint32_t bits, n_dirs;
};

__device__ __forceinline__ float adam_update(float& m, float& v, float g, float lr, float b1, float b2, float eps,
                                             float c1, float c2) {
  m = b1 * m + (1.0f - b1) * g;
  v = b2 * v + (1.0f - b2) * g * g;
  const float mh = m / c1, vh = v / c2;
  return lr * mh / (sqrtf(vh) + eps);
}

constexpr uint32_t kAdamThreads = 256;
constexpr uint32_t kAdamParamCtas = (mlp::kParams + kAdamThreads - 1) / kAdamThreads;

// One launch after each training step. CTAs [0, kAdamParamCtas) apply Adam
// to the fp32 master parameters and refresh their fp16 copy; the others
// apply lazy Adam to the latent rows the step touched: one thread per
// sample of the step recomputes its splat from the epoch's shuffle, and the
// first thread to stamp the row with the step (step + 1) updates it (16
// elements as float4s), so a row sampled twice is updated once with its
// summed gradient. The last CTA to finish closes the step: records its loss
// and advances the step counter.
__global__ void __launch_bounds__(kAdamThreads) k_adam(float* __restrict__ p32, float* __restrict__ pm,
                                                       float* __restrict__ pv, uint16_t* __restrict__ p16,
                                                       float* __restrict__ grad, float* __restrict__ lat32,
                                                       float* __restrict__ lm, float* __restrict__ lv,
                                                       uint16_t* __restrict__ lat16, float* __restrict__ lat_grad,
                                                       uint32_t* __restrict__ stamp, StepState* st, AdamArgs a) {
  const uint64_t step = *reinterpret_cast<volatile unsigned long long*>(&st->step);
  const uint64_t k = step % a.steps_per_epoch;
  const uint64_t active = min((uint64_t)a.batch, a.samples - k * a.batch);
  const float inv = 1.0f / (kLossScale * (float)active);
  const float t = (float)(step + 1);
  const float c1 = 1.0f - powf(a.b1, t), c2 = 1.0f - powf(a.b2, t);
  // A step whose training kernel gave up on a wait is dropped: its partial
  // gradients are cleared and nothing is updated or counted.
  const bool dropped = *reinterpret_cast<volatile unsigned int*>(&st->error) != 0u;
  if (dropped) {
    if (blockIdx.x < kAdamParamCtas) {
      const uint32_t i = blockIdx.x * kAdamThreads + threadIdx.x;
      if (i < mlp::kParams) grad[i] = 0.0f;
    } else {
      const uint64_t key = epoch_key(a.seed, step / a.steps_per_epoch);
      for (uint32_t q = (blockIdx.x - kAdamParamCtas) * kAdamThreads + threadIdx.x; q < active;
           q += (gridDim.x - kAdamParamCtas) * kAdamThreads) {
        const uint64_t splat = mlp::shuffle_index(k * a.batch + q, a.samples, key, a.bits) / a.n_dirs;
        float4* g4 = reinterpret_cast<float4*>(lat_grad + splat * 16);
        for (int c = 0; c < 4; c++) g4[c] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  } else if (blockIdx.x < kAdamParamCtas) {
    const uint32_t i = blockIdx.x * kAdamThreads + threadIdx.x;
    if (i < mlp::kParams) {
      const float g = grad[i] * inv;
      grad[i] = 0.0f;
      float m = pm[i], v = pv[i];
      const float p = p32[i] - adam_update(m, v, g, a.lr, a.b1, a.b2, a.eps, c1, c2);
      pm[i] = m;
      pv[i] = v;
      p32[i] = p;
      p16[i] = __half_as_ushort(__float2half_rn(p));
    }
  } else {
    const uint64_t key = epoch_key(a.seed, step / a.steps_per_epoch);
    const uint32_t tag = (uint32_t)(step + 1);
    for (uint32_t q = (blockIdx.x - kAdamParamCtas) * kAdamThreads + threadIdx.x; q < active;
         q += (gridDim.x - kAdamParamCtas) * kAdamThreads) {
      const uint64_t splat = mlp::shuffle_index(k * a.batch + q, a.samples, key, a.bits) / a.n_dirs;
      if (atomicExch(stamp + splat, tag) == tag) continue;  // another sample of the row updates it
      const uint64_t row = splat * 16;
      float4* g4 = reinterpret_cast<float4*>(lat_grad + row);
      float4* m4 = reinterpret_cast<float4*>(lm + row);
      float4* v4 = reinterpret_cast<float4*>(lv + row);
      float4* p4 = reinterpret_cast<float4*>(lat32 + row);
      float4 g[4], m[4], v[4], p[4];
#pragma unroll
      for (int c = 0; c < 4; c++) {
        g[c] = g4[c];
        m[c] = m4[c];
        v[c] = v4[c];
        p[c] = p4[c];
      }
      uint32_t h[8];
#pragma unroll
      for (int c = 0; c < 4; c++) {
        float* gg = &g[c].x;
        float* mm = &m[c].x;
        float* vv = &v[c].x;
        float* pp = &p[c].x;
#pragma unroll
        for (int e = 0; e < 4; e++) pp[e] -= adam_update(mm[e], vv[e], gg[e] * inv, a.lr, a.b1, a.b2, a.eps, c1, c2);
        h[2 * c] = mlp::pack_half2(p[c].x, p[c].y);
        h[2 * c + 1] = mlp::pack_half2(p[c].z, p[c].w);
        g4[c] = make_float4(0.f, 0.f, 0.f, 0.f);
        m4[c] = m[c];
        v4[c] = v[c];
        p4[c] = p[c];
      }
      uint4* o = reinterpret_cast<uint4*>(lat16 + row);
      o[0] = make_uint4(h[0], h[1], h[2], h[3]);
      o[1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
  }
  // The last CTA closes the step.
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&st->adam_done, 1u) == gridDim.x - 1) {
      __threadfence();
      if (dropped) {
        st->loss_step = 0.0;
        st->adam_done = 0;
        return;
      }
      const double ls = *reinterpret_cast<volatile double*>(&st->loss_step) / (3.0 * (double)active);
      st->loss_step = 0.0;
      st->loss_sum += ls;
      st->loss_steps += 1;
      st->last_loss = (float)ls;
      st->adam_done = 0;
      __threadfence();
      st->step = step + 1;
    }
  }
}

__global__ void k_to_half(const float* __restrict__ src, uint16_t* __restrict__ dst, uint64_t count) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = __half_as_ushort(__float2half_rn(src[i]));
}

// Latent initialisation: a fixed Gaussian random projection of the splat's
// centred colour coefficients (base colour - 0.5, then the SH rest), so the
// latents start out distinct and informative; training takes it from there.
__global__ void k_init_latents(TrainArgs a, uint32_t sh_degree, const float* __restrict__ proj, float* __restrict__ lat32,
                               uint16_t* __restrict__ lat16) {
  const uint32_t coefs = (sh_degree + 1) * (sh_degree + 1) * 3;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < a.n; s += (uint64_t)gridDim.x * blockDim.x) {
    float z[16];
    for (int k = 0; k < 16; k++) z[k] = 0.0f;
    for (uint32_t c = 0; c < coefs; c++) {
      float x;
      if (a.sh16)
        x = __half2float(__ushort_as_half(__ldg(a.sh16 + (uint64_t)c * a.n + s)));
      else
        x = c < 3 ? __ldg(a.color + (uint64_t)c * a.n + s) : __ldg(a.sh + (uint64_t)(c - 3) * a.n + s);
      if (c < 3) x -= 0.5f;
      for (int k = 0; k < 16; k++) z[k] += __ldg(proj + c * 16 + k) * x;
    }
    for (int k = 0; k < 16; k++) {
      lat32[s * 16 + k] = z[k];
      lat16[s * 16 + k] = __half_as_ushort(__float2half_rn(z[k]));
    }
  }
}

template <Src SRC>
cudaError_t launch_train(const TrainArgs& a, uint32_t grid, uint32_t sh_degree, cudaStream_t s) {
  const size_t smem = sizeof(TrainSmem);
  cudaError_t e = cudaSuccess;
#define SPLAT_TRAIN(D)                                                                                   \
  do {                                                                                                   \
    e = cudaFuncSetAttribute(k_train<SRC, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
    if (e == cudaSuccess) k_train<SRC, D><<<grid, kTrainThreads, smem, s>>>(a);                          \
  } while (0)
  if constexpr (SRC == Src::kExplicit) {
    SPLAT_TRAIN(0);
  } else {
    switch (sh_degree) {
      case 0: SPLAT_TRAIN(0); break;
      case 1: SPLAT_TRAIN(1); break;
      case 2: SPLAT_TRAIN(2); break;
      default: SPLAT_TRAIN(3); break;
    }
  }
#undef SPLAT_TRAIN
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

// SplitMix64 (the reference's generator, src/gen.rs:22-54) for host-side
// initial values.
struct SplitMix {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {
    const double u1 = std::max(uniform(), 1e-300), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

thread_local std::string g_learner_error;

}  // namespace

struct splat_cuda_learner {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  uint64_t n = 0;
  uint32_t sh_degree = 0;
  uint32_t n_dirs = 256;
  uint32_t batch = 65536;
  uint32_t steps_per_epoch = 1;
  uint32_t grid = 1;
  uint64_t samples = 0;
  uint32_t bits = 1;
  uint64_t seed = 0;
  AdamArgs adam{};
  TrainArgs args{};
  float *p32 = nullptr, *pm = nullptr, *pv = nullptr, *grad = nullptr;
  uint16_t* p16 = nullptr;
  float *lat32 = nullptr, *lm = nullptr, *lv = nullptr, *lgrad = nullptr;
  uint16_t* lat16 = nullptr;
  uint32_t* stamp = nullptr;
  float4* dirs = nullptr;
  float* shs = nullptr;
  StepState* st = nullptr;
  cudaGraphExec_t graph = nullptr;  // kGraphSteps steps
  uint32_t launches = 0;
  uint32_t inject_lost_us = 0;  // SPLAT_FAULT_LOST_WAIT for the next call
  std::string err;
};

namespace {

constexpr uint32_t kGraphSteps = 16;

int lfail(splat_cuda_learner* L, int code, const std::string& msg) {
  L->err = msg;
  return code;
}
int lcuda(splat_cuda_learner* L, cudaError_t e, const char* what) {
  return lfail(L, e == cudaErrorMemoryAllocation ? SPLAT_ERR_OOM : SPLAT_ERR_DEVICE,
               std::string(what) + ": " + cudaGetErrorString(e));
}
#define LCK(expr, what)                               \
  do {                                                \
    cudaError_t e_ = (expr);                          \
    if (e_ != cudaSuccess) return lcuda(L, e_, what); \
  } while (0)

void enqueue_adam(splat_cuda_learner* L, cudaStream_t s) {
  const uint32_t lat_ctas = std::max(1u, std::min((L->batch + kAdamThreads - 1) / kAdamThreads, 4u * L->num_sms));
  k_adam<<<kAdamParamCtas + lat_ctas, kAdamThreads, 0, s>>>(L->p32, L->pm, L->pv, L->p16, L->grad, L->lat32, L->lm,
                                                             L->lv, L->lat16, L->lgrad, L->stamp, L->st, L->adam);
}

// One step: train, then Adam on the parameters and the touched latents.
cudaError_t enqueue_step(splat_cuda_learner* L, cudaStream_t s) {
  cudaError_t e = launch_train<Src::kScene>(L->args, L->grid, L->sh_degree, s);
  if (e != cudaSuccess) return e;
  enqueue_adam(L, s);
  L->launches += 2;
  return cudaGetLastError();
}

// Waits for the learner's stream and reads the step state. A step whose
// training kernel gave up on a wait was dropped (k_adam); the error is
// reported once and cleared, so that the next call trains again. An
// injected lost completion fires for one call only.
int sync_state(splat_cuda_learner* L, StepState* out) {
  LCK(cudaStreamSynchronize(L->stream), "training step");
  LCK(cudaMemcpy(out, L->st, sizeof(StepState), cudaMemcpyDeviceToHost), "read step state");
  if (out->lost_wait_us || out->error) {
    LCK(cudaMemsetAsync(&L->st->error, 0, 2 * sizeof(unsigned int), L->stream), "clear step error");
    LCK(cudaStreamSynchronize(L->stream), "clear step error");
  }
  if (out->error) return lfail(L, SPLAT_ERR_TIMEOUT, "a tensor-core wait in the training kernel gave up");
  return SPLAT_OK;
}

}  // namespace

SPLAT_API const char* splat_cuda_learner_create_error(void) { return g_learner_error.c_str(); }

SPLAT_API int splat_cuda_learner_create(const splat_cuda_handle* h, const splat_learn_config* cfg,
                                        splat_cuda_learner** out) {
  g_learner_error.clear();
  if (!out) return SPLAT_ERR_INVALID_ARG;
  *out = nullptr;
  if (!h || !cfg) {
    g_learner_error = "null scene or config";
    return SPLAT_ERR_INVALID_ARG;
  }
  if (h->lat16 || (!h->sh && !h->color && !h->sh16) || h->n == 0) {
    g_learner_error = "the scene must be a non-empty SH scene";
    return SPLAT_ERR_INVALID_ARG;
  }
  if (cfg->directions == 0 || cfg->batch == 0 || cfg->batch % mlp::kRows != 0 || cfg->batch > (1u << 22)) {
    g_learner_error = "directions must be > 0 and batch a multiple of 128 up to 2^22";
    return SPLAT_ERR_INVALID_ARG;
  }
  auto* L = new splat_cuda_learner();
  auto bail = [&](int rc) {
    g_learner_error = L->err;
    splat_cuda_learner_destroy(L);
    return rc;
  };
  L->device = h->device;
  L->n = h->n;
  L->sh_degree = h->sh_degree;
  L->n_dirs = cfg->directions;
  L->batch = cfg->batch;
  L->samples = L->n * L->n_dirs;
  L->steps_per_epoch = (uint32_t)((L->samples + L->batch - 1) / L->batch);
  L->bits = 1;
  while ((1ull << L->bits) < L->samples) L->bits++;
  L->seed = cfg->seed;
  L->adam = AdamArgs{cfg->lr, cfg->beta1, cfg->beta2, cfg->eps, L->batch, L->steps_per_epoch, L->samples,
                     L->seed, L->bits, L->n_dirs};
  cudaError_t e = cudaSetDevice(L->device);
  if (e != cudaSuccess) return bail(lcuda(L, e, "cudaSetDevice"));
  if ((e = cudaDeviceGetAttribute(&L->num_sms, cudaDevAttrMultiProcessorCount, L->device)) != cudaSuccess)
    return bail(lcuda(L, e, "device attributes"));
  if ((e = cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(lcuda(L, e, "cudaStreamCreate"));
  const uint32_t tiles = L->batch / mlp::kRows;
  const uint32_t slots = 2u * (uint32_t)L->num_sms;  // two CTAs per SM (TMEM: 256 columns each)
  const uint32_t per = (tiles + slots - 1) / slots;
  L->grid = (tiles + per - 1) / per;
  const uint64_t nl = L->n * 16;
  // Zeroed on the learner's own stream: it is non-blocking, so a memset on
  // the legacy stream could still land after the packing kernel and the
  // uploads below have written these buffers.
  auto dalloc = [&](void** p, size_t bytes, const char* what) -> int {
    cudaError_t er = cudaMalloc(p, bytes);
    if (er != cudaSuccess) return lcuda(L, er, what);
    er = cudaMemsetAsync(*p, 0, bytes, L->stream);
    if (er != cudaSuccess) return lcuda(L, er, what);
    return SPLAT_OK;
  };
  int rc;
  if ((rc = dalloc((void**)&L->p32, mlp::kParams * 4, "parameters")) ||
      (rc = dalloc((void**)&L->pm, mlp::kParams * 4, "parameters")) ||
      (rc = dalloc((void**)&L->pv, mlp::kParams * 4, "parameters")) ||
      (rc = dalloc((void**)&L->grad, mlp::kParams * 4, "parameters")) ||
      (rc = dalloc((void**)&L->p16, mlp::kParams * 2, "parameters")) ||
      (rc = dalloc((void**)&L->lat32, nl * 4, "latents")) || (rc = dalloc((void**)&L->lm, nl * 4, "latents")) ||
      (rc = dalloc((void**)&L->lv, nl * 4, "latents")) || (rc = dalloc((void**)&L->lgrad, nl * 4, "latents")) ||
      (rc = dalloc((void**)&L->lat16, nl * 2, "latents")) || (rc = dalloc((void**)&L->stamp, L->n * 4, "latents")) ||
      (rc = dalloc((void**)&L->dirs, (size_t)L->n_dirs * sizeof(float4), "directions")) ||
      (rc = dalloc((void**)&L->shs,
                   (size_t)L->n * (((L->sh_degree + 1) * (L->sh_degree + 1) * 3 + 3) / 4) * sizeof(float4),
                   "coefficient rows")) ||
      (rc = dalloc((void**)&L->st, sizeof(StepState), "state")))
    return bail(rc);

  // Fibonacci-sphere directions (the construction of src/gen.rs:213-219):
  // y = 1 - 2 (i + 0.5) / n, radius sqrt(1 - y^2), angle i * pi (3 - sqrt 5).
  std::vector<float4> dirs(L->n_dirs);
  const double golden = 3.14159265358979323846 * (3.0 - std::sqrt(5.0));
  for (uint32_t i = 0; i < L->n_dirs; i++) {
    const double y = 1.0 - 2.0 * (i + 0.5) / L->n_dirs;
    const double r = std::sqrt(std::max(0.0, 1.0 - y * y));
    const double th = golden * i;
    dirs[i] = make_float4((float)(r * std::cos(th)), (float)y, (float)(r * std::sin(th)), 0.0f);
  }
  // Uploads go on the learner's stream (which does not wait for the legacy
  // stream that a plain cudaMemcpy from pageable memory may still be using).
  if ((e = cudaMemcpyAsync(L->dirs, dirs.data(), dirs.size() * sizeof(float4), cudaMemcpyHostToDevice, L->stream)) !=
      cudaSuccess)
    return bail(lcuda(L, e, "upload directions"));

  TrainArgs& a = L->args;
  a.p16 = L->p16;
  a.grad = L->grad;
  a.st = L->st;
  if (h->precision == SPLAT_PRECISION_FP16) {
    a.sh16 = h->sh16;
  } else {
    a.color = h->color;
    a.sh = h->sh;
  }
  a.n = L->n;
  a.shs = reinterpret_cast<const float4*>(L->shs);
  a.sh_row4 = ((L->sh_degree + 1) * (L->sh_degree + 1) * 3 + 3) / 4;
  {
    const uint32_t coefs = (L->sh_degree + 1) * (L->sh_degree + 1) * 3;
    k_pack_sh<<<(uint32_t)std::min<uint64_t>((L->n * a.sh_row4 * 4 + 255) / 256, 8192), 256, 0, L->stream>>>(
        a.color, a.sh, a.sh16, L->n, coefs, a.sh_row4, L->shs);
    if ((e = cudaGetLastError()) != cudaSuccess) return bail(lcuda(L, e, "coefficient rows"));
  }
  a.dirs = L->dirs;
  a.n_dirs = L->n_dirs;
  a.lat16 = reinterpret_cast<const uint4*>(L->lat16);
  a.lat_grad = L->lgrad;
  a.samples = L->samples;
  a.seed = L->seed;
  a.bits = L->bits;
  a.batch = L->batch;
  a.steps_per_epoch = L->steps_per_epoch;
  a.tiles = tiles;

  // Initial parameters: He-uniform hidden layers, Xavier-uniform output,
  // zero biases; latents from a random projection of the colour coefficients.
  SplitMix rng{cfg->seed ^ 0x5EEDBA5Eull};
  std::vector<float> p(mlp::kParams, 0.0f);
  const double l1 = std::sqrt(6.0 / 20.0), l2 = std::sqrt(6.0 / 64.0), l3 = std::sqrt(6.0 / (64.0 + 3.0));
  for (uint32_t o = 0; o < 64; o++)
    for (uint32_t i = 0; i < 19; i++) p[mlp::kW1 + o * 32 + i] = (float)((2.0 * rng.uniform() - 1.0) * l1);
  for (uint32_t q = 0; q < 64 * 64; q++) p[mlp::kW2 + q] = (float)((2.0 * rng.uniform() - 1.0) * l2);
  for (uint32_t o = 0; o < 3; o++)
    for (uint32_t i = 0; i < 64; i++) p[mlp::kW3 + o * 64 + i] = (float)((2.0 * rng.uniform() - 1.0) * l3);
  const uint32_t coefs = (L->sh_degree + 1) * (L->sh_degree + 1) * 3;
  std::vector<float> proj((size_t)coefs * 16);
  // Scaled so a coefficient vector of typical size maps to latents of ~0.5.
  for (auto& v : proj) v = (float)(rng.normal() * 2.0 / std::sqrt((double)coefs));
  float* dproj = nullptr;
  if ((rc = dalloc((void**)&dproj, proj.size() * 4, "init"))) return bail(rc);
  e = cudaMemcpyAsync(dproj, proj.data(), proj.size() * 4, cudaMemcpyHostToDevice, L->stream);
  if (e == cudaSuccess) {
    k_init_latents<<<std::min<uint64_t>((L->n + 255) / 256, 4096), 256, 0, L->stream>>>(a, L->sh_degree, dproj,
                                                                                          L->lat32, L->lat16);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
  cudaFree(dproj);
  if (e != cudaSuccess) return bail(lcuda(L, e, "latent initialisation"));
  if ((rc = splat_cuda_learner_set_params(L, p.data(), nullptr))) return bail(rc);
  *out = L;
  return SPLAT_OK;
}

namespace {

// Learner checkpoint layout: this header, then the fp32 parameter masters and
// their two Adam moments (kParams floats each), the latent masters and their
// moments (n * 16 floats each) and the latent rows' stamps (n u32): the state
// that the next step reads, so that training resumes where it stopped.
struct LearnerStateHeader {
  char magic[8];  // "SPLATLRN"
  uint32_t version, header_bytes;
  uint64_t n;
  uint32_t directions, batch;
  uint64_t seed;
  uint32_t sh_degree, params;
  uint64_t step;        // completed steps (the Adam bias correction and the shuffle position)
  double loss_sum;      // the loss record of the current call
  uint64_t loss_steps;
  float last_loss, pad;
};
constexpr uint32_t kStateVersion = 1;

size_t state_bytes(const splat_cuda_learner* L) {
  return sizeof(LearnerStateHeader) + 3ull * mlp::kParams * 4 + 3ull * L->n * 64 + L->n * 4;
}

}  // namespace

SPLAT_API size_t splat_cuda_learner_state_bytes(const splat_cuda_learner* L) { return L ? state_bytes(L) : 0; }

SPLAT_API int splat_cuda_learner_save_state(splat_cuda_learner* L, void* out, size_t bytes) {
  if (!L || !out) return SPLAT_ERR_INVALID_ARG;
  if (bytes < state_bytes(L)) return lfail(L, SPLAT_ERR_INVALID_ARG, "buffer smaller than splat_cuda_learner_state_bytes");
  LCK(cudaSetDevice(L->device), "cudaSetDevice");
  LCK(cudaStreamSynchronize(L->stream), "learner stream");
  StepState st{};
  LCK(cudaMemcpy(&st, L->st, sizeof(st), cudaMemcpyDeviceToHost), "read step state");
  LearnerStateHeader hd{};
  std::memcpy(hd.magic, "SPLATLRN", 8);
  hd.version = kStateVersion;
  hd.header_bytes = sizeof(LearnerStateHeader);
  hd.n = L->n;
  hd.directions = L->n_dirs;
  hd.batch = L->batch;
  hd.seed = L->seed;
  hd.sh_degree = L->sh_degree;
  hd.params = mlp::kParams;
  hd.step = st.step;
  hd.loss_sum = st.loss_sum;
  hd.loss_steps = st.loss_steps;
  hd.last_loss = st.last_loss;
  uint8_t* o = static_cast<uint8_t*>(out);
  std::memcpy(o, &hd, sizeof(hd));
  o += sizeof(hd);
  const size_t pb = mlp::kParams * 4, lb = L->n * 64;
  for (const auto& part : {std::make_pair((const void*)L->p32, pb), std::make_pair((const void*)L->pm, pb),
                           std::make_pair((const void*)L->pv, pb), std::make_pair((const void*)L->lat32, lb),
                           std::make_pair((const void*)L->lm, lb), std::make_pair((const void*)L->lv, lb),
                           std::make_pair((const void*)L->stamp, (size_t)L->n * 4)}) {
    LCK(cudaMemcpy(o, part.first, part.second, cudaMemcpyDeviceToHost), "read learner state");
    o += part.second;
  }
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_learner_load_state(splat_cuda_learner* L, const void* data, size_t bytes) {
  if (!L || !data) return SPLAT_ERR_INVALID_ARG;
  LearnerStateHeader hd{};
  if (bytes < sizeof(hd)) return lfail(L, SPLAT_ERR_INVALID_ARG, "not a learner state (too short)");
  std::memcpy(&hd, data, sizeof(hd));
  if (std::memcmp(hd.magic, "SPLATLRN", 8) != 0 || hd.header_bytes != sizeof(hd))
    return lfail(L, SPLAT_ERR_INVALID_ARG, "not a learner state");
  if (hd.version != kStateVersion) return lfail(L, SPLAT_ERR_UNSUPPORTED, "unsupported learner state version");
  if (hd.n != L->n || hd.directions != L->n_dirs || hd.batch != L->batch || hd.seed != L->seed ||
      hd.sh_degree != L->sh_degree || hd.params != mlp::kParams)
    return lfail(L, SPLAT_ERR_INVALID_ARG,
                 "learner state of another scene or configuration (splats, directions, batch, seed, SH degree)");
  if (bytes < state_bytes(L)) return lfail(L, SPLAT_ERR_INVALID_ARG, "learner state truncated");
  LCK(cudaSetDevice(L->device), "cudaSetDevice");
  LCK(cudaStreamSynchronize(L->stream), "learner stream");
  const uint8_t* p = static_cast<const uint8_t*>(data) + sizeof(hd);
  const size_t pb = mlp::kParams * 4, lb = L->n * 64;
  for (const auto& part : {std::make_pair((void*)L->p32, pb), std::make_pair((void*)L->pm, pb),
                           std::make_pair((void*)L->pv, pb), std::make_pair((void*)L->lat32, lb),
                           std::make_pair((void*)L->lm, lb), std::make_pair((void*)L->lv, lb),
                           std::make_pair((void*)L->stamp, (size_t)L->n * 4)}) {
    LCK(cudaMemcpy(part.first, p, part.second, cudaMemcpyHostToDevice), "upload learner state");
    p += part.second;
  }
  // A cudaMemcpy from pageable memory may return before its DMA lands, and
  // the learner's non-blocking stream does not wait for the legacy stream
  // that carries it.
  LCK(cudaDeviceSynchronize(), "upload learner state");
  k_to_half<<<(mlp::kParams + 255) / 256, 256, 0, L->stream>>>(L->p32, L->p16, mlp::kParams);
  k_to_half<<<(uint32_t)std::min<uint64_t>((L->n * 16 + 255) / 256, 8192), 256, 0, L->stream>>>(L->lat32, L->lat16,
                                                                                                 L->n * 16);
  LCK(cudaGetLastError(), "learner state");
  StepState st{};
  st.step = hd.step;
  st.loss_sum = hd.loss_sum;
  st.loss_steps = hd.loss_steps;
  st.last_loss = hd.last_loss;
  LCK(cudaMemcpyAsync(L->st, &st, sizeof(st), cudaMemcpyHostToDevice, L->stream), "upload step state");
  LCK(cudaMemsetAsync(L->grad, 0, mlp::kParams * 4, L->stream), "clear gradients");
  LCK(cudaMemsetAsync(L->lgrad, 0, L->n * 64, L->stream), "clear gradients");
  LCK(cudaStreamSynchronize(L->stream), "learner state");  // &st is a local
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_learner_set_params(splat_cuda_learner* L, const float* params, const float* latents) {
  if (!L) return SPLAT_ERR_INVALID_ARG;
  LCK(cudaSetDevice(L->device), "cudaSetDevice");
  LCK(cudaStreamSynchronize(L->stream), "learner stream");
  if (params) {
    LCK(cudaMemcpyAsync(L->p32, params, mlp::kParams * 4, cudaMemcpyHostToDevice, L->stream), "upload parameters");
    k_to_half<<<(mlp::kParams + 255) / 256, 256, 0, L->stream>>>(L->p32, L->p16, mlp::kParams);
    LCK(cudaGetLastError(), "parameters");
  }
  if (latents) {
    LCK(cudaMemcpyAsync(L->lat32, latents, L->n * 64, cudaMemcpyHostToDevice, L->stream), "upload latents");
    k_to_half<<<(uint32_t)std::min<uint64_t>((L->n * 16 + 255) / 256, 8192), 256, 0, L->stream>>>(L->lat32, L->lat16,
                                                                                                   L->n * 16);
    LCK(cudaGetLastError(), "latents");
  }
  // Fresh optimiser state and step count.
  LCK(cudaMemsetAsync(L->pm, 0, mlp::kParams * 4, L->stream), "reset");
  LCK(cudaMemsetAsync(L->pv, 0, mlp::kParams * 4, L->stream), "reset");
  LCK(cudaMemsetAsync(L->lm, 0, L->n * 64, L->stream), "reset");
  LCK(cudaMemsetAsync(L->lv, 0, L->n * 64, L->stream), "reset");
  LCK(cudaMemsetAsync(L->stamp, 0, L->n * 4, L->stream), "reset");
  LCK(cudaMemsetAsync(L->st, 0, sizeof(StepState), L->stream), "reset");
  LCK(cudaStreamSynchronize(L->stream), "reset");
  return SPLAT_OK;
}

// Arms an injected lost completion (SPLAT_FAULT_LOST_WAIT) for the steps the
// call enqueues next; sync_state clears it.
int arm_injection(splat_cuda_learner* L) {
  if (!L->inject_lost_us) return SPLAT_OK;
  LCK(cudaMemcpyAsync(&L->st->lost_wait_us, &L->inject_lost_us, sizeof(unsigned int), cudaMemcpyHostToDevice,
                      L->stream),
      "fault injection");
  LCK(cudaStreamSynchronize(L->stream), "fault injection");
  L->inject_lost_us = 0;
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_learner_train(splat_cuda_learner* L, uint64_t steps, splat_learn_stats* stats) {
  if (!L) return SPLAT_ERR_INVALID_ARG;
  LCK(cudaSetDevice(L->device), "cudaSetDevice");
  if (int rc = arm_injection(L)) return rc;
  LCK(cudaMemsetAsync(&L->st->loss_sum, 0, sizeof(double) + sizeof(unsigned long long), L->stream), "reset loss");
  if (!L->graph && steps >= kGraphSteps) {
    cudaGraph_t g = nullptr;
    LCK(cudaStreamBeginCapture(L->stream, cudaStreamCaptureModeThreadLocal), "capture");
    cudaError_t e = cudaSuccess;
    for (uint32_t i = 0; i < kGraphSteps && e == cudaSuccess; i++) e = enqueue_step(L, L->stream);
    cudaError_t e2 = cudaStreamEndCapture(L->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return lcuda(L, e != cudaSuccess ? e : e2, "capture training steps");
    }
    e = cudaGraphInstantiate(&L->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      L->graph = nullptr;
      return lcuda(L, e, "instantiate training graph");
    }
    L->launches -= 2 * kGraphSteps;  // counted again at each replay
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  LCK(cudaEventCreate(&e0), "event");
  LCK(cudaEventCreate(&e1), "event");
  LCK(cudaEventRecord(e0, L->stream), "event");
  uint64_t left = steps;
  while (L->graph && left >= kGraphSteps) {
    LCK(cudaGraphLaunch(L->graph, L->stream), "training graph");
    L->launches += 2 * kGraphSteps;
    left -= kGraphSteps;
  }
  for (; left; left--) LCK(enqueue_step(L, L->stream), "training step");
  LCK(cudaEventRecord(e1, L->stream), "event");
  StepState st;
  int rc = sync_state(L, &st);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (stats) {
    stats->steps = st.step;
    stats->epochs = (double)st.step / L->steps_per_epoch;
    stats->mean_loss = st.loss_steps ? st.loss_sum / (double)st.loss_steps : 0.0;
    stats->last_loss = st.last_loss;
    stats->ms = ms;
    stats->steps_per_epoch = L->steps_per_epoch;
    stats->samples_per_epoch = L->samples;
  }
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_learner_step_debug(splat_cuda_learner* L, float* grad_params, float* grad_latents) {
  if (!L) return SPLAT_ERR_INVALID_ARG;
  LCK(cudaSetDevice(L->device), "cudaSetDevice");
  if (int rc = arm_injection(L)) return rc;
  LCK(launch_train<Src::kScene>(L->args, L->grid, L->sh_degree, L->stream), "training kernel");
  L->launches += 1;
  StepState st;
  int rc = sync_state(L, &st);
  if (rc) return rc;
  const uint64_t k = st.step % L->steps_per_epoch;
  const uint64_t active = std::min<uint64_t>(L->batch, L->samples - k * L->batch);
  const double inv = 1.0 / (kLossScale * (double)active);
  if (grad_params) {
    LCK(cudaMemcpy(grad_params, L->grad, mlp::kParams * 4, cudaMemcpyDeviceToHost), "read gradient");
    for (uint32_t i = 0; i < mlp::kParams; i++) grad_params[i] = (float)(grad_params[i] * inv);
  }
  if (grad_latents) {
    LCK(cudaMemcpy(grad_latents, L->lgrad, L->n * 64, cudaMemcpyDeviceToHost), "read gradient");
    for (uint64_t i = 0; i < L->n * 16; i++) grad_latents[i] = (float)(grad_latents[i] * inv);
  }
  enqueue_adam(L, L->stream);
  L->launches += 1;
  LCK(cudaGetLastError(), "Adam kernel");
  return sync_state(L, &st);
}

SPLAT_API int splat_cuda_learner_params(splat_cuda_learner* L, float* params, float* latents, uint16_t* params_f16,
                                        uint16_t* latents_f16) {
  if (!L) return SPLAT_ERR_INVALID_ARG;
  LCK(cudaSetDevice(L->device), "cudaSetDevice");
  LCK(cudaStreamSynchronize(L->stream), "learner stream");
  if (params) LCK(cudaMemcpy(params, L->p32, mlp::kParams * 4, cudaMemcpyDeviceToHost), "read parameters");
  if (latents) LCK(cudaMemcpy(latents, L->lat32, L->n * 64, cudaMemcpyDeviceToHost), "read latents");
  if (params_f16) LCK(cudaMemcpy(params_f16, L->p16, mlp::kParams * 2, cudaMemcpyDeviceToHost), "read parameters");
  if (latents_f16) LCK(cudaMemcpy(latents_f16, L->lat16, L->n * 32, cudaMemcpyDeviceToHost), "read latents");
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_learner_directions(const splat_cuda_learner* L, float* dirs) {
  if (!L || !dirs) return SPLAT_ERR_INVALID_ARG;
  std::vector<float4> d(L->n_dirs);
  if (cudaSetDevice(L->device) != cudaSuccess ||
      cudaMemcpy(d.data(), L->dirs, d.size() * sizeof(float4), cudaMemcpyDeviceToHost) != cudaSuccess)
    return SPLAT_ERR_DEVICE;
  for (uint32_t i = 0; i < L->n_dirs; i++) {
    dirs[3 * i] = d[i].x;
    dirs[3 * i + 1] = d[i].y;
    dirs[3 * i + 2] = d[i].z;
  }
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_learner_get_option(const splat_cuda_learner* L, uint32_t option, uint64_t* value) {
  if (!L || !value) return SPLAT_ERR_INVALID_ARG;
  switch (option) {
    case SPLAT_OPT_KERNEL_LAUNCHES: *value = L->launches; return SPLAT_OK;
    case SPLAT_LEARN_STEPS_PER_EPOCH: *value = L->steps_per_epoch; return SPLAT_OK;
    case SPLAT_LEARN_SHUFFLE_BITS: *value = L->bits; return SPLAT_OK;
    case SPLAT_LEARN_TRAIN_CTAS: *value = L->grid; return SPLAT_OK;
    default: return SPLAT_ERR_UNSUPPORTED;
  }
}

SPLAT_API int splat_cuda_learner_set_option(splat_cuda_learner* L, uint32_t option, uint64_t value) {
  if (!L) return SPLAT_ERR_INVALID_ARG;
  switch (option) {
    case SPLAT_OPT_INJECT_FAULT:
      if ((value & 0xFFu) == SPLAT_FAULT_LOST_WAIT) {
        L->inject_lost_us = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(value >> 8, 10000000ull));
        return SPLAT_OK;
      }
      if (value == 0) {
        L->inject_lost_us = 0;
        return SPLAT_OK;
      }
      return lfail(L, SPLAT_ERR_UNSUPPORTED, "the learner injects SPLAT_FAULT_LOST_WAIT only");
    default:
      return lfail(L, SPLAT_ERR_UNSUPPORTED, "unknown option");
  }
}

SPLAT_API const char* splat_cuda_learner_last_error(const splat_cuda_learner* L) { return L ? L->err.c_str() : ""; }

SPLAT_API int splat_cuda_learner_destroy(splat_cuda_learner* L) {
  if (!L) return SPLAT_OK;
  cudaSetDevice(L->device);
  if (L->stream) cudaStreamSynchronize(L->stream);
  if (L->graph) cudaGraphExecDestroy(L->graph);
  for (void* p : {(void*)L->p32, (void*)L->pm, (void*)L->pv, (void*)L->grad, (void*)L->p16, (void*)L->lat32,
                  (void*)L->lm, (void*)L->lv, (void*)L->lgrad, (void*)L->lat16, (void*)L->stamp,
                  (void*)L->dirs, (void*)L->shs, (void*)L->st})
    if (p) cudaFree(p);
  if (L->stream) cudaStreamDestroy(L->stream);
  delete L;
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_mlp_gradient(int device, const float* params, const uint16_t* latents, const float* dirs,
                                      const float* targets, uint32_t count, float* grad_params, float* grad_latents,
                                      float* outputs, double* loss) {
  if (!params || !latents || !dirs || !targets || count == 0 || count > (1u << 20)) return SPLAT_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return SPLAT_ERR_DEVICE;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  float *d_p = nullptr, *d_dir = nullptr, *d_tgt = nullptr, *d_gl = nullptr, *d_out = nullptr, *d_g = nullptr;
  uint16_t *d_p16 = nullptr, *d_lat = nullptr;
  double* d_loss = nullptr;
  StepState* d_st = nullptr;
  int rc = SPLAT_OK;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == SPLAT_OK) rc = e == cudaErrorMemoryAllocation ? SPLAT_ERR_OOM : SPLAT_ERR_DEVICE;
    return rc == SPLAT_OK;
  };
  ok(cudaMalloc(&d_p, mlp::kParams * 4)) && ok(cudaMalloc(&d_p16, mlp::kParams * 2)) &&
      ok(cudaMalloc(&d_g, mlp::kParams * 4)) && ok(cudaMalloc(&d_lat, (size_t)count * 32)) &&
      ok(cudaMalloc(&d_dir, (size_t)count * 12)) && ok(cudaMalloc(&d_tgt, (size_t)count * 12)) &&
      ok(cudaMalloc(&d_gl, (size_t)count * 64)) && ok(cudaMalloc(&d_out, (size_t)count * 12)) &&
      ok(cudaMalloc(&d_loss, 8)) && ok(cudaMalloc(&d_st, sizeof(StepState)));
  if (rc == SPLAT_OK) {
    ok(cudaMemcpy(d_p, params, mlp::kParams * 4, cudaMemcpyHostToDevice)) &&
        ok(cudaMemcpy(d_lat, latents, (size_t)count * 32, cudaMemcpyHostToDevice)) &&
        ok(cudaMemcpy(d_dir, dirs, (size_t)count * 12, cudaMemcpyHostToDevice)) &&
        ok(cudaMemcpy(d_tgt, targets, (size_t)count * 12, cudaMemcpyHostToDevice)) &&
        ok(cudaMemset(d_g, 0, mlp::kParams * 4)) && ok(cudaMemset(d_loss, 0, 8)) &&
        ok(cudaMemset(d_st, 0, sizeof(StepState)));
  }
  if (rc == SPLAT_OK) {
    k_to_half<<<(mlp::kParams + 255) / 256, 256>>>(d_p, d_p16, mlp::kParams);
    TrainArgs a{};
    a.p16 = d_p16;
    a.grad = d_g;
    a.st = d_st;
    a.ex_lat = reinterpret_cast<const uint4*>(d_lat);
    a.ex_dir = d_dir;
    a.ex_tgt = d_tgt;
    a.ex_glat = d_gl;
    a.ex_out = d_out;
    a.ex_loss = d_loss;
    a.ex_count = count;
    a.tiles = (count + mlp::kRows - 1) / mlp::kRows;
    const uint32_t slots = 2u * (uint32_t)sms, per = (a.tiles + slots - 1) / slots;
    ok(cudaGetLastError()) && ok(launch_train<Src::kExplicit>(a, (a.tiles + per - 1) / per, 0, nullptr)) &&
        ok(cudaDeviceSynchronize());
  }
  StepState st{};
  if (rc == SPLAT_OK) ok(cudaMemcpy(&st, d_st, sizeof(st), cudaMemcpyDeviceToHost));
  if (rc == SPLAT_OK && st.error) rc = SPLAT_ERR_TIMEOUT;
  if (rc == SPLAT_OK) {
    const double inv = 1.0 / (kLossScale * (double)count);
    std::vector<float> g(mlp::kParams);
    std::vector<float> gl((size_t)count * 16);
    double ls = 0.0;
    ok(cudaMemcpy(g.data(), d_g, mlp::kParams * 4, cudaMemcpyDeviceToHost)) &&
        ok(cudaMemcpy(gl.data(), d_gl, gl.size() * 4, cudaMemcpyDeviceToHost)) &&
        ok(cudaMemcpy(&ls, d_loss, 8, cudaMemcpyDeviceToHost)) &&
        (!outputs || ok(cudaMemcpy(outputs, d_out, (size_t)count * 12, cudaMemcpyDeviceToHost)));
    if (rc == SPLAT_OK) {
      if (grad_params)
        for (uint32_t i = 0; i < mlp::kParams; i++) grad_params[i] = (float)(g[i] * inv);
      if (grad_latents)
        for (size_t i = 0; i < gl.size(); i++) grad_latents[i] = (float)(gl[i] * inv);
      if (loss) *loss = ls / (3.0 * count);
    }
  }
  for (void* p : {(void*)d_p, (void*)d_p16, (void*)d_g, (void*)d_lat, (void*)d_dir, (void*)d_tgt, (void*)d_gl,
                  (void*)d_out, (void*)d_loss, (void*)d_st})
    if (p) cudaFree(p);
  return rc;
}
