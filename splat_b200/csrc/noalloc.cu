// splat_cuda_sort_tile_noalloc: one tile's depth sort for callers that cannot
// allocate device memory.
//
// Some hosts cannot call cudaMalloc: a process whose device memory belongs to
// another allocator (a framework's caching allocator or a fixed memory pool),
// or code that must not allocate while it runs (a real-time frame loop, a
// launch sequence being recorded). The renderer's own long-tile sort
// (k_sort_long in binning.cu) ping-pongs through a second pair buffer that the
// handle allocates. This variant takes only the caller's pairs and keeps its
// ping-pong buffer in a file-scope device array instead, so the call
// allocates nothing: every GPU that loads the library holds the array
// (kNoAllocMaxPairs words, 8 MiB) until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents; nothing in it needs to start at zero (each pass writes every word
// it later reads). Calls whose kernels overlap on the GPU (concurrent streams)
// race on the array and must not be issued. Host code cannot pass the array's
// name to a kernel (in host code it is only a stand-in, not a device
// address), so the first call on each device looks up the array's device
// address with cudaGetSymbolAddress and caches it; that first call should
// come before any stream capture.
#include <mutex>

#include "../../include/splat_cuda.h"
#include "common.cuh"
#include "tilesort.cuh"

#define SPLAT_API extern "C" __attribute__((visibility("default")))

namespace splat {
namespace {

constexpr uint32_t kNoAllocMaxPairs = 1u << 20;
static __device__ __align__(256) uint64_t g_noalloc_scratch[kNoAllocMaxPairs];

constexpr int kChunk = 4096;

struct NoAllocSmem {
  TileSortSmem t;
  uint32_t run[256];  // running start of each digit across chunks
  uint32_t key[kChunk];
};

// The tile sort of words[0, n): stable LSD passes over the 8-bit digits of the
// depth bits that are not shared by every word, run chunk by chunk through
// shared memory with the digit starts carried across chunks (ping-pong with
// `scratch`), then runs of equal depth ordered by splat index (fix_ties,
// src/render/cpu.rs:396-414). One CTA.
__global__ void __launch_bounds__(kTileThreads) k_sort_tile_noalloc(uint64_t* __restrict__ words, uint32_t n,
                                                                    uint64_t* __restrict__ scratch) {
  __shared__ NoAllocSmem sm;
  constexpr int kChunks = kChunk / (32 * kTileWarps);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint32_t a = 0xFFFFFFFFu, o = 0u;
  for (uint32_t e = tid; e < n; e += kTileThreads) {
    const uint32_t k = (uint32_t)(words[e] >> 32);
    a &= k;
    o |= k;
  }
  uint32_t and_all, or_all;
  block_and_or(a, o, sm.t, and_all, or_all);
  const uint32_t vary = and_all ^ or_all;
  uint64_t* src = words;
  uint64_t* dst = scratch;
  for (int d = 0; d < 4; d++) {
    const int shift = 32 + 8 * d;
    if (((vary >> (8 * d)) & 255u) == 0u) continue;
    clear_counts(sm.t);
    __syncthreads();
    for (uint32_t e = tid; e < n; e += kTileThreads) atomicAdd(&sm.t.wh[warp][(src[e] >> shift) & 255u], 1u);
    __syncthreads();
    digit_offsets(sm.t);
    sm.run[tid] = sm.t.dstart[tid];
    __syncthreads();
    for (uint32_t c0 = 0; c0 < n; c0 += kChunk) {
      const uint32_t cn = min((uint32_t)kChunk, n - c0);
      for (uint32_t e = tid; e < cn; e += kTileThreads) sm.key[e] = (uint32_t)(src[c0 + e] >> 32);
      clear_counts(sm.t);
      __syncthreads();
      const uint32_t seg = (cn + kTileWarps - 1) / kTileWarps;
      const uint32_t seg0 = min(cn, (uint32_t)warp * seg), seg1 = min(cn, seg0 + seg);
      uint32_t k[kChunks], dr[kChunks];
      warp_rank<kChunks>(sm.key, seg0, seg1, 8 * d, sm.t, k, dr);
      __syncthreads();
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
  if (src != words)
    for (uint32_t e = tid; e < n; e += kTileThreads) words[e] = src[e];
  __syncthreads();
  for (uint32_t e = tid + 1; e < n; e += kTileThreads) {
    const uint32_t kk = (uint32_t)(words[e] >> 32);
    if (kk == (uint32_t)(words[e - 1] >> 32) && (e == 1 || (uint32_t)(words[e - 2] >> 32) != kk)) {
      uint32_t r1 = e + 1;
      while (r1 < n && (uint32_t)(words[r1] >> 32) == kk) r1++;
      for (uint32_t i = e; i < r1; i++) {
        const uint64_t x = words[i];
        uint32_t j = i;
        while (j > e - 1 && (uint32_t)words[j - 1] > (uint32_t)x) {
          words[j] = words[j - 1];
          j--;
        }
        words[j] = x;
      }
    }
  }
}

constexpr int kMaxDevices = 64;
uint64_t* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of the scratch array on the current device (looked up once
// per device, with that device current).
cudaError_t scratch_address(int device, uint64_t** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<uint64_t*>(p);
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

}  // namespace
}  // namespace splat

SPLAT_API int splat_cuda_sort_tile_noalloc(uint64_t* words, uint32_t n, void* stream) {
  using namespace splat;
  if (n > kNoAllocMaxPairs) return SPLAT_ERR_INVALID_ARG;  // more pairs than the scratch array holds
  if (n < 2) return SPLAT_OK;
  if (!words) return SPLAT_ERR_INVALID_ARG;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return SPLAT_ERR_DEVICE;
  uint64_t* scratch = nullptr;
  if (scratch_address(device, &scratch) != cudaSuccess) return SPLAT_ERR_DEVICE;
  k_sort_tile_noalloc<<<1, kTileThreads, 0, (cudaStream_t)stream>>>(words, n, scratch);
  return cudaGetLastError() == cudaSuccess ? SPLAT_OK : SPLAT_ERR_DEVICE;
}
