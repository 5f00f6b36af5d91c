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

// The tile sort of words[0, n) with `scratch` as its ping-pong range
// (long_tile_sort: stable LSD passes over the varying bytes of the depth
// bits, run chunk by chunk through shared memory with the digit starts
// carried across chunks; ties of depth ordered by splat index, fix_ties of
// src/render/cpu.rs:396-414, with linear LSD passes). One CTA.
__global__ void __launch_bounds__(kTileThreads) k_sort_tile_noalloc(uint64_t* __restrict__ words, uint32_t n,
                                                                    uint64_t* __restrict__ scratch) {
  __shared__ ChunkSortSmem sm;
  long_tile_sort(words, scratch, n, sm);
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
