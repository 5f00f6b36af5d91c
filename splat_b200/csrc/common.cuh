// Shared definitions of the sm_100a rasterizer kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace splat {

// src/render/mod.rs:23-33
constexpr float kDilation = 0.3f;
constexpr float kAlphaMin = 1.0f / 255.0f;
constexpr float kAlphaMax = 0.99f;
constexpr float kTMin = 1e-4f;
constexpr uint32_t kMaxDim = 16384;
// src/render/cpu.rs:34 (16x16 tiles; row masks there, one CTA per tile here)
constexpr uint32_t kTile = 16;
constexpr uint32_t kTilePixels = kTile * kTile;

// Marks a culled splat in BinInfo::rect_lo.
constexpr uint32_t kCulled = 0xFFFFFFFFu;

// Largest pair count the sort's 30-bit look-back words can carry.
constexpr uint64_t kMaxPairs = (1ull << 30) - 1;

// Bounded spin of every device-side wait (decoupled look-back). A wait that
// runs out sets an error bit and the kernel carries on without writing out of
// bounds; the host turns the bit into SPLAT_ERR_TIMEOUT.
constexpr uint32_t kSpinLimit = 1u << 20;

enum ErrorBits : uint32_t {
  kErrEmitTimeout = 1u,
  kErrSortTimeout = 2u,
  kErrSortRange = 4u,
};

// Per-frame constants (ProjectCtx, src/render/mod.rs:155-196) plus grid sizes.
struct FrameParams {
  float rot[9];  // row-major: rows are right, down, forward (View::rotation)
  float eye[3];
  float focal, cx, cy, width, height, near_plane, lim_x, lim_y;
  float bg[3];
  uint32_t w, h;
  uint32_t tiles_x, tiles_y;
  uint32_t downsample;      // 1 = none
  uint32_t out_w, out_h;    // floor(w/f), floor(h/f)
};

// Device-resident scene, FP32 storage (layout chosen for coalesced loads).
struct SceneDev {
  const float4* pos_op;   // x, y, z, opacity
  const float4* cov_a;    // xx, xy, xz, yy
  const float4* cov_b;    // yz, zz, k = sqrt(2 ln(op / ALPHA_MIN)), 0
  const float* color;     // 3 planes of n: r, g, b (base colour)
  const float* sh;        // rest*3 planes of n: plane (coef*3 + channel)
  uint64_t n;
  uint32_t sh_degree;
};

// A projected splat as the blend reads it: 48 bytes, three float4.
//  r0 = x, y, -0.5*conic_a, -conic_b
//  r1 = -0.5*conic_c, opacity, red, green
//  r2 = blue, bbox x0 | x1 << 16, bbox y0 | y1 << 16, depth
struct __align__(16) Record {
  float4 r0, r1, r2;
};

// Per-splat binning input written by the projection: the tile rectangle of
// its pixel bbox (tx0 | ty0 << 16, tx1 | ty1 << 16), depth bits, pair count.
// rect_lo == kCulled marks a culled splat.
struct __align__(16) BinInfo {
  uint32_t rect_lo, rect_hi, depth_bits, count;
};

constexpr int kMaxDigits = 8;

// Frame state in device memory, cleared at the start of every frame.
struct DevState {
  unsigned long long total_pairs;  // sum of per-splat pair counts (may exceed capacity)
  unsigned int visible;
  unsigned int error;
  unsigned int emit_ticket;
  unsigned int sort_ticket[kMaxDigits];
  int pass_src[kMaxDigits];        // per digit pass: source buffer (0/1) or -1 to skip
  int final_sel;                   // buffer holding the sorted pairs
  unsigned int pad[5];
  unsigned int hist[kMaxDigits][256];  // digit histograms, then exclusive starts
};

// Decoupled look-back descriptor flags (emit scan: 64-bit words).
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagInc = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1;

// Launchers (each returns the cudaGetLastError of its launches).
cudaError_t launch_project(const FrameParams& fp, const SceneDev& s, Record* rec, BinInfo* bin, float* dbg_proj,
                           float* dbg_color, DevState* st, cudaStream_t stream);
cudaError_t launch_emit(const FrameParams& fp, const BinInfo* bin, uint64_t n, unsigned long long* emit_desc,
                        uint64_t* keys, uint32_t* vals, uint64_t cap, DevState* st, cudaStream_t stream);
cudaError_t launch_sort(uint32_t key_bits, uint64_t cap, uint64_t* keys0, uint32_t* vals0, uint64_t* keys1,
                        uint32_t* vals1, uint32_t* lookback, uint64_t lookback_parts, DevState* st,
                        int num_sms, cudaStream_t stream);
cudaError_t launch_ranges(uint64_t cap, uint64_t* const* keys, uint2* ranges, uint32_t tiles, DevState* st,
                          int num_sms, cudaStream_t stream);
cudaError_t launch_blend(const FrameParams& fp, const Record* rec, const uint32_t* const* vals, const uint2* ranges,
                         const DevState* st, bool exact, uint8_t* out, uint8_t* full_scratch, cudaStream_t stream);

// Partition size (pairs) of one onesweep CTA.
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortPart = kSortThreads * kSortItems;

}  // namespace splat
