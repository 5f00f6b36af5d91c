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
// FP16 storage: a 2D covariance determinant below this is recomputed in FP64.
constexpr float kFp64DetBelow = 1e-6f;
constexpr uint32_t kMaxDim = 16384;
// src/render/cpu.rs:34 (16x16 tiles; row masks there, one CTA per tile here)
constexpr uint32_t kTile = 16;
constexpr uint32_t kTilePixels = kTile * kTile;

// Marks a culled splat in BinInfo::rect_lo.
constexpr uint32_t kCulled = 0xFFFFFFFFu;

// Largest pair capacity (pair offsets and tile ranges are 32-bit).
constexpr uint64_t kMaxPairs = (1ull << 30) - 1;

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
  // FP32 storage
  const float4* pos_op;   // x, y, z, opacity
  const float4* cov_a;    // xx, xy, xz, yy
  const float4* cov_b;    // yz, zz, k = sqrt(2 ln(op / ALPHA_MIN)), 0
  const float* color;     // 3 planes of n: r, g, b (base colour)
  const float* sh;        // rest*3 planes of n: plane (coef*3 + channel)
  // FP16 storage (128 bytes per splat)
  const float4* pos_k;    // x, y, z, k
  const uint4* geom16;    // 8 halves: scale x, y, z, rotation x, y, z, w, opacity
  const uint16_t* sh16;   // (rest+1)*3 planes of n halves: base colour, then the rest
  uint64_t n;
  uint32_t sh_degree;
  uint32_t fp16;
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
// rect_lo == kCulled marks a culled splat; a visible splat whose bbox holds
// no pixel has count 0.
struct __align__(16) BinInfo {
  uint32_t rect_lo, rect_hi, depth_bits, count;
};

// Per-tile depth sort sizes: tiles up to kWarpSortCap pairs are sorted by one
// warp, up to kMidSortCap by one CTA in shared memory, longer ones in chunks.
constexpr uint32_t kWarpSortCap = 512;
constexpr uint32_t kMidSortCap = 4096;

// Frame state in device memory, cleared at the start of every frame.
struct DevState {
  unsigned long long visible;      // splats that survived culling
  unsigned long long total_pairs;  // (splat, tile) pairs, may exceed the capacity
  unsigned int error;
  unsigned int mid_tiles;          // tiles with (kWarpSortCap, kMidSortCap] pairs
  unsigned int long_tiles;         // tiles with more than kMidSortCap pairs
  unsigned int fp64_conics;        // splats whose 2D conic was recomputed in FP64
};

// Launchers (each returns the cudaGetLastError of its launches).
// (a) projection: records, tile rectangles and pair counts, visible count.
cudaError_t launch_project(const FrameParams& fp, const SceneDev& s, Record* rec, BinInfo* bin, float* dbg_proj,
                           float* dbg_color, DevState* st, cudaStream_t stream, uint32_t* launches);
// (b) binning into per-tile buckets (count matrix of bin_rows() x tiles,
// tile totals, ranges, mid/long tile lists) and (c) the per-tile depth sorts.
uint32_t bin_rows(int num_sms);
cudaError_t launch_binning(const FrameParams& fp, const BinInfo* bin, uint64_t n, uint32_t* counts, uint32_t* totals,
                           uint2* ranges, uint32_t* mid_list, uint32_t* long_list, uint64_t* pairs,
                           uint64_t* pairs_alt, uint64_t cap, DevState* st, int num_sms, size_t max_smem,
                           cudaStream_t stream, uint32_t* launches);
// (d) blend + downsample over the depth-sorted buckets.
cudaError_t launch_blend(const FrameParams& fp, const Record* rec, const uint64_t* pairs, const uint2* ranges,
                         bool exact, uint8_t* out, uint8_t* full_scratch, cudaStream_t stream, uint32_t* launches);

}  // namespace splat
