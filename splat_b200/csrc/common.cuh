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

constexpr int kMaxPasses = 4;  // 8-bit digits of a 32-bit sort field

// One stable LSD sort of 64-bit words on (part of) their upper 32 bits.
struct SortState {
  unsigned int ticket[kMaxPasses];
  int pass_src[kMaxPasses];  // per digit pass: source buffer (0/1) or -1 to skip
  int final_sel;             // buffer holding the sorted words
  unsigned int pad[3];
  unsigned int hist[kMaxPasses][256];  // digit histograms, then exclusive starts
};

// Frame state in device memory, cleared at the start of every frame.
struct DevState {
  unsigned long long visible;      // splats that survived culling
  unsigned long long total_pairs;  // sum of per-splat pair counts (may exceed capacity)
  unsigned int error;
  unsigned int project_ticket;
  unsigned int emit_ticket;
  unsigned int pad[5];
  SortState depth;  // visible splats by depth: words (depth bits << 32 | splat)
  SortState tile;   // pairs by tile: words (tile << 32 | splat), already in depth order
};

// Decoupled look-back descriptor flags (scans: 64-bit words).
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagInc = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1;

// Launchers (each returns the cudaGetLastError of its launches).
// (a) projection; a depth word per splat and the depth-digit histograms.
cudaError_t launch_project(const FrameParams& fp, const SceneDev& s, Record* rec, BinInfo* bin, uint64_t* depth_words,
                           float* dbg_proj, float* dbg_color, DevState* st, cudaStream_t stream);
// (b) pair emission over the depth-sorted visible splats; counts the tile
// sort's digit histograms.
cudaError_t launch_emit(const FrameParams& fp, int tile_digits, const BinInfo* bin, uint64_t n,
                        unsigned long long* scan_desc, uint64_t* const* depth_words, uint64_t* pairs, uint64_t cap,
                        DevState* st, cudaStream_t stream);
// (c) stable LSD sort of words[0] (ping-pong with words[1]) on `digits` 8-bit
// digits from bit 32, whose schedule is already in ss; count may be null
// (then cap words are sorted).
cudaError_t launch_sort(SortState* ss, const unsigned long long* count, uint64_t cap, int digits, uint64_t* words0,
                        uint64_t* words1, uint32_t* lookback, uint64_t lookback_parts, DevState* st, int num_sms,
                        cudaStream_t stream);
// (c) pass schedules (exclusive digit starts, skipped digits) of the depth
// sort (histograms from the projection, all n words) and of the tile sort
// (histograms from the emission, total_pairs words capped at cap).
cudaError_t launch_depth_schedule(DevState* st, uint64_t n, cudaStream_t stream);
cudaError_t launch_tile_schedule(DevState* st, uint64_t cap, int digits, cudaStream_t stream);
// (c) per-tile [begin, end) ranges from the tile-sorted pairs (ranges zeroed first).
cudaError_t launch_ranges(uint64_t cap, uint64_t* const* pairs, uint2* ranges, uint32_t tiles, DevState* st,
                          int num_sms, cudaStream_t stream);
// (d) blend + downsample.
cudaError_t launch_blend(const FrameParams& fp, const Record* rec, uint64_t* const* pairs, const uint2* ranges,
                         const DevState* st, bool exact, uint8_t* out, uint8_t* full_scratch, cudaStream_t stream);

// Partition size (pairs) of one onesweep CTA.
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kScanThreads = 256;  // splats per projection / emission partition
constexpr int kSortPart = kSortThreads * kSortItems;

}  // namespace splat
