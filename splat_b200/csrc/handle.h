// The renderer handle behind the C ABI (include/splat_cuda.h) and the host
// helpers that the single-view entry points (api.cu) and the batch entry
// points (batch.cu) share.
#pragma once

#include <string>

#include "../../include/splat_cuda.h"
#include "common.cuh"

struct splat_cuda_handle {
  int device = 0;
  int num_sms = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  uint64_t n = 0;
  uint32_t sh_degree = 0;
  uint32_t precision = SPLAT_PRECISION_FP32;
  // scene (device)
  float4* pos_op = nullptr;
  float4* cov_a = nullptr;
  float4* cov_b = nullptr;
  float* color = nullptr;
  float* sh = nullptr;
  float4* pos_k = nullptr;   // FP16 storage: x, y, z, k
  uint4* geom16 = nullptr;   // FP16 storage: scale, rotation, opacity halves
  uint16_t* sh16 = nullptr;  // FP16 storage: base colour + SH planes
  uint4* lat16 = nullptr;     // learned colour: 16 fp16 latents per splat
  uint16_t* mlp16 = nullptr;  // learned colour: the MLP's fp16 parameters
  uint32_t* bin_order = nullptr;  // the binning order (SceneDev::order)
  // per-splat frame buffers
  splat::Record* rec = nullptr;
  splat::BinInfo* bin = nullptr;
  splat::BinSkip* skip = nullptr;  // kept-tile lists of the wide rectangles
  // splat-sharded frames: the records a splat_cuda_render_records call draws
  // (caller-owned device memory, set for the duration of the call) and their
  // binning input; the record selection's scratch and host copy of its totals
  bool rx = false;
  const splat::Record* rx_rec = nullptr;
  uint64_t rx_n = 0;
  splat::BinInfo* rx_bin = nullptr;
  splat::BinSkip* rx_skip = nullptr;
  uint64_t rx_bin_cap = 0;
  void* shard_scratch = nullptr;
  size_t shard_scratch_cap = 0;
  unsigned long long* shard_totals = nullptr;       // device, kMaxShardWindows
  unsigned long long* shard_totals_host = nullptr;  // pinned, kMaxShardWindows
  // pair buffers: per-tile buckets and the long-tile sort's scratch
  uint64_t cap = 0;
  uint64_t pair_limit = splat::kMaxPairs;  // largest capacity; beyond it frames are drawn in windows
  uint64_t* pairs[2] = {nullptr, nullptr};
  // per-size buffers
  uint2* ranges = nullptr;
  uint32_t* counts = nullptr;     // bin_rows x tiles
  size_t counts_cap = 0;          // words
  uint32_t* totals = nullptr;     // tiles
  uint32_t* order = nullptr;      // kTileClasses x tiles (tile_class lists)
  uint64_t ranges_cap = 0;        // tiles
  size_t max_smem = 48 * 1024;
  uint8_t* out_dev = nullptr;
  size_t out_cap = 0;
  uint8_t* full_dev = nullptr;
  size_t full_cap = 0;
  uint8_t* cells_dev = nullptr;  // terminal cells of the last splat_cuda_render_cells
  size_t cells_cap = 0;
  // frame state
  splat::DevState* st = nullptr;       // the frame counters (splat::DevState first)
  splat::DevState* st_host = nullptr;  // pinned copy of splat::DevState + the view's counters
  uint32_t chunks_cap = 0;      // tile-scan chunks the counters hold
  splat::ViewTask* table = nullptr;    // the view table (one entry)
  splat::BlendConfig blend{splat::kTile, splat::kTile, 512};  // two 16x16 tile groups per CTA
  uint8_t* stage = nullptr;     // pinned staging for pageable outputs
  size_t stage_cap = 0;
  // debug capture
  float* dbg_proj = nullptr;
  float* dbg_color = nullptr;
  bool debug_capture = false;
  // options
  bool exact = false;
  bool stage_events = true;
  bool count_evals = false;  // SPLAT_OPT_COUNT_EVALS
  bool bbox_pairs = false;   // SPLAT_OPT_BBOX_PAIRS
  // fault injection (SPLAT_OPT_INJECT_FAULT), each fires once
  bool inject_alloc = false;    // the next device allocation fails as out of memory
  uint32_t inject_lost_us = 0;  // the next frame's tensor-core waits meet a lost completion
  uint32_t launches = 0;  // kernels this handle has launched (wraps at 2^32)
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // last frame: the tile grid it was drawn with; the frame as requested,
  // its destination and whether that is mapped host memory (for a frame
  // that splat_cuda_finish has to draw again in windows)
  splat::FrameParams last_fp{};
  splat::FrameParams last_req{};
  uint8_t* last_out = nullptr;
  bool last_mapped = false;
  bool have_frame = false;
  std::string err;
};


namespace splat {

// ProjectCtx::new with View::rotation/focal, in f32 as the reference computes it.
FrameParams make_params(const splat_view_desc& v, uint32_t w, uint32_t h, const float bg[3], uint32_t f);
// Sets the tile shape (powers of two), its logs and the tile grid of a frame.
void set_tile_shape(FrameParams& p, uint32_t tile_w, uint32_t tile_h);
// The handle's device scene as the kernels read it.
SceneDev scene_dev(const splat_cuda_handle* h);
// A handle for the scene shape of `d` (n, sh_degree, precision) whose scene
// arrays are allocated on the device but not filled; d's pointers are not
// read. On failure *err gets the reason.
int create_unfilled(const splat_scene_desc* d, int device, splat_cuda_handle** out, std::string* err);
// Sets the text splat_cuda_create_error reports on this thread.
void set_create_error(const std::string& msg);
// Computes the scene's binning order from its positions on the device.
int build_binning_order(splat_cuda_handle* h);

}  // namespace splat
