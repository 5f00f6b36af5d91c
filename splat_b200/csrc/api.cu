// C ABI of the B200 rasterizer (include/splat_cuda.h): scene upload, buffer
// management, the per-frame launch sequence and the host<->device boundary.
//
// One frame is: clear the frame state -> project (a) -> bin pairs into
// per-tile buckets: count, scans, ranges, scatter, sort of long tiles (b, c)
// -> per-tile depth sort + blend + downsample (c, d) -> one device-to-host
// copy of the frame and the frame state. The host never waits in the middle of a frame; pair counts
// that exceed the allocated capacity are detected from the frame state after
// the frame, the buffers grow and the frame is rendered again (the
// reference's grow-and-retry, src/render/gpu.rs:1040-1056).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/splat_cuda.h"
#include "common.cuh"
#include "handle.h"

#define SPLAT_API extern "C" __attribute__((visibility("default")))

using namespace splat;

namespace {

thread_local std::string g_create_error;

int fail(splat_cuda_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int cuda_fail(splat_cuda_handle* h, cudaError_t e, const char* what) {
  const int code = (e == cudaErrorMemoryAllocation) ? SPLAT_ERR_OOM : SPLAT_ERR_DEVICE;
  return fail(h, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(expr, what)                            \
  do {                                            \
    cudaError_t e_ = (expr);                      \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, what); \
  } while (0)

// IEEE binary16 bit pattern to binary32 (exact: every half is a float).
float half_bits_to_float(uint16_t b) {
  const uint32_t sign = (uint32_t)(b >> 15) << 31;
  const uint32_t e = (b >> 10) & 31u, m = b & 1023u;
  uint32_t bits;
  if (e == 31u) {
    bits = sign | 0x7F800000u | (m << 13);  // inf / NaN
  } else if (e != 0u) {
    bits = sign | ((e + 112u) << 23) | (m << 13);  // rebias 15 -> 127
  } else if (m == 0u) {
    bits = sign;  // signed zero
  } else {  // subnormal half: m * 2^-24, normal as a float
    int ex = -1;
    uint32_t mm = m;
    do {
      mm <<= 1;
      ex++;
    } while (!(mm & 1024u));
    bits = sign | ((uint32_t)(112 - ex) << 23) | ((mm & 1023u) << 13);
  }
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

template <class T> void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// cudaMalloc for the handle's per-frame buffers; an injected allocation
// failure (SPLAT_FAULT_ALLOC) makes the next one report out of memory
// without calling the allocator.
template <class T> cudaError_t dmalloc(splat_cuda_handle* h, T** p, size_t bytes) {
  if (h->inject_alloc) {
    h->inject_alloc = false;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

void free_pairs(splat_cuda_handle* h) {
  for (int b = 0; b < 2; b++) dfree(h->pairs[b]);
  h->cap = 0;
}

int ensure_pairs(splat_cuda_handle* h, uint64_t cap) {
  if (cap <= h->cap) return SPLAT_OK;
  if (cap > kMaxPairs) return fail(h, SPLAT_ERR_CAPACITY, "more than 2^30 - 1 gaussian/tile pairs");
  free_pairs(h);
  // Two words of slack: the blend's bulk copy of a tile rounds its end up to 16 bytes.
  for (int b = 0; b < 2; b++) CK(dmalloc(h, &h->pairs[b], (cap + 2) * sizeof(uint64_t)), "cudaMalloc pairs");
  h->cap = cap;
  return SPLAT_OK;
}

// Grows the pair buffers towards `want` pairs (at most the pair limit). When
// the device cannot hold that many, smaller capacities are tried, halving,
// down to the current one; frames that then do not fit are drawn in windows
// of tiles. Fails only when not even the current capacity can be restored.
int grow_pairs(splat_cuda_handle* h, uint64_t want) {
  want = std::min(want, h->pair_limit);
  const uint64_t old = h->cap;
  if (want <= old) return SPLAT_OK;
  for (uint64_t c = want; c > old; c /= 2) {
    const int rc = ensure_pairs(h, c);
    if (rc == SPLAT_OK) return SPLAT_OK;
    if (rc != SPLAT_ERR_OOM) return rc;
    cudaGetLastError();  // the failed allocation is not a sticky error
  }
  return ensure_pairs(h, std::max<uint64_t>(old, 1));
}

int ensure_size(splat_cuda_handle* h, uint64_t tiles, uint32_t rows, size_t out_bytes, size_t full_bytes) {
  if (tiles > h->ranges_cap) {
    dfree(h->ranges);
    dfree(h->totals);
    dfree(h->order);
    h->ranges_cap = 0;
    CK(dmalloc(h, &h->ranges, tiles * sizeof(uint2)), "cudaMalloc ranges");
    CK(dmalloc(h, &h->totals, tiles * sizeof(uint32_t)), "cudaMalloc totals");
    CK(dmalloc(h, &h->order, kTileClasses * tiles * sizeof(uint32_t)), "cudaMalloc tile classes");
    h->ranges_cap = tiles;
  }
  const size_t words = (size_t)rows * tiles;
  if (words > h->counts_cap) {  // with room for windows and record counts that vary
    const size_t cap = words + words / 4;
    dfree(h->counts);
    h->counts_cap = 0;
    CK(dmalloc(h, &h->counts, cap * sizeof(uint32_t)), "cudaMalloc counts");
    h->counts_cap = cap;
  }
  const uint32_t chunks = (uint32_t)((tiles + kScanChunk - 1) / kScanChunk);
  if (chunks > h->chunks_cap || !h->st) {
    dfree(h->st);
    h->chunks_cap = 0;
    CK(dmalloc(h, &h->st, frame_counters_bytes(1, std::max(chunks, 1u))), "cudaMalloc frame counters");
    h->chunks_cap = std::max(chunks, 1u);
  }
  if (out_bytes > h->out_cap) {
    dfree(h->out_dev);
    CK(dmalloc(h, &h->out_dev, out_bytes), "cudaMalloc frame");
    h->out_cap = out_bytes;
  }
  if (full_bytes > h->full_cap) {
    dfree(h->full_dev);
    CK(dmalloc(h, &h->full_dev, full_bytes), "cudaMalloc full-resolution frame");
    h->full_cap = full_bytes;
  }
  return SPLAT_OK;
}

bool is_device_memory(const void* p, int device) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice && a.device == device;
}

bool is_pinned_host(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// The device's address of page-locked host memory it can write directly
// (mapped pinned memory: every cudaHostAlloc / cudaMallocHost buffer under
// unified addressing), or null.
uint8_t* mapped_host(void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? static_cast<uint8_t*>(a.devicePointer) : nullptr;
}

}  // namespace

namespace splat {

// ProjectCtx::new (src/render/mod.rs:169-196) with View::rotation/focal
// (src/camera.rs:172-181), in f32 exactly as the reference computes it.
FrameParams make_params(const splat_view_desc& v, uint32_t w, uint32_t hgt, const float bg[3], uint32_t f) {
  FrameParams p{};
  for (int c = 0; c < 3; c++) {
    p.rot[c] = v.right[c];
    p.rot[3 + c] = v.down[c];
    p.rot[6 + c] = v.forward[c];
    p.eye[c] = v.eye[c];
    p.bg[c] = bg[c];
  }
  p.focal = ((float)hgt * 0.5f) / std::tan(v.fov_y * 0.5f);
  const float fw = (float)w, fh = (float)hgt;
  auto lim = [&](float half) {
    const float l = 1.3f * (half / p.focal);
    return std::isfinite(l) ? l : 0.0f;
  };
  p.cx = fw * 0.5f;
  p.cy = fh * 0.5f;
  p.width = fw;
  p.height = fh;
  p.near_plane = v.near_plane;
  p.lim_x = lim(fw * 0.5f);
  p.lim_y = lim(fh * 0.5f);
  p.w = w;
  p.h = hgt;
  p.downsample = f;
  p.out_w = w / f;
  p.out_h = hgt / f;
  p.win_y0 = 0;
  p.win_rows = hgt;
  p.out_y0 = 0;
  p.win_x0 = 0;
  p.win_cols = w;
  return p;
}

SceneDev scene_dev(const splat_cuda_handle* h) {
  SceneDev s{};
  s.pos_op = h->pos_op;
  s.cov_a = h->cov_a;
  s.cov_b = h->cov_b;
  s.color = h->color;
  s.sh = h->sh;
  s.pos_k = h->pos_k;
  s.geom16 = h->geom16;
  s.sh16 = h->sh16;
  s.n = h->n;
  s.sh_degree = h->sh_degree;
  s.fp16 = h->precision == SPLAT_PRECISION_FP16 ? 1u : 0u;
  s.lat16 = h->lat16;
  s.mlp16 = h->mlp16;
  s.learned = h->lat16 ? 1u : 0u;
  s.order = h->bin_order;
  s.lost_wait_us = 0u;
  return s;
}

// The binning order (SceneDev::order): the splats sorted by the 3D Morton
// code of their position (10 bits per axis over the positions' bounding
// box; non-finite positions first), equal codes in scene order. Computed once
// per scene from the device copy of the positions.
int build_binning_order(splat_cuda_handle* h) {
  const uint64_t n = h->n;
  if (n < 2) return SPLAT_OK;
  std::vector<float4> pos(n);
  const float4* src = h->precision == SPLAT_PRECISION_FP16 ? h->pos_k : h->pos_op;
  cudaError_t e = cudaMemcpy(pos.data(), src, n * sizeof(float4), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(h, e, "read positions");
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const float4& p : pos) {
    const float c[3] = {p.x, p.y, p.z};
    for (int k = 0; k < 3; k++)
      if (std::isfinite(c[k])) {
        lo[k] = std::min(lo[k], c[k]);
        hi[k] = std::max(hi[k], c[k]);
      }
  }
  auto spread = [](uint32_t v) {  // 10 bits -> every third bit of 30
    v &= 1023u;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
  };
  std::vector<uint64_t> key(n), tmp(n);
  for (uint64_t i = 0; i < n; i++) {
    const float c[3] = {pos[i].x, pos[i].y, pos[i].z};
    uint32_t code = 0;
    bool finite = true;
    for (int k = 0; k < 3; k++) {
      finite = finite && std::isfinite(c[k]);
      const float ext = hi[k] - lo[k];
      const float t = ext > 0.0f ? (c[k] - lo[k]) / ext : 0.0f;
      const uint32_t q = finite ? (uint32_t)std::min(1023.0f, std::max(0.0f, t * 1023.0f)) : 0u;
      code |= spread(q) << k;
    }
    key[i] = ((uint64_t)(finite ? code + 1 : 0) << 32) | i;
  }
  // LSD radix sort of the codes (bits 32..62), stable: equal codes keep scene order.
  for (int shift = 32; shift < 63; shift += 11) {
    std::vector<uint32_t> cnt(2049, 0);
    for (uint64_t k : key) cnt[((k >> shift) & 2047u) + 1]++;
    for (int d = 0; d < 2048; d++) cnt[d + 1] += cnt[d];
    for (uint64_t k : key) tmp[cnt[(k >> shift) & 2047u]++] = k;
    key.swap(tmp);
  }
  std::vector<uint32_t> order(n);
  for (uint64_t i = 0; i < n; i++) order[i] = (uint32_t)key[i];
  if (!h->bin_order && (e = cudaMalloc(&h->bin_order, n * sizeof(uint32_t))) != cudaSuccess)
    return cuda_fail(h, e, "cudaMalloc binning order");
  if ((e = cudaMemcpy(h->bin_order, order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail(h, e, "upload binning order");
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cuda_fail(h, e, "upload binning order");
  return SPLAT_OK;
}

// Tile shape of a frame: sets tile_w/h, their logs and the tile grid.
void set_tile_shape(FrameParams& p, uint32_t tile_w, uint32_t tile_h) {
  p.tile_w = tile_w;
  p.tile_h = tile_h;
  p.tile_sx = (uint32_t)__builtin_ctz(tile_w);
  p.tile_sy = (uint32_t)__builtin_ctz(tile_h);
  p.win_tx0 = p.win_x0 / tile_w;
  p.tiles_x = (p.win_x0 + p.win_cols + tile_w - 1) / tile_w - p.win_tx0;
  p.win_ty0 = p.win_y0 / tile_h;
  p.tiles_y = (p.win_y0 + p.win_rows + tile_h - 1) / tile_h - p.win_ty0;
}

}  // namespace splat

namespace {

// Enqueues one frame into dev_out (no host synchronisation); host_mapped:
// dev_out is the device address of mapped pinned host memory. While
// h->rx is set (splat_cuda_render_records) the frame draws the h->rx_n
// records at h->rx_rec: their binning input replaces the projection.
int enqueue_frame(splat_cuda_handle* h, const FrameParams& fp_in, uint8_t* dev_out, bool host_mapped = false) {
  FrameParams fp = fp_in;
  set_tile_shape(fp, h->blend.tile_w, h->blend.tile_h);
  fp.flags = (h->debug_capture ? kFrameKeepSortedPairs : 0u) |  // splat_cuda_debug_dump reads the sorted pairs
             (h->bbox_pairs ? kFrameBboxPairs : 0u);
  const uint64_t tiles = (uint64_t)fp.tiles_x * fp.tiles_y;
  const uint32_t f = fp.downsample;
  const bool scratch = f > 1 && (fp.tile_w % f != 0 || fp.tile_h % f != 0);
  const size_t full_bytes = scratch ? (size_t)fp.w * fp.h * 3 : 0;
  const bool records = h->rx;
  const uint32_t rows = bin_rows(records ? h->rx_n : h->n, h->num_sms, 1024);
  int rc = ensure_size(h, tiles, rows, 0, full_bytes);
  if (rc) return rc;
  const uint32_t chunks = (uint32_t)((tiles + kScanChunk - 1) / kScanChunk);
  cudaStream_t s = h->stream;
  CK(cudaMemsetAsync(h->st, 0, frame_counters_bytes(1, chunks), s), "clear frame state");
  const FrameCounters fc = frame_counters_at(h->st, 1);
  ViewTask t{};
  t.fp = fp;
  t.s = scene_dev(h);
  t.s.lost_wait_us = h->inject_lost_us;  // fault injection: this frame only
  h->inject_lost_us = 0;
  t.rec = h->rec;
  t.bin = h->bin;
  t.skip = h->skip;
  t.counts = h->counts;
  t.out = dev_out;
  t.full = scratch ? h->full_dev : nullptr;
  t.rows = rows;
  if (records) {
    t.s.n = h->rx_n;
    t.s.order = nullptr;  // the records' order is the scene order
    t.rec = const_cast<Record*>(h->rx_rec);
    t.bin = h->rx_bin;
    t.skip = h->rx_skip;
  }
  if (h->stage_events) CK(cudaEventRecord(h->ev[0], s), "event");
  if (records)
    CK(launch_records_bin(t, h->table, fc, s, &h->launches), "records kernel");
  else
    CK(launch_project(t, h->table, h->debug_capture ? h->dbg_proj : nullptr,
                      h->debug_capture ? h->dbg_color : nullptr, fc, s, &h->launches),
       "project kernel");
  if (h->stage_events) CK(cudaEventRecord(h->ev[1], s), "event");
  BinLaunch bl{};
  bl.n_views = 1;
  bl.bin_ctas = rows;
  bl.col_ctas = (uint32_t)((tiles + 31) / 32);
  bl.n_tiles = (uint32_t)tiles;
  bl.max_tiles = (uint32_t)tiles;
  bl.counts_all = h->counts;
  bl.counts_bytes = (size_t)rows * tiles * sizeof(uint32_t);
  CK(launch_binning(h->table, bl, h->totals, h->ranges, h->order, h->pairs[0], h->pairs[1], h->cap,
                    fc, h->num_sms, h->max_smem, s, &h->launches, !blend_sorts_tiles(h->blend)),
     "binning kernels");
  if (h->stage_events) CK(cudaEventRecord(h->ev[2], s), "event");
  CK(launch_blend(h->table, 1, (uint32_t)tiles, h->pairs[0], h->ranges, h->order, h->exact, h->blend, fc.st,
                  h->num_sms, s, &h->launches, host_mapped, h->count_evals),
     "blend kernel");
  if (scratch) CK(launch_downsample(fp, h->full_dev, dev_out, s, &h->launches), "downsample kernel");
  if (h->stage_events) CK(cudaEventRecord(h->ev[3], s), "event");
  CK(cudaMemcpyAsync(h->st_host, h->st, frame_counters_bytes(1, 0), cudaMemcpyDeviceToHost, s), "copy frame state");
  h->last_fp = fp;
  h->last_req = fp_in;
  h->last_out = dev_out;
  h->last_mapped = host_mapped;
  return SPLAT_OK;
}

// Waits for the enqueued frame and interprets its state. *regrown: 0 the
// frame is complete; 1 it needed more pairs than the buffers held, which
// have grown to hold them (draw it again); 2 it needs more pairs than the
// buffers can hold (the pair limit, or device memory): draw it in windows.
int finish_frame(splat_cuda_handle* h, splat_render_stats* stats, int* regrown) {
  *regrown = 0;
  CK(cudaStreamSynchronize(h->stream), "frame");
  const DevState& st = *h->st_host;
  if (stats) {
    stats->visible = st.visible;
    stats->overlaps = st.total_pairs;
    if (h->stage_events) {
      float a = 0, b = 0, c = 0;
      if (cudaEventElapsedTime(&a, h->ev[0], h->ev[1]) != cudaSuccess ||
          cudaEventElapsedTime(&b, h->ev[1], h->ev[2]) != cudaSuccess ||
          cudaEventElapsedTime(&c, h->ev[2], h->ev[3]) != cudaSuccess)
        cudaGetLastError();  // stage times unavailable; do not leave the error pending
      stats->project_ms = a;
      stats->sort_ms = b;
      stats->raster_ms = c;
    }
  }
  if (st.error) {
    const unsigned code = st.error;
    cudaMemsetAsync(h->st, 0, sizeof(DevState), h->stream);
    return fail(h, SPLAT_ERR_TIMEOUT,
                code == 2u   ? "the projection's bulk copies did not complete in time"
                : code == 3u ? "the blend's bulk copy of a tile's pairs did not complete in time"
                             : "a tensor-core wait in the learned-colour projection gave up");
  }
  h->have_frame = true;
  if (st.total_pairs > h->cap) {
    const uint64_t total = st.total_pairs;
    const int rc = grow_pairs(h, std::max<uint64_t>(total + total / 4, h->cap + 1));
    if (rc) return rc;
    *regrown = h->cap >= total ? 1 : 2;
  }
  return SPLAT_OK;
}

// Draws the frame `req` (a whole frame or a window of rows) into `target`
// as windows of whole tiles whose pairs fit the buffers: bands of tile rows
// sized from the frame's pair count, a band that still overflows split in
// two (by tile rows, then by tile columns), each window a complete
// projection plus the binning, sorts and blend of its own tiles, written in
// place into the frame. Every pixel sees the same splats in the same order
// as in one pass, so the frame is identical to the one-pass frame. stats:
// the visible splats of the frame, the pairs and stage times summed over
// the windows. Fails (SPLAT_ERR_CAPACITY) only if a single tile holds more
// pairs than the buffers can.
int render_windows(splat_cuda_handle* h, FrameParams req, uint8_t* target, bool mapped, splat_render_stats* stats) {
  struct Win {
    uint32_t y0, y1, x0, x1;
  };
  const uint32_t tw = h->blend.tile_w, th = h->blend.tile_h;
  const uint32_t y0 = req.win_y0, y1 = req.win_y0 + req.win_rows;
  const uint32_t ty0 = y0 / th, nty = (y1 + th - 1) / th - ty0;
  const uint64_t per = std::max<uint64_t>(h->cap - h->cap / 4, 1);
  const uint64_t bands = std::min<uint64_t>(nty, std::max<uint64_t>(2, (h->st_host->total_pairs + per - 1) / per));
  std::vector<Win> todo;
  for (uint64_t b = bands; b-- > 0;) {
    const uint32_t a = std::max(y0, (uint32_t)((ty0 + b * nty / bands) * th));
    const uint32_t e = std::min(y1, (uint32_t)((ty0 + (b + 1) * nty / bands) * th));
    if (e > a) todo.push_back({a, e, 0u, req.w});
  }
  splat_render_stats sum{};
  int rc = SPLAT_OK;
  uint32_t passes = 0;
  while (!todo.empty()) {
    const Win w = todo.back();
    todo.pop_back();
    FrameParams fp = req;
    fp.win_y0 = w.y0;
    fp.win_rows = w.y1 - w.y0;
    fp.win_x0 = w.x0;
    fp.win_cols = w.x1 - w.x0;
    if ((rc = enqueue_frame(h, fp, target, mapped))) break;
    splat_render_stats ws{};
    int rg = 0;
    if ((rc = finish_frame(h, &ws, &rg))) break;
    if (rg == 1 && ++passes < 64) {  // the buffers grew: this window again
      todo.push_back(w);
      continue;
    }
    if (rg) {  // split: by tile rows while there are several, then by tile columns
      const uint32_t r0 = w.y0 / th, nr = (w.y1 + th - 1) / th - r0;
      const uint32_t c0 = w.x0 / tw, nc = (w.x1 + tw - 1) / tw - c0;
      if (nr > 1) {
        const uint32_t m = (r0 + nr / 2) * th;
        todo.push_back({m, w.y1, w.x0, w.x1});
        todo.push_back({w.y0, m, w.x0, w.x1});
      } else if (nc > 1) {
        const uint32_t m = (c0 + nc / 2) * tw;
        todo.push_back({w.y0, w.y1, m, w.x1});
        todo.push_back({w.y0, w.y1, w.x0, m});
      } else {
        rc = fail(h, SPLAT_ERR_CAPACITY, "one tile holds more (splat, tile) pairs than the pair buffers can");
        break;
      }
      continue;
    }
    sum.visible = ws.visible;
    sum.overlaps += ws.overlaps;
    sum.project_ms += ws.project_ms;
    sum.sort_ms += ws.sort_ms;
    sum.raster_ms += ws.raster_ms;
  }
  h->last_req = req;
  h->last_out = target;
  h->last_mapped = mapped;
  if (rc == SPLAT_OK && stats) *stats = sum;
  return rc;
}

int check_view_args(splat_cuda_handle* h, const splat_view_desc* view, uint32_t w, uint32_t hgt, const float* bg) {
  if (!h) return SPLAT_ERR_INVALID_ARG;
  if (!view || !bg) return fail(h, SPLAT_ERR_INVALID_ARG, "null view or background");
  if (w > SPLAT_MAX_DIM || hgt > SPLAT_MAX_DIM)
    return fail(h, SPLAT_ERR_INVALID_ARG,
                "frame " + std::to_string(w) + "x" + std::to_string(hgt) + " exceeds the 16384 pixel limit");
  return SPLAT_OK;
}

int check_frame_args(splat_cuda_handle* h, const splat_view_desc* view, uint32_t w, uint32_t hgt, const float* bg,
                     uint32_t f, size_t out_bytes, const void* out) {
  const int rc = check_view_args(h, view, w, hgt, bg);
  if (rc) return rc;
  if (f == 0) f = 1;
  const size_t need = (size_t)(w / f) * (hgt / f) * 3;
  if (need && (!out || out_bytes < need))
    return fail(h, SPLAT_ERR_INVALID_ARG, "output buffer smaller than floor(w/f)*floor(h/f)*3 bytes");
  return SPLAT_OK;
}

}  // namespace

SPLAT_API int splat_cuda_abi_version(void) { return SPLAT_CUDA_ABI_VERSION; }

SPLAT_API const char* splat_cuda_backend_name(void) { return "cuda"; }

SPLAT_API const char* splat_cuda_create_error(void) { return g_create_error.c_str(); }

namespace {

// splat_cuda_create; with upload = false the scene's device arrays are
// allocated but not filled (the caller fills them on the device) and the
// desc's array pointers are not read.
int create_impl(const splat_scene_desc* d, int device, splat_cuda_handle** out, bool upload) {
  g_create_error.clear();
  if (!out) return SPLAT_ERR_INVALID_ARG;
  *out = nullptr;
  if (!d) {
    g_create_error = "null scene";
    return SPLAT_ERR_INVALID_ARG;
  }
  if (d->sh_degree > 3) {
    g_create_error = "sh_degree must be 0..3";
    return SPLAT_ERR_INVALID_ARG;
  }
  if (d->precision != SPLAT_PRECISION_FP32 && d->precision != SPLAT_PRECISION_FP16) {
    g_create_error = "unknown scene precision";
    return SPLAT_ERR_UNSUPPORTED;
  }
  if (d->n > 0xFFFFFFFFull) {
    g_create_error = "more than 2^32 - 1 gaussians";
    return SPLAT_ERR_INVALID_ARG;
  }
  const uint64_t n = d->n;
  const bool f16 = d->precision == SPLAT_PRECISION_FP16;
  if (upload && n && !f16 &&
      (!d->positions || !d->opacities || !d->colors || !d->cov3d || (d->sh_degree && !d->sh_rest))) {
    g_create_error = "null scene array";
    return SPLAT_ERR_INVALID_ARG;
  }
  if (upload && n && f16 && (!d->positions || !d->scales_f16 || !d->rotations_f16 || !d->opacities_f16 || !d->sh_f16)) {
    g_create_error = "null FP16 scene array";
    return SPLAT_ERR_INVALID_ARG;
  }
  auto* h = new splat_cuda_handle();
  auto bail = [&](int rc) {
    g_create_error = h->err;
    splat_cuda_destroy(h);
    return rc;
  };
  h->device = device;
  h->n = n;
  h->sh_degree = d->sh_degree;
  h->precision = d->precision;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return bail(cuda_fail(h, e, "cudaSetDevice"));
  e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return bail(cuda_fail(h, e, "device attributes"));
  int optin = 0;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (e != cudaSuccess) return bail(cuda_fail(h, e, "device attributes"));
  h->max_smem = (size_t)optin;
  if ((e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(cuda_fail(h, e, "cudaStreamCreate"));
  h->stream = h->own_stream;
  for (auto& ev : h->ev)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return bail(cuda_fail(h, e, "cudaEventCreate"));
  if ((e = cudaMalloc(&h->table, sizeof(ViewTask))) != cudaSuccess) return bail(cuda_fail(h, e, "cudaMalloc views"));
  if ((e = cudaMallocHost(&h->st_host, frame_counters_bytes(1, 0))) != cudaSuccess)
    return bail(cuda_fail(h, e, "cudaMallocHost state"));
  std::memset(h->st_host, 0, frame_counters_bytes(1, 0));

  if (n && f16) {
    // FP16 layout, 128 bytes per splat: float4 (pos, k); 8 halves (scale xyz,
    // rotation xyzw, opacity) as one uint4; base colour and SH as planes of n
    // halves. k is computed from the decoded opacity as in the FP32 layout.
    const uint32_t planes = d->sh_degree ? (d->sh_degree + 1) * (d->sh_degree + 1) * 3 : 3;
    std::vector<float4> pk(upload ? n : 0);
    std::vector<uint4> g(upload ? n : 0);
    for (uint64_t i = 0; upload && i < n; i++) {
      const float* p = d->positions + 3 * i;
      const uint16_t* sc = d->scales_f16 + 3 * i;
      const uint16_t* q = d->rotations_f16 + 4 * i;
      const uint16_t ob = d->opacities_f16[i];
      const float o = std::fmin(std::fmax(half_bits_to_float(ob), 0.0f), 1.0f);  // as the device clamps it
      const float k = o < kAlphaMin ? 0.0f : std::sqrt(2.0f * std::log(o / kAlphaMin));
      pk[i] = make_float4(p[0], p[1], p[2], k);
      g[i] = make_uint4(sc[0] | ((uint32_t)sc[1] << 16), sc[2] | ((uint32_t)q[0] << 16), q[1] | ((uint32_t)q[2] << 16),
                        q[3] | ((uint32_t)ob << 16));
    }
    std::vector<uint16_t> sh(upload ? (size_t)planes * n : 0);
    for (uint64_t i = 0; upload && i < n; i++)
      for (uint32_t k = 0; k < planes; k++) sh[(size_t)k * n + i] = d->sh_f16[i * planes + k];
    auto up = [&](void** dst, const void* src, size_t bytes, const char* what) -> int {
      cudaError_t er = cudaMalloc(dst, bytes);
      if (er != cudaSuccess) return cuda_fail(h, er, what);
      if (!upload) return SPLAT_OK;
      er = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
      if (er != cudaSuccess) return cuda_fail(h, er, what);
      return SPLAT_OK;
    };
    int rc;
    if ((rc = up((void**)&h->pos_k, pk.data(), n * sizeof(float4), "upload positions"))) return bail(rc);
    if ((rc = up((void**)&h->geom16, g.data(), n * sizeof(uint4), "upload FP16 geometry"))) return bail(rc);
    if ((rc = up((void**)&h->sh16, sh.data(), (size_t)planes * n * sizeof(uint16_t), "upload FP16 SH")))
      return bail(rc);
    if ((e = cudaMalloc(&h->rec, n * sizeof(Record))) != cudaSuccess) return bail(cuda_fail(h, e, "cudaMalloc records"));
    if ((e = cudaMalloc(&h->bin, n * sizeof(BinInfo))) != cudaSuccess ||
        (e = cudaMalloc(&h->skip, n * sizeof(BinSkip))) != cudaSuccess) return bail(cuda_fail(h, e, "cudaMalloc bins"));
  } else if (n) {
    // Upload in the device layout: float4 (pos, opacity), float4 + float4 for
    // the covariance (with k = sqrt(2 ln(opacity / ALPHA_MIN)), the bbox
    // radius the reference's cpu backend also precomputes, cpu.rs:384-388),
    // colour and SH as planes of n floats for coalesced loads.
    const uint32_t rest = d->sh_degree ? (d->sh_degree + 1) * (d->sh_degree + 1) - 1 : 0;
    std::vector<float4> a(upload ? n : 0), b(upload ? n : 0), c(upload ? n : 0);
    for (uint64_t i = 0; upload && i < n; i++) {
      const float* p = d->positions + 3 * i;
      const float o = d->opacities[i];
      a[i] = make_float4(p[0], p[1], p[2], o);
      const float* cv = d->cov3d + 6 * i;
      b[i] = make_float4(cv[0], cv[1], cv[2], cv[3]);
      const float k = o < kAlphaMin ? 0.0f : std::sqrt(2.0f * std::log(o / kAlphaMin));
      c[i] = make_float4(cv[4], cv[5], k, 0.0f);
    }
    std::vector<float> col(upload ? 3 * n : 0);
    for (uint64_t i = 0; upload && i < n; i++)
      for (int ch = 0; ch < 3; ch++) col[ch * n + i] = d->colors[3 * i + ch];
    // 16 bytes of slack after every array: the projection's bulk copies
    // round a plane's slice out to 16-byte boundaries.
    auto up = [&](void** dst, const void* src, size_t bytes, const char* what) -> int {
      cudaError_t er = cudaMalloc(dst, bytes + 16);
      if (er != cudaSuccess) return cuda_fail(h, er, what);
      if (!upload) return SPLAT_OK;
      er = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
      if (er != cudaSuccess) return cuda_fail(h, er, what);
      return SPLAT_OK;
    };
    int rc;
    if ((rc = up((void**)&h->pos_op, a.data(), n * sizeof(float4), "upload positions"))) return bail(rc);
    if ((rc = up((void**)&h->cov_a, b.data(), n * sizeof(float4), "upload covariance"))) return bail(rc);
    if ((rc = up((void**)&h->cov_b, c.data(), n * sizeof(float4), "upload covariance"))) return bail(rc);
    if ((rc = up((void**)&h->color, col.data(), 3 * n * sizeof(float), "upload colours"))) return bail(rc);
    if (rest) {
      std::vector<float> sh(upload ? (size_t)rest * 3 * n : 0);
      for (uint64_t i = 0; upload && i < n; i++)
        for (uint32_t k = 0; k < rest * 3; k++) sh[(size_t)k * n + i] = d->sh_rest[i * rest * 3 + k];
      if ((rc = up((void**)&h->sh, sh.data(), (size_t)rest * 3 * n * sizeof(float), "upload SH"))) return bail(rc);
    }
    if ((e = cudaMalloc(&h->rec, n * sizeof(Record))) != cudaSuccess) return bail(cuda_fail(h, e, "cudaMalloc records"));
    if ((e = cudaMalloc(&h->bin, n * sizeof(BinInfo))) != cudaSuccess ||
        (e = cudaMalloc(&h->skip, n * sizeof(BinSkip))) != cudaSuccess) return bail(cuda_fail(h, e, "cudaMalloc bins"));

  }
  int rc = ensure_pairs(h, std::max<uint64_t>(4 * n, 1u << 16));
  if (rc) return bail(rc);
  // A cudaMemcpy from pageable memory may return before its DMA has landed,
  // and the handle's stream does not wait for the legacy stream that carries
  // it: the scene must be on the device before the first kernel reads it.
  if (upload && (e = cudaDeviceSynchronize()) != cudaSuccess) return bail(cuda_fail(h, e, "upload scene"));
  if (upload && (rc = build_binning_order(h))) return bail(rc);
  *out = h;
  return SPLAT_OK;
}

}  // namespace

SPLAT_API int splat_cuda_create(const splat_scene_desc* d, int device, splat_cuda_handle** out) {
  return create_impl(d, device, out, true);
}

namespace splat {
int create_unfilled(const splat_scene_desc* d, int device, splat_cuda_handle** out, std::string* err) {
  const int rc = create_impl(d, device, out, false);
  if (rc && err) *err = g_create_error;
  return rc;
}
void set_create_error(const std::string& msg) { g_create_error = msg; }
}  // namespace splat

SPLAT_API int splat_cuda_render_device(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width,
                                       uint32_t height, const float bg[3], uint32_t downsample, uint8_t* dev_out,
                                       size_t out_bytes) {
  int rc = check_frame_args(h, view, width, height, bg, downsample, out_bytes, dev_out);
  if (rc) return rc;
  if (width == 0 || height == 0) return SPLAT_OK;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  const uint32_t f = downsample ? downsample : 1;
  return enqueue_frame(h, make_params(*view, width, height, bg, f), dev_out);
}

SPLAT_API int splat_cuda_finish(splat_cuda_handle* h, splat_render_stats* stats, int* regrown) {
  if (!h) return SPLAT_ERR_INVALID_ARG;
  int dummy = 0;
  if (!regrown) regrown = &dummy;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  int rc = finish_frame(h, stats, regrown);
  if (rc == SPLAT_OK && *regrown == 2) {
    // More pairs than the buffers can hold: the frame is drawn again, in
    // windows, into the same destination before this call returns.
    *regrown = 0;
    rc = render_windows(h, h->last_req, h->last_out, h->last_mapped, stats);
  }
  return rc;
}

namespace {

// A frame (or a window of rows) into caller-owned host memory (or, with
// device_ok, device memory of the handle's device, written in place): bytes
// = out_w * out_h * 3 of fp.
int render_to_host(splat_cuda_handle* h, const FrameParams& fp, uint8_t* rgb_out, splat_render_stats* stats,
                   std::chrono::steady_clock::time_point t0, bool device_ok = false) {
  int rc = SPLAT_OK;
  const size_t bytes = (size_t)fp.out_w * fp.out_h * 3;
  if (bytes && device_ok && is_device_memory(rgb_out, h->device)) {
    for (int attempt = 0; attempt < 8; attempt++) {
      if ((rc = enqueue_frame(h, fp, rgb_out))) return rc;
      int regrown = 0;
      if ((rc = finish_frame(h, stats, &regrown))) return rc;
      if (regrown == 2) {
        if ((rc = render_windows(h, fp, rgb_out, false, stats))) return rc;
        CK(cudaStreamSynchronize(h->stream), "frame");
        regrown = 0;
      }
      if (!regrown) {
        if (stats)
          stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return SPLAT_OK;
      }
    }
    return fail(h, SPLAT_ERR_CAPACITY, "pair buffers kept overflowing");
  }
  if ((rc = ensure_size(h, 0, 0, bytes, 0))) return rc;
  // Pinned output the device can address: the default blend writes the
  // frame straight into it as whole words of tile rows, overlapped with the
  // frame's own compute, instead of a copy after the frame. Other blend
  // configurations, the exact blend and downsampled frames (whose stores
  // would cross the host link byte by byte) draw into device memory and copy
  // the frame, as other pinned memory does; pageable memory goes through the
  // handle's pinned staging buffer.
  const bool rows_ok = fp.downsample == 1 && blend_writes_host_rows(h->blend, h->exact);
  uint8_t* const mapped = bytes && rows_ok ? mapped_host(rgb_out) : nullptr;
  const bool direct = bytes && (mapped || is_pinned_host(rgb_out));
  if (!direct && bytes > h->stage_cap) {
    if (h->stage) cudaFreeHost(h->stage);
    h->stage = nullptr;
    h->stage_cap = 0;
    CK(cudaMallocHost(&h->stage, bytes), "cudaMallocHost staging");
    h->stage_cap = bytes;
  }
  for (int attempt = 0; attempt < 8; attempt++) {
    if ((rc = enqueue_frame(h, fp, mapped ? mapped : h->out_dev, mapped != nullptr))) return rc;
    if (bytes && !mapped)
      CK(cudaMemcpyAsync(direct ? rgb_out : h->stage, h->out_dev, bytes, cudaMemcpyDeviceToHost, h->stream),
         "copy frame");
    int regrown = 0;
    if ((rc = finish_frame(h, stats, &regrown))) return rc;
    if (regrown == 2) {  // more pairs than the buffers can hold: windows of tiles
      if ((rc = render_windows(h, fp, mapped ? mapped : h->out_dev, mapped != nullptr, stats))) return rc;
      if (bytes && !mapped)
        CK(cudaMemcpyAsync(direct ? rgb_out : h->stage, h->out_dev, bytes, cudaMemcpyDeviceToHost, h->stream),
           "copy frame");
      CK(cudaStreamSynchronize(h->stream), "frame");
      regrown = 0;
    }
    if (!regrown) {
      if (!direct && bytes) std::memcpy(rgb_out, h->stage, bytes);
      if (stats)
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      return SPLAT_OK;
    }
  }
  return fail(h, SPLAT_ERR_CAPACITY, "pair buffers kept overflowing");
}

}  // namespace

SPLAT_API int splat_cuda_render(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width, uint32_t height,
                                const float bg[3], uint32_t downsample, uint8_t* rgb_out, size_t out_bytes,
                                splat_render_stats* stats) {
  const auto t0 = std::chrono::steady_clock::now();
  if (stats) std::memset(stats, 0, sizeof(*stats));
  int rc = check_frame_args(h, view, width, height, bg, downsample, out_bytes, rgb_out);
  if (rc) return rc;
  if (width == 0 || height == 0) return SPLAT_OK;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  const uint32_t f = downsample ? downsample : 1;
  return render_to_host(h, make_params(*view, width, height, bg, f), rgb_out, stats, t0);
}

SPLAT_API int splat_cuda_render_rows(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width,
                                     uint32_t height, const float bg[3], uint32_t row0, uint32_t rows,
                                     uint8_t* rgb_out, size_t out_bytes, splat_render_stats* stats) {
  const auto t0 = std::chrono::steady_clock::now();
  if (stats) std::memset(stats, 0, sizeof(*stats));
  int rc = check_view_args(h, view, width, height, bg);
  if (rc) return rc;
  if ((uint64_t)row0 + rows > height)
    return fail(h, SPLAT_ERR_INVALID_ARG, "rows [row0, row0 + rows) exceed the frame height");
  const size_t need = (size_t)width * rows * 3;
  if (need && (!rgb_out || out_bytes < need))
    return fail(h, SPLAT_ERR_INVALID_ARG, "output buffer smaller than width*rows*3 bytes");
  if (need == 0) return SPLAT_OK;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  FrameParams fp = make_params(*view, width, height, bg, 1);
  fp.win_y0 = row0;
  fp.win_rows = rows;
  fp.out_y0 = row0;
  fp.out_h = rows;
  return render_to_host(h, fp, rgb_out, stats, t0);
}

SPLAT_API int splat_cuda_shard_records(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width,
                                       uint32_t height, uint32_t n_windows, const uint32_t* row_bounds, void* send,
                                       uint64_t send_capacity, uint64_t* counts, uint64_t* visible) {
  if (visible) *visible = 0;
  const float bg[3] = {0.0f, 0.0f, 0.0f};
  int rc = check_view_args(h, view, width, height, bg);
  if (rc) return rc;
  if (n_windows == 0 || n_windows > kMaxShardWindows || !row_bounds || !counts)
    return fail(h, SPLAT_ERR_INVALID_ARG, "1 to 64 row windows, their n + 1 bounds and a counts array of n");
  ShardWindows w{};
  w.n = n_windows;
  for (uint32_t k = 0; k <= n_windows; k++) {
    if (row_bounds[k] > height || (k && row_bounds[k] < row_bounds[k - 1]))
      return fail(h, SPLAT_ERR_INVALID_ARG, "row window bounds must be nondecreasing and at most the frame height");
    w.bound[k] = row_bounds[k];
  }
  if (send_capacity && (!send || (reinterpret_cast<uintptr_t>(send) & 15u) || !is_device_memory(send, h->device)))
    return fail(h, SPLAT_ERR_INVALID_ARG, "the send buffer must be 16-byte aligned device memory of the handle's device");
  for (uint32_t k = 0; k < n_windows; k++) counts[k] = 0;
  if (width == 0 || height == 0 || h->n == 0) return SPLAT_OK;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  const size_t scratch = shard_scratch_bytes(h->n, n_windows);
  if (scratch > h->shard_scratch_cap) {
    dfree(h->shard_scratch);
    h->shard_scratch_cap = 0;
    CK(dmalloc(h, reinterpret_cast<uint8_t**>(&h->shard_scratch), scratch), "cudaMalloc record selection");
    h->shard_scratch_cap = scratch;
  }
  const size_t totals_bytes = kMaxShardWindows * sizeof(unsigned long long);
  if (!h->shard_totals) CK(dmalloc(h, &h->shard_totals, totals_bytes), "cudaMalloc record totals");
  if (!h->shard_totals_host) CK(cudaMallocHost(&h->shard_totals_host, totals_bytes), "cudaMallocHost record totals");
  if ((rc = ensure_size(h, 0, 0, 0, 0))) return rc;  // the frame counters
  FrameParams fp = make_params(*view, width, height, bg, 1);
  set_tile_shape(fp, h->blend.tile_w, h->blend.tile_h);
  cudaStream_t s = h->stream;
  CK(cudaMemsetAsync(h->st, 0, frame_counters_bytes(1, 0), s), "clear frame state");
  const FrameCounters fc = frame_counters_at(h->st, 1);
  ViewTask t{};
  t.fp = fp;
  t.s = scene_dev(h);
  t.s.lost_wait_us = h->inject_lost_us;
  h->inject_lost_us = 0;
  t.rec = h->rec;
  t.bin = h->bin;
  t.skip = h->skip;
  CK(launch_project(t, h->table, nullptr, nullptr, fc, s, &h->launches), "project kernel");
  CK(launch_shard_count(h->rec, h->bin, h->n, w, h->shard_scratch, h->shard_totals, s, &h->launches),
     "record selection kernels");
  CK(cudaMemcpyAsync(h->shard_totals_host, h->shard_totals, n_windows * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, s),
     "copy record totals");
  CK(cudaMemcpyAsync(h->st_host, h->st, sizeof(DevState), cudaMemcpyDeviceToHost, s), "copy frame state");
  CK(cudaStreamSynchronize(s), "record selection");
  if (h->st_host->error) {
    const unsigned code = h->st_host->error;
    cudaMemsetAsync(h->st, 0, sizeof(DevState), s);
    return fail(h, SPLAT_ERR_TIMEOUT,
                code == 2u ? "the projection's bulk copies did not complete in time"
                           : "a tensor-core wait in the learned-colour projection gave up");
  }
  uint64_t total = 0;
  for (uint32_t k = 0; k < n_windows; k++) total += (counts[k] = h->shard_totals_host[k]);
  if (visible) *visible = h->st_host->visible;
  if (total > send_capacity)
    return fail(h, SPLAT_ERR_CAPACITY,
                "the send buffer holds " + std::to_string(send_capacity) + " records, the windows take " +
                    std::to_string(total) + " (counts are filled in)");
  if (total) {
    CK(launch_shard_scatter(h->rec, h->bin, h->n, w, h->shard_scratch, h->shard_totals, static_cast<Record*>(send),
                            send_capacity, s, &h->launches),
       "record scatter kernel");
    CK(cudaStreamSynchronize(s), "record scatter");
  }
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_render_records(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width,
                                        uint32_t height, const float bg[3], const void* records, uint64_t n_records,
                                        uint32_t row0, uint32_t rows, uint8_t* out, size_t out_bytes,
                                        splat_render_stats* stats) {
  const auto t0 = std::chrono::steady_clock::now();
  if (stats) std::memset(stats, 0, sizeof(*stats));
  int rc = check_view_args(h, view, width, height, bg);
  if (rc) return rc;
  if ((uint64_t)row0 + rows > height)
    return fail(h, SPLAT_ERR_INVALID_ARG, "rows [row0, row0 + rows) exceed the frame height");
  const size_t need = (size_t)width * rows * 3;
  if (need && (!out || out_bytes < need))
    return fail(h, SPLAT_ERR_INVALID_ARG, "output buffer smaller than width*rows*3 bytes");
  if (n_records && (!records || (reinterpret_cast<uintptr_t>(records) & 15u) || !is_device_memory(records, h->device)))
    return fail(h, SPLAT_ERR_INVALID_ARG, "the records must be 16-byte aligned device memory of the handle's device");
  if (n_records > 0xFFFFFFFFull) return fail(h, SPLAT_ERR_INVALID_ARG, "more than 2^32 - 1 records");
  if (need == 0) return SPLAT_OK;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  const uint64_t slots = std::max<uint64_t>(n_records, 1);
  if (slots > h->rx_bin_cap) {  // with room for the next frames' counts to vary
    const uint64_t cap = slots + slots / 4;
    dfree(h->rx_bin);
    dfree(h->rx_skip);
    h->rx_bin_cap = 0;
    CK(dmalloc(h, &h->rx_bin, cap * sizeof(BinInfo)), "cudaMalloc record binning input");
    CK(dmalloc(h, &h->rx_skip, cap * sizeof(BinSkip)), "cudaMalloc record binning input");
    h->rx_bin_cap = cap;
  }
  FrameParams fp = make_params(*view, width, height, bg, 1);
  fp.win_y0 = row0;
  fp.win_rows = rows;
  fp.out_y0 = row0;
  fp.out_h = rows;
  h->rx = true;
  h->rx_rec = static_cast<const Record*>(records);
  h->rx_n = n_records;
  rc = render_to_host(h, fp, out, stats, t0, true);
  h->rx = false;
  h->rx_rec = nullptr;
  h->rx_n = 0;
  return rc;
}

SPLAT_API int splat_cuda_render_cells(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width,
                                      uint32_t height, const float bg[3], uint32_t downsample, uint32_t mode,
                                      uint8_t* cells_out, size_t out_bytes, uint32_t* cols, uint32_t* rows,
                                      splat_render_stats* stats) {
  const auto t0 = std::chrono::steady_clock::now();
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (!h) return SPLAT_ERR_INVALID_ARG;
  if (mode != SPLAT_CELLS_TRUECOLOR && mode != SPLAT_CELLS_ANSI256)
    return fail(h, SPLAT_ERR_INVALID_ARG, "unknown cell colour mode");
  const uint32_t f = downsample ? downsample : 1;
  const uint32_t nc = width / f, nr = (height / f) / 2;
  const size_t need = (size_t)nc * nr * (mode == SPLAT_CELLS_TRUECOLOR ? 6 : 2);
  if (cols) *cols = nc;
  if (rows) *rows = nr;
  int rc = check_frame_args(h, view, width, height, bg, downsample, (size_t)-1, h);
  if (rc) return rc;
  if (need && (!cells_out || out_bytes < need))
    return fail(h, SPLAT_ERR_INVALID_ARG, "cell buffer smaller than cols * rows * bytes per cell");
  if (width == 0 || height == 0) return SPLAT_OK;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  const FrameParams fp = make_params(*view, width, height, bg, f);
  if ((rc = ensure_size(h, 0, 0, (size_t)fp.out_w * fp.out_h * 3, 0))) return rc;
  if (need > h->cells_cap) {
    if (h->cells_dev) cudaFree(h->cells_dev);
    h->cells_dev = nullptr;
    h->cells_cap = 0;
    CK(dmalloc(h, &h->cells_dev, need), "cudaMalloc cells");
    h->cells_cap = need;
  }
  const bool direct = need && is_pinned_host(cells_out);
  if (!direct && need > h->stage_cap) {
    if (h->stage) cudaFreeHost(h->stage);
    h->stage = nullptr;
    h->stage_cap = 0;
    CK(cudaMallocHost(&h->stage, need), "cudaMallocHost staging");
    h->stage_cap = need;
  }
  for (int attempt = 0; attempt < 8; attempt++) {
    if ((rc = enqueue_frame(h, fp, h->out_dev))) return rc;
    CK(launch_cells(h->out_dev, fp.out_w, nc, nr, mode, h->cells_dev, h->stream, &h->launches), "cells kernel");
    if (need)
      CK(cudaMemcpyAsync(direct ? cells_out : h->stage, h->cells_dev, need, cudaMemcpyDeviceToHost, h->stream),
         "copy cells");
    int regrown = 0;
    if ((rc = finish_frame(h, stats, &regrown))) return rc;
    if (regrown == 2) {  // more pairs than the buffers can hold: windows of tiles
      if ((rc = render_windows(h, fp, h->out_dev, false, stats))) return rc;
      CK(launch_cells(h->out_dev, fp.out_w, nc, nr, mode, h->cells_dev, h->stream, &h->launches), "cells kernel");
      if (need)
        CK(cudaMemcpyAsync(direct ? cells_out : h->stage, h->cells_dev, need, cudaMemcpyDeviceToHost, h->stream),
           "copy cells");
      CK(cudaStreamSynchronize(h->stream), "frame");
      regrown = 0;
    }
    if (!regrown) {
      if (!direct && need) std::memcpy(cells_out, h->stage, need);
      if (stats)
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      return SPLAT_OK;
    }
  }
  return fail(h, SPLAT_ERR_CAPACITY, "pair buffers kept overflowing");
}

SPLAT_API int splat_cuda_set_stream(splat_cuda_handle* h, void* stream) {
  if (!h) return SPLAT_ERR_INVALID_ARG;
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return SPLAT_OK;
}

SPLAT_API void* splat_cuda_get_stream(splat_cuda_handle* h) { return h ? (void*)h->stream : nullptr; }

SPLAT_API int splat_cuda_set_option(splat_cuda_handle* h, uint32_t option, uint64_t value) {
  if (!h) return SPLAT_ERR_INVALID_ARG;
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  switch (option) {
    case SPLAT_OPT_EXACT_BLEND:
      h->exact = value != 0;
      return SPLAT_OK;
    case SPLAT_OPT_PAIR_CAPACITY: {
      if (value == 0 || value > h->pair_limit)
        return fail(h, SPLAT_ERR_INVALID_ARG, "pair capacity out of range (1 .. the pair limit)");
      // Shrinking is allowed: reallocate at exactly `value`.
      free_pairs(h);
      return ensure_pairs(h, value);
    }
    case SPLAT_OPT_PAIR_LIMIT: {
      if (value < 1024 || value > kMaxPairs) return fail(h, SPLAT_ERR_INVALID_ARG, "pair limit out of range");
      h->pair_limit = value;
      if (h->cap > value) {  // the buffers shrink to the new limit
        free_pairs(h);
        return ensure_pairs(h, value);
      }
      return SPLAT_OK;
    }
    case SPLAT_OPT_STAGE_EVENTS:
      h->stage_events = value != 0;
      return SPLAT_OK;
    case SPLAT_OPT_BBOX_PAIRS:
      h->bbox_pairs = value != 0;
      return SPLAT_OK;
    case SPLAT_OPT_COUNT_EVALS:
      h->count_evals = value != 0;
      return SPLAT_OK;
    case SPLAT_OPT_BLEND_EVALS:
      return fail(h, SPLAT_ERR_INVALID_ARG, "SPLAT_OPT_BLEND_EVALS is read-only");
    case SPLAT_OPT_FP64_CONICS:
      return fail(h, SPLAT_ERR_INVALID_ARG, "SPLAT_OPT_FP64_CONICS is read-only");
    case SPLAT_OPT_KERNEL_LAUNCHES:
      h->launches = (uint32_t)value;
      return SPLAT_OK;
    case SPLAT_OPT_BLEND_CONFIG: {
      const BlendConfig c{(uint32_t)(value & 0xFF), (uint32_t)((value >> 8) & 0xFF), (uint32_t)(value >> 16)};
      if (!blend_config_supported(c)) return fail(h, SPLAT_ERR_UNSUPPORTED, "unsupported tile shape or thread count");
      h->blend = c;
      return SPLAT_OK;
    }
    case SPLAT_OPT_INJECT_FAULT:
      switch (value & 0xFFu) {
        case 0: h->inject_alloc = false; h->inject_lost_us = 0; return SPLAT_OK;
        case SPLAT_FAULT_ALLOC: h->inject_alloc = true; return SPLAT_OK;
        case SPLAT_FAULT_LOST_WAIT:
          h->inject_lost_us = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(value >> 8, 10000000ull));
          return SPLAT_OK;
        default: return fail(h, SPLAT_ERR_UNSUPPORTED, "unknown fault kind");
      }
    case SPLAT_OPT_DEBUG_CAPTURE: {
      h->debug_capture = value != 0;
      if (h->debug_capture && h->n && !h->dbg_proj) {
        CK(cudaMalloc(&h->dbg_proj, h->n * 8 * sizeof(float)), "cudaMalloc debug");
        CK(cudaMalloc(&h->dbg_color, h->n * 3 * sizeof(float)), "cudaMalloc debug");
      }
      return SPLAT_OK;
    }
    default:
      return fail(h, SPLAT_ERR_UNSUPPORTED, "unknown option");
  }
}

SPLAT_API int splat_cuda_get_option(splat_cuda_handle* h, uint32_t option, uint64_t* value) {
  if (!h || !value) return SPLAT_ERR_INVALID_ARG;
  switch (option) {
    case SPLAT_OPT_EXACT_BLEND: *value = h->exact; return SPLAT_OK;
    case SPLAT_OPT_PAIR_CAPACITY: *value = h->cap; return SPLAT_OK;
    case SPLAT_OPT_PAIR_LIMIT: *value = h->pair_limit; return SPLAT_OK;
    case SPLAT_OPT_STAGE_EVENTS: *value = h->stage_events; return SPLAT_OK;
    case SPLAT_OPT_COUNT_EVALS: *value = h->count_evals; return SPLAT_OK;
    case SPLAT_OPT_BBOX_PAIRS: *value = h->bbox_pairs; return SPLAT_OK;
    case SPLAT_OPT_BLEND_EVALS: *value = h->have_frame ? h->st_host->evals : 0; return SPLAT_OK;
    case SPLAT_OPT_DEBUG_CAPTURE: *value = h->debug_capture; return SPLAT_OK;
    case SPLAT_OPT_FP64_CONICS: *value = h->have_frame ? h->st_host->fp64_conics : 0; return SPLAT_OK;
    case SPLAT_OPT_KERNEL_LAUNCHES: *value = h->launches; return SPLAT_OK;
    case SPLAT_OPT_BLEND_CONFIG:
      *value = h->blend.tile_w | (h->blend.tile_h << 8) | ((uint64_t)h->blend.threads << 16);
      return SPLAT_OK;
    case SPLAT_OPT_SCENE_SPLATS:
      *value = h->n;
      return SPLAT_OK;
    case SPLAT_OPT_INJECT_FAULT:
      *value = h->inject_alloc ? SPLAT_FAULT_ALLOC : h->inject_lost_us ? (SPLAT_FAULT_LOST_WAIT | ((uint64_t)h->inject_lost_us << 8)) : 0;
      return SPLAT_OK;
    default: return fail(h, SPLAT_ERR_UNSUPPORTED, "unknown option");
  }
}

SPLAT_API int splat_cuda_debug_dump(splat_cuda_handle* h, float* proj, uint8_t* visible, float* color,
                                    uint64_t* keys, uint32_t* values, uint64_t key_capacity, uint32_t* ranges,
                                    uint64_t range_capacity, uint64_t* n_pairs) {
  if (!h) return SPLAT_ERR_INVALID_ARG;
  if (!h->have_frame) return fail(h, SPLAT_ERR_INVALID_ARG, "no frame rendered yet");
  CK(cudaSetDevice(h->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(h->stream), "sync");
  const DevState& st = *h->st_host;
  const uint64_t P = std::min<uint64_t>(st.total_pairs, h->cap);
  if (n_pairs) *n_pairs = P;
  if ((proj || color) && !h->dbg_proj)
    return fail(h, SPLAT_ERR_INVALID_ARG, "enable SPLAT_OPT_DEBUG_CAPTURE before rendering");
  if (proj) CK(cudaMemcpy(proj, h->dbg_proj, h->n * 8 * sizeof(float), cudaMemcpyDeviceToHost), "dump");
  if (color) CK(cudaMemcpy(color, h->dbg_color, h->n * 3 * sizeof(float), cudaMemcpyDeviceToHost), "dump");
  std::vector<BinInfo> bin;
  if (visible || keys) {
    bin.resize(h->n);
    if (h->n) CK(cudaMemcpy(bin.data(), h->bin, h->n * sizeof(BinInfo), cudaMemcpyDeviceToHost), "dump");
  }
  if (visible)
    for (uint64_t i = 0; i < h->n; i++) visible[i] = bin[i].rect_lo != kCulled;
  const uint64_t m = std::min(P, key_capacity);
  if ((keys || values) && m) {
    // The buckets hold each tile's pairs (depth bits << 32 | splat) in blend
    // order; the reference's key of a pair is tile << 32 | depth bits.
    const uint64_t tiles = (uint64_t)h->last_fp.tiles_x * h->last_fp.tiles_y;
    std::vector<uint64_t> pw(m);
    std::vector<uint2> rg(tiles);
    CK(cudaMemcpy(pw.data(), h->pairs[0], m * 8, cudaMemcpyDeviceToHost), "dump");
    CK(cudaMemcpy(rg.data(), h->ranges, tiles * sizeof(uint2), cudaMemcpyDeviceToHost), "dump");
    for (uint64_t t = 0; t < tiles; t++)
      for (uint64_t p = rg[t].x; p < rg[t].y && p < m; p++) {
        if (values) values[p] = (uint32_t)pw[p];
        if (keys) keys[p] = (t << 32) | (pw[p] >> 32);
      }
  }
  if (ranges) {
    const uint64_t tiles = (uint64_t)h->last_fp.tiles_x * h->last_fp.tiles_y;
    const uint64_t r = std::min<uint64_t>(tiles * 2, range_capacity);
    if (r) CK(cudaMemcpy(ranges, h->ranges, r * 4, cudaMemcpyDeviceToHost), "dump");
  }
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_create_learned(const splat_scene_desc* d, const uint16_t* latents, const uint16_t* mlp_params,
                                        int device, splat_cuda_handle** out) {
  g_create_error.clear();
  if (!out) return SPLAT_ERR_INVALID_ARG;
  *out = nullptr;
  if (!d || !mlp_params || (d->n && !latents)) {
    g_create_error = "null geometry, latents or MLP parameters";
    return SPLAT_ERR_INVALID_ARG;
  }
  if (d->precision != SPLAT_PRECISION_FP16) {
    g_create_error = "learned colour needs FP16 geometry (SPLAT_PRECISION_FP16)";
    return SPLAT_ERR_UNSUPPORTED;
  }
  // The geometry through the FP16 upload, with a zero base colour in place
  // of the SH (never read: the colour comes from the MLP).
  splat_scene_desc g = *d;
  g.sh_degree = 0;
  std::vector<uint16_t> zero_colour(d->n ? (size_t)d->n * 3 : 1, 0);
  g.sh_f16 = zero_colour.data();
  splat_cuda_handle* h = nullptr;
  int rc = splat_cuda_create(&g, device, &h);
  if (rc) return rc;
  auto up = [&](void** dst, const void* src, size_t bytes, const char* what) -> int {
    cudaError_t er = cudaMalloc(dst, bytes);
    if (er != cudaSuccess) return cuda_fail(h, er, what);
    er = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    if (er != cudaSuccess) return cuda_fail(h, er, what);
    return SPLAT_OK;
  };
  if ((rc = up((void**)&h->mlp16, mlp_params, SPLAT_MLP_PARAMS * sizeof(uint16_t), "upload MLP parameters")) ||
      (d->n && (rc = up((void**)&h->lat16, latents, d->n * SPLAT_MLP_LATENT * sizeof(uint16_t), "upload latents")))) {
    g_create_error = h->err;
    splat_cuda_destroy(h);
    return rc;
  }
  if (!d->n) {  // an empty scene still marks the handle learned
    if ((rc = up((void**)&h->lat16, mlp_params, 16, "latents"))) {
      g_create_error = h->err;
      splat_cuda_destroy(h);
      return rc;
    }
  }
  const cudaError_t se = cudaDeviceSynchronize();  // the uploads have landed (see create_impl)
  if (se != cudaSuccess) {
    rc = cuda_fail(h, se, "upload latents");
    g_create_error = h->err;
    splat_cuda_destroy(h);
    return rc;
  }
  *out = h;
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_destroy(splat_cuda_handle* h) {
  if (!h) return SPLAT_OK;
  cudaSetDevice(h->device);
  if (h->own_stream) cudaStreamSynchronize(h->own_stream);
  if (h->stream && h->stream != h->own_stream) cudaStreamSynchronize(h->stream);
  dfree(h->pos_op);
  dfree(h->cov_a);
  dfree(h->cov_b);
  dfree(h->color);
  dfree(h->sh);
  dfree(h->pos_k);
  dfree(h->geom16);
  dfree(h->sh16);
  dfree(h->lat16);
  dfree(h->mlp16);
  dfree(h->cells_dev);
  dfree(h->rec);
  dfree(h->bin);
  dfree(h->skip);
  dfree(h->rx_bin);
  dfree(h->rx_skip);
  dfree(h->shard_scratch);
  dfree(h->shard_totals);
  if (h->shard_totals_host) cudaFreeHost(h->shard_totals_host);
  free_pairs(h);
  dfree(h->ranges);
  dfree(h->counts);
  dfree(h->totals);
  dfree(h->order);
  dfree(h->out_dev);
  dfree(h->full_dev);
  dfree(h->st);
  dfree(h->table);
  dfree(h->dbg_proj);
  dfree(h->dbg_color);
  dfree(h->bin_order);
  if (h->st_host) cudaFreeHost(h->st_host);
  if (h->stage) cudaFreeHost(h->stage);
  for (auto& ev : h->ev)
    if (ev) cudaEventDestroy(ev);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return SPLAT_OK;
}

SPLAT_API const char* splat_cuda_last_error(const splat_cuda_handle* h) { return h ? h->err.c_str() : ""; }
