// Batched rendering (include/splat_cuda.h, splat_cuda_batch_*): many views of
// uneven resolution over several scenes, each pipeline stage one launch over
// all views, recorded once as a CUDA graph and replayed.
//
// Planning lays the views out one after another: their splats in the
// projection launch (256 per CTA), their count-matrix rows in the count and
// scatter launches, their tiles in one global tile space (each view's first
// tile aligned to kTileAlign) shared by the ranges, the pair buffer, the
// per-tile sorts and the persistent blend. Kernels find their view by binary
// search over the view table. A batch is:
//   clear counters -> project (all views) -> count -> column scan ->
//   tile ranges -> scatter -> sorts -> blend (all views) -> counters to host
// with no host synchronisation in between; the graph holds exactly that.
//
// The pair buffers are sized by one plain run before the graph is recorded
// (the views are fixed, so later runs need the same); an overflow is still
// detected from the counters, grows the buffers and re-records the graph.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/splat_cuda.h"
#include "common.cuh"
#include "handle.h"

#define SPLAT_API extern "C" __attribute__((visibility("default")))

using namespace splat;

struct splat_cuda_batch {
  int device = 0;
  int num_sms = 148;
  size_t max_smem = 48 * 1024;
  std::vector<splat_cuda_handle*> scenes;
  std::vector<splat_batch_view> views;
  BlendConfig cfg{kTile, kTile, 512};
  bool exact = false;
  uint32_t launches = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // per-view buffers (independent of the tile configuration)
  Record* rec = nullptr;
  BinInfo* bin = nullptr;
  BinSkip* skip = nullptr;  // kept-tile lists of the wide rectangles
  std::vector<uint64_t> splat_off;  // first record of each view
  // plan (depends on the tile configuration)
  std::vector<ViewTask> tasks;
  ViewTask* table = nullptr;
  std::vector<ViewTask> ltasks;  // the learned-colour views (their own projection launch)
  ViewTask* ltable = nullptr;
  uint64_t learned_tiles = 0;
  uint32_t n_tiles = 0, n_chunks = 0, proj_ctas = 0, bin_ctas = 0, col_ctas = 0, max_tiles = 0;
  uint32_t* counts = nullptr;
  size_t counts_words = 0;
  uint32_t* totals = nullptr;
  uint2* ranges = nullptr;
  uint32_t* order = nullptr;  // kTileClasses lists of n_tiles tiles
  void* counters = nullptr;        // FrameCounters block (device)
  void* counters_host = nullptr;   // pinned copy
  size_t counters_bytes = 0;
  uint64_t* pairs[2] = {nullptr, nullptr};
  uint64_t cap = 0;
  // the recorded batch
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};     // around a graph launch
  cudaEvent_t stage[4] = {nullptr, nullptr, nullptr, nullptr};  // between stages, inside the graph
  bool ran = false;
  std::string err;
};

namespace {

thread_local std::string g_batch_create_error;

int bfail(splat_cuda_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

int bcuda(splat_cuda_batch* b, cudaError_t e, const char* what) {
  const int code = (e == cudaErrorMemoryAllocation) ? SPLAT_ERR_OOM : SPLAT_ERR_DEVICE;
  return bfail(b, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BK(expr, what)                              \
  do {                                              \
    const cudaError_t e_ = (expr);                  \
    if (e_ != cudaSuccess) return bcuda(b, e_, what); \
  } while (0)

template <class T> void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void drop_graph(splat_cuda_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

void free_plan(splat_cuda_batch* b) {
  drop_graph(b);
  dfree(b->table);
  dfree(b->ltable);
  dfree(b->counts);
  dfree(b->totals);
  dfree(b->ranges);
  dfree(b->order);
  dfree(b->counters);
  if (b->counters_host) cudaFreeHost(b->counters_host);
  b->counters_host = nullptr;
}

int ensure_pairs(splat_cuda_batch* b, uint64_t cap) {
  if (cap <= b->cap) return SPLAT_OK;
  if (cap > kMaxPairs) return bfail(b, SPLAT_ERR_CAPACITY, "more than 2^30 - 1 gaussian/tile pairs in the batch");
  for (auto& p : b->pairs) dfree(p);
  b->cap = 0;
  // Two words of slack: the blend's bulk copy of a tile rounds its end up to 16 bytes.
  for (auto& p : b->pairs) BK(cudaMalloc(&p, (cap + 2) * sizeof(uint64_t)), "cudaMalloc pairs");
  b->cap = cap;
  return SPLAT_OK;
}

bool downsample_fits(const splat_batch_view& v, const BlendConfig& c) {
  const uint32_t f = v.downsample ? v.downsample : 1;
  return f == 1 || (c.tile_w % f == 0 && c.tile_h % f == 0);
}

// Lays the views out for configuration b->cfg and allocates the
// configuration-dependent buffers.
int plan(splat_cuda_batch* b) {
  free_plan(b);
  const uint32_t nv = (uint32_t)b->views.size();
  b->tasks.assign(nv, ViewTask{});
  b->ltasks.clear();
  b->learned_tiles = 0;
  uint64_t tile = 0, proj = 0, bins = 0, cols = 0, words = 0;
  uint32_t max_tiles = 0;
  for (uint32_t i = 0; i < nv; i++) {
    const splat_batch_view& v = b->views[i];
    const splat_cuda_handle* h = b->scenes[v.scene];
    ViewTask& t = b->tasks[i];
    t.fp = make_params(v.view, v.width, v.height, v.bg, v.downsample ? v.downsample : 1);
    set_tile_shape(t.fp, b->cfg.tile_w, b->cfg.tile_h);
    t.s = scene_dev(h);
    t.rec = b->rec + b->splat_off[i];
    t.bin = b->bin + b->splat_off[i];
    t.skip = b->skip + b->splat_off[i];
    t.out = v.dev_out;
    t.full = nullptr;
    t.rows = bin_rows(h->n, b->num_sms);
    const uint32_t tiles = t.fp.tiles_x * t.fp.tiles_y;
    tile = (tile + kTileAlign - 1) / kTileAlign * kTileAlign;
    t.tile0 = (uint32_t)tile;
    t.proj_cta0 = (uint32_t)proj;
    t.bin_cta0 = (uint32_t)bins;
    t.col_cta0 = (uint32_t)cols;
    tile += tiles;
    if (h->lat16) {  // projected by the learned-colour launch, in tiles of 128 splats
      t.pad[0] = i;
      b->ltasks.push_back(t);
      b->ltasks.back().proj_cta0 = (uint32_t)b->learned_tiles;
      b->learned_tiles += (h->n + 127) / 128;
    } else {
      proj += (h->n + kProjectSplatsPerCta - 1) / kProjectSplatsPerCta;
    }
    bins += t.rows;
    cols += (tiles + 31) / 32;
    words += (uint64_t)t.rows * tiles;
    max_tiles = std::max(max_tiles, tiles);
  }
  if (tile >= (1ull << 31) || proj >= (1ull << 31) || bins >= (1ull << 31) || cols >= (1ull << 31) ||
      b->learned_tiles >= (1ull << 31))
    return bfail(b, SPLAT_ERR_CAPACITY, "batch too large for one launch per stage");
  b->n_tiles = (uint32_t)tile;
  b->n_chunks = (uint32_t)((tile + kScanChunk - 1) / kScanChunk);
  b->proj_ctas = (uint32_t)proj;
  b->bin_ctas = (uint32_t)bins;
  b->col_ctas = (uint32_t)cols;
  b->max_tiles = max_tiles;
  b->counts_words = words;
  BK(cudaMalloc(&b->counts, std::max<uint64_t>(words, 1) * sizeof(uint32_t)), "cudaMalloc counts");
  uint64_t off = 0;
  for (uint32_t i = 0; i < nv; i++) {
    b->tasks[i].counts = b->counts + off;
    off += (uint64_t)b->tasks[i].rows * b->tasks[i].fp.tiles_x * b->tasks[i].fp.tiles_y;
  }
  BK(cudaMalloc(&b->table, nv * sizeof(ViewTask)), "cudaMalloc views");
  BK(cudaMemcpy(b->table, b->tasks.data(), nv * sizeof(ViewTask), cudaMemcpyHostToDevice), "upload views");
  if (!b->ltasks.empty()) {
    for (auto& lt : b->ltasks) lt.counts = b->tasks[lt.pad[0]].counts;
    BK(cudaMalloc(&b->ltable, b->ltasks.size() * sizeof(ViewTask)), "cudaMalloc learned views");
    BK(cudaMemcpy(b->ltable, b->ltasks.data(), b->ltasks.size() * sizeof(ViewTask), cudaMemcpyHostToDevice),
       "upload learned views");
  }
  const size_t nt = std::max<uint32_t>(b->n_tiles, 1);
  BK(cudaMalloc(&b->totals, nt * sizeof(uint32_t)), "cudaMalloc totals");
  BK(cudaMalloc(&b->ranges, nt * sizeof(uint2)), "cudaMalloc ranges");
  BK(cudaMalloc(&b->order, kTileClasses * nt * sizeof(uint32_t)), "cudaMalloc tile classes");
  // Padding tiles between views are never written by the column scan: their
  // totals stay zero (empty ranges).
  BK(cudaMemset(b->totals, 0, nt * sizeof(uint32_t)), "clear totals");
  // A cudaMemcpy from pageable memory may return before its DMA lands, and a
  // device memset is asynchronous; the batch's stream does not wait for the
  // legacy stream that carries both, so they must land before its first use.
  BK(cudaDeviceSynchronize(), "upload views");
  b->counters_bytes = frame_counters_bytes(nv, std::max<uint32_t>(b->n_chunks, 1));
  BK(cudaMalloc(&b->counters, b->counters_bytes), "cudaMalloc counters");
  BK(cudaMallocHost(&b->counters_host, b->counters_bytes), "cudaMallocHost counters");
  std::memset(b->counters_host, 0, b->counters_bytes);
  return SPLAT_OK;
}

// Records stage event k on `s`; under stream capture as an external event
// node, so that the graph's replays record it.
cudaError_t stage_event(splat_cuda_batch* b, int k, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const cudaError_t e = cudaStreamIsCapturing(s, &cs);
  if (e != cudaSuccess) return e;
  return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(b->stage[k], s, cudaEventRecordExternal)
                                             : cudaEventRecord(b->stage[k], s);
}

// Elapsed time between two events, 0 when it is not available (the error is
// cleared so that it does not surface at a later launch check).
float elapsed_ms(cudaEvent_t a, cudaEvent_t c) {
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, a, c) != cudaSuccess) {
    cudaGetLastError();
    ms = 0.0f;
  }
  return ms;
}

// Enqueues one batch on `s` (plain or under stream capture).
int enqueue(splat_cuda_batch* b, cudaStream_t s) {
  const uint32_t nv = (uint32_t)b->views.size();
  const FrameCounters fc = frame_counters_at(b->counters, nv);
  BK(cudaMemsetAsync(b->counters, 0, b->counters_bytes, s), "clear counters");
  BK(stage_event(b, 0, s), "event");
  BK(launch_project_batch(b->table, nv, b->proj_ctas, fc, s, &b->launches), "project kernel");
  BK(launch_project_learned_batch(b->ltable, (uint32_t)b->ltasks.size(), b->learned_tiles, fc, s, &b->launches),
     "learned-colour project kernel");
  BK(stage_event(b, 1, s), "event");
  BinLaunch bl{};
  bl.n_views = nv;
  bl.bin_ctas = b->bin_ctas;
  bl.col_ctas = b->col_ctas;
  bl.n_tiles = b->n_tiles;
  bl.max_tiles = b->max_tiles;
  bl.counts_all = b->counts;
  bl.counts_bytes = b->counts_words * sizeof(uint32_t);
  BK(launch_binning(b->table, bl, b->totals, b->ranges, b->order, b->pairs[0], b->pairs[1], b->cap,
                    fc, b->num_sms, b->max_smem, s, &b->launches, !blend_sorts_tiles(b->cfg)),
     "binning kernels");
  BK(stage_event(b, 2, s), "event");
  BK(launch_blend(b->table, nv, b->n_tiles, b->pairs[0], b->ranges, b->order, b->exact, b->cfg, fc.st,
                  b->num_sms, s, &b->launches),
     "blend kernel");
  BK(stage_event(b, 3, s), "event");
  BK(cudaMemcpyAsync(b->counters_host, b->counters, b->counters_bytes, cudaMemcpyDeviceToHost, s), "copy counters");
  return SPLAT_OK;
}

// Records the batch as a graph on the batch's own stream.
int record(splat_cuda_batch* b) {
  drop_graph(b);
  const uint32_t launches = b->launches;
  BK(cudaStreamBeginCapture(b->own_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  const int rc = enqueue(b, b->own_stream);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->own_stream, &g);
  b->launches = launches;  // recording launches nothing
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return bcuda(b, e, "end capture");
  b->graph = g;
  BK(cudaGraphInstantiate(&b->exec, b->graph, 0), "instantiate graph");
  return SPLAT_OK;
}

// Kernels per batch (the launch count one graph replay adds).
uint32_t kernels_per_batch(const splat_cuda_batch* b) {
  if (!b->n_tiles) return 0u;
  // count, column scan, ranges, scatter, long sort, blend, and the small and
  // mid tile sorts unless the blend sorts those tiles itself
  return (blend_sorts_tiles(b->cfg) ? 6u : 8u) + (b->proj_ctas ? 1u : 0u) + (b->learned_tiles ? 1u : 0u);
}

const DevState& host_state(const splat_cuda_batch* b) { return *static_cast<const DevState*>(b->counters_host); }

// One plain (unrecorded) batch, then the pair buffers grown until it fits.
int size_pairs(splat_cuda_batch* b) {
  for (int attempt = 0; attempt < 8; attempt++) {
    int rc = enqueue(b, b->own_stream);
    if (rc) return rc;
    BK(cudaStreamSynchronize(b->own_stream), "batch");
    const uint64_t total = host_state(b).total_pairs;
    if (total <= b->cap) return SPLAT_OK;
    rc = ensure_pairs(b, std::max<uint64_t>(total + total / 8, b->cap + 1));
    if (rc) return rc;
  }
  return bfail(b, SPLAT_ERR_CAPACITY, "pair count did not settle");
}

// plan + size + record for the current configuration.
int prepare(splat_cuda_batch* b) {
  for (const auto& v : b->views)
    if (!downsample_fits(v, b->cfg))
      return bfail(b, SPLAT_ERR_UNSUPPORTED, "a view's downsample factor does not divide the tile shape");
  int rc = plan(b);
  if (rc) return rc;
  if ((rc = size_pairs(b))) return rc;
  return record(b);
}

void destroy(splat_cuda_batch* b) {
  cudaSetDevice(b->device);
  if (b->own_stream) cudaStreamSynchronize(b->own_stream);
  if (b->stream && b->stream != b->own_stream) cudaStreamSynchronize(b->stream);
  free_plan(b);
  for (auto& p : b->pairs) dfree(p);
  dfree(b->rec);
  dfree(b->bin);
  dfree(b->skip);
  for (auto& e : b->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : b->stage)
    if (e) cudaEventDestroy(e);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
}

}  // namespace

SPLAT_API const char* splat_cuda_batch_create_error(void) { return g_batch_create_error.c_str(); }

SPLAT_API int splat_cuda_batch_create(splat_cuda_handle* const* scenes, uint32_t n_scenes,
                                      const splat_batch_view* views, uint32_t n_views, splat_cuda_batch** out) {
  g_batch_create_error.clear();
  if (!out) return SPLAT_ERR_INVALID_ARG;
  *out = nullptr;
  auto reject = [&](int code, const std::string& msg) {
    g_batch_create_error = msg;
    return code;
  };
  if (!scenes || n_scenes == 0 || !views || n_views == 0) return reject(SPLAT_ERR_INVALID_ARG, "no scenes or views");
  for (uint32_t i = 0; i < n_scenes; i++) {
    if (!scenes[i]) return reject(SPLAT_ERR_INVALID_ARG, "null scene handle");
    if (scenes[i]->device != scenes[0]->device) return reject(SPLAT_ERR_INVALID_ARG, "scenes on different devices");
  }
  for (uint32_t i = 0; i < n_views; i++) {
    const splat_batch_view& v = views[i];
    if (v.scene >= n_scenes) return reject(SPLAT_ERR_INVALID_ARG, "view " + std::to_string(i) + ": no such scene");
    if (v.width == 0 || v.height == 0 || v.width > SPLAT_MAX_DIM || v.height > SPLAT_MAX_DIM)
      return reject(SPLAT_ERR_INVALID_ARG, "view " + std::to_string(i) + ": size outside 1..16384");
    const uint32_t f = v.downsample ? v.downsample : 1;
    if (v.width / f == 0 || v.height / f == 0)
      return reject(SPLAT_ERR_INVALID_ARG, "view " + std::to_string(i) + ": empty after downsampling");
    if (!v.dev_out) return reject(SPLAT_ERR_INVALID_ARG, "view " + std::to_string(i) + ": null output");
  }
  auto* b = new splat_cuda_batch();
  auto bail = [&](int rc) {
    g_batch_create_error = b->err;
    destroy(b);
    return rc;
  };
  b->device = scenes[0]->device;
  b->num_sms = scenes[0]->num_sms;
  b->max_smem = scenes[0]->max_smem;
  b->scenes.assign(scenes, scenes + n_scenes);
  b->views.assign(views, views + n_views);
  cudaError_t e = cudaSetDevice(b->device);
  if (e != cudaSuccess) return bail(bcuda(b, e, "cudaSetDevice"));
  if ((e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(bcuda(b, e, "cudaStreamCreate"));
  b->stream = b->own_stream;
  for (auto& ev : b->ev)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return bail(bcuda(b, e, "cudaEventCreate"));
  for (auto& ev : b->stage)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return bail(bcuda(b, e, "cudaEventCreate"));
  uint64_t splats = 0;
  b->splat_off.resize(n_views);
  for (uint32_t i = 0; i < n_views; i++) {
    b->splat_off[i] = splats;
    splats += scenes[views[i].scene]->n;
  }
  if ((e = cudaMalloc(&b->rec, std::max<uint64_t>(splats, 1) * sizeof(Record))) != cudaSuccess)
    return bail(bcuda(b, e, "cudaMalloc records"));
  if ((e = cudaMalloc(&b->bin, std::max<uint64_t>(splats, 1) * sizeof(BinInfo))) != cudaSuccess)
    return bail(bcuda(b, e, "cudaMalloc bins"));
  if ((e = cudaMalloc(&b->skip, std::max<uint64_t>(splats, 1) * sizeof(BinSkip))) != cudaSuccess)
    return bail(bcuda(b, e, "cudaMalloc bin skips"));
  int rc = ensure_pairs(b, std::max<uint64_t>(4 * splats, 1u << 16));
  if (rc) return bail(rc);
  if ((rc = prepare(b))) return bail(rc);
  *out = b;
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_batch_set_config(splat_cuda_batch* b, const splat_blend_config* config) {
  if (!b || !config) return SPLAT_ERR_INVALID_ARG;
  const BlendConfig c{config->tile_w, config->tile_h, config->threads};
  if (!blend_config_supported(c)) return bfail(b, SPLAT_ERR_UNSUPPORTED, "unsupported tile shape or thread count");
  BK(cudaSetDevice(b->device), "cudaSetDevice");
  BK(cudaStreamSynchronize(b->stream), "batch");
  const BlendConfig old = b->cfg;
  b->cfg = c;
  const int rc = prepare(b);
  if (rc) {
    b->cfg = old;
    const std::string why = b->err;
    prepare(b);
    b->err = why;
  }
  return rc;
}

SPLAT_API int splat_cuda_batch_get_config(const splat_cuda_batch* b, splat_blend_config* config) {
  if (!b || !config) return SPLAT_ERR_INVALID_ARG;
  *config = splat_blend_config{b->cfg.tile_w, b->cfg.tile_h, b->cfg.threads};
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_batch_run(splat_cuda_batch* b) {
  if (!b) return SPLAT_ERR_INVALID_ARG;
  if (!b->exec) return bfail(b, SPLAT_ERR_INVALID_ARG, "batch has no recorded graph");
  BK(cudaSetDevice(b->device), "cudaSetDevice");
  BK(cudaEventRecord(b->ev[0], b->stream), "event");
  BK(cudaGraphLaunch(b->exec, b->stream), "graph launch");
  BK(cudaEventRecord(b->ev[1], b->stream), "event");
  b->launches += kernels_per_batch(b);
  b->ran = true;
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_batch_finish(splat_cuda_batch* b, splat_render_stats* per_view, double* total_ms,
                                      int* regrown) {
  if (!b) return SPLAT_ERR_INVALID_ARG;
  if (regrown) *regrown = 0;
  BK(cudaSetDevice(b->device), "cudaSetDevice");
  BK(cudaStreamSynchronize(b->stream), "batch");
  const uint32_t nv = (uint32_t)b->views.size();
  const FrameCounters fc = frame_counters_at(b->counters_host, nv);
  float ms = 0.0f, st[3] = {0.0f, 0.0f, 0.0f};
  if (b->ran) {
    ms = elapsed_ms(b->ev[0], b->ev[1]);
    for (int k = 0; k < 3; k++) st[k] = elapsed_ms(b->stage[k], b->stage[k + 1]);
  }
  if (total_ms) *total_ms = ms;
  if (per_view)
    for (uint32_t i = 0; i < nv; i++) {
      per_view[i] = splat_render_stats{};
      per_view[i].visible = fc.view_visible[i];
      per_view[i].overlaps = fc.view_pairs[i];
      per_view[i].project_ms = st[0];  // stage times of the whole batch
      per_view[i].sort_ms = st[1];
      per_view[i].raster_ms = st[2];
      per_view[i].total_ms = ms;
    }
  if (fc.st->total_pairs > b->cap) {
    int rc = ensure_pairs(b, fc.st->total_pairs + fc.st->total_pairs / 8);
    if (!rc) rc = record(b);
    if (rc) return rc;
    if (regrown) *regrown = 1;
  }
  return SPLAT_OK;
}

SPLAT_API int splat_cuda_batch_autotune(splat_cuda_batch* b, uint32_t reps, splat_tune_result* results,
                                        uint32_t capacity, uint32_t* n_results) {
  if (!b) return SPLAT_ERR_INVALID_ARG;
  if (n_results) *n_results = 0;
  if (reps == 0) reps = 1;
  BK(cudaSetDevice(b->device), "cudaSetDevice");
  BK(cudaStreamSynchronize(b->stream), "batch");
  static const BlendConfig kCandidates[] = {{16, 16, 256}, {16, 16, 128}, {16, 16, 512}, {8, 8, 128}, {8, 8, 256},
                                            {8, 8, 512},   {32, 16, 128}, {32, 16, 256}, {32, 16, 512}};
  const BlendConfig start = b->cfg;
  BlendConfig best = start;
  double best_ms = -1.0;
  // Two rounds over the candidates, each keeping its faster time: a
  // configuration timed while the clock dipped gets a second chance.
  constexpr uint32_t kCand = sizeof(kCandidates) / sizeof(kCandidates[0]);
  double per_ms[kCand];
  bool fits[kCand];
  for (uint32_t k = 0; k < kCand; k++) {
    fits[k] = true;
    for (const auto& v : b->views) fits[k] = fits[k] && downsample_fits(v, kCandidates[k]);
    per_ms[k] = -1.0;
  }
  for (int round = 0; round < 2; round++) {
    for (uint32_t k = 0; k < kCand; k++) {
      if (!fits[k]) continue;
      b->cfg = kCandidates[k];
      int rc = prepare(b);
      if (rc) return rc;
      BK(cudaGraphLaunch(b->exec, b->own_stream), "graph launch");  // warm-up
      BK(cudaEventRecord(b->ev[0], b->own_stream), "event");
      for (uint32_t r = 0; r < reps; r++) BK(cudaGraphLaunch(b->exec, b->own_stream), "graph launch");
      BK(cudaEventRecord(b->ev[1], b->own_stream), "event");
      BK(cudaEventSynchronize(b->ev[1]), "tuning");
      b->launches += (reps + 1) * kernels_per_batch(b);
      float ms = 0.0f;
      BK(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]), "event time");
      const double per = ms / reps;
      if (per_ms[k] < 0.0 || per < per_ms[k]) per_ms[k] = per;
    }
  }
  uint32_t count = 0;
  for (uint32_t k = 0; k < kCand; k++) {
    if (!fits[k]) continue;
    const BlendConfig& c = kCandidates[k];
    if (results && count < capacity)
      results[count] = splat_tune_result{splat_blend_config{c.tile_w, c.tile_h, c.threads}, 0u, per_ms[k]};
    count++;
    if (best_ms < 0.0 || per_ms[k] < best_ms) {
      best_ms = per_ms[k];
      best = c;
    }
  }
  if (n_results) *n_results = std::min(count, capacity);
  b->cfg = best;
  b->ran = false;
  return prepare(b);
}

SPLAT_API int splat_cuda_batch_set_option(splat_cuda_batch* b, uint32_t option, uint64_t value) {
  if (!b) return SPLAT_ERR_INVALID_ARG;
  switch (option) {
    case SPLAT_OPT_EXACT_BLEND: {
      if ((value != 0) == b->exact) return SPLAT_OK;
      BK(cudaSetDevice(b->device), "cudaSetDevice");
      BK(cudaStreamSynchronize(b->stream), "batch");
      b->exact = value != 0;
      return record(b);
    }
    case SPLAT_OPT_KERNEL_LAUNCHES:
      b->launches = (uint32_t)value;
      return SPLAT_OK;
    default:
      return bfail(b, SPLAT_ERR_UNSUPPORTED, "unknown batch option");
  }
}

SPLAT_API int splat_cuda_batch_get_option(const splat_cuda_batch* b, uint32_t option, uint64_t* value) {
  if (!b || !value) return SPLAT_ERR_INVALID_ARG;
  switch (option) {
    case SPLAT_OPT_EXACT_BLEND: *value = b->exact; return SPLAT_OK;
    case SPLAT_OPT_KERNEL_LAUNCHES: *value = b->launches; return SPLAT_OK;
    case SPLAT_OPT_BLEND_CONFIG:
      *value = b->cfg.tile_w | (b->cfg.tile_h << 8) | ((uint64_t)b->cfg.threads << 16);
      return SPLAT_OK;
    default: return SPLAT_ERR_UNSUPPORTED;
  }
}

SPLAT_API int splat_cuda_batch_set_stream(splat_cuda_batch* b, void* stream) {
  if (!b) return SPLAT_ERR_INVALID_ARG;
  BK(cudaSetDevice(b->device), "cudaSetDevice");
  BK(cudaStreamSynchronize(b->stream), "batch");
  b->stream = stream ? static_cast<cudaStream_t>(stream) : b->own_stream;
  return SPLAT_OK;
}

SPLAT_API void* splat_cuda_batch_get_stream(const splat_cuda_batch* b) { return b ? b->stream : nullptr; }

SPLAT_API const char* splat_cuda_batch_last_error(const splat_cuda_batch* b) { return b ? b->err.c_str() : ""; }

SPLAT_API int splat_cuda_batch_destroy(splat_cuda_batch* b) {
  if (!b) return SPLAT_OK;
  destroy(b);
  return SPLAT_OK;
}
