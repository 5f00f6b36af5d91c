/*
 * splat_cuda.h — C ABI of the B200 (sm_100a) Gaussian-splat tile rasterizer.
 *
 * This is the boundary a `cuda` backend of farmerchris/splat binds over FFI.
 * It replaces the body of `Renderer::render` (src/render/mod.rs:86-97) for a
 * scene bound at construction (`render::create`, src/render/mod.rs:115-121):
 *
 *   reference                                   replaced by
 *   ------------------------------------------  -----------------------------
 *   CpuTiled::new / GpuRenderer::new            splat_cuda_create
 *     (src/render/cpu.rs:82-91, gpu.rs:510-707)
 *   Renderer::render                            splat_cuda_render
 *     (src/render/mod.rs:89-96; cpu.rs:109-222)
 *   Renderer::render + term::downsample         splat_cuda_render with
 *     (src/app.rs:203-206, src/term.rs:74-99)     downsample > 1
 *   Renderer::name (src/render/mod.rs:87)       splat_cuda_backend_name
 *   drop(Box<dyn Renderer>)                     splat_cuda_destroy
 *   anyhow error text (src/bench.rs:147)        splat_cuda_last_error
 *
 * All entry points return a splat_status and never abort the process. A
 * handle is used by one thread at a time (the reference trait is Send, not
 * Sync, and render takes &mut self). Every call makes the handle's device
 * current; all device work runs on the handle's stream.
 *
 * Layouts follow the reference's Scene (src/scene.rs:11-28): glam Vec3 is
 * three packed f32, so `Vec<Vec3>` / `Vec<[f32; 6]>` can be passed as plain
 * float pointers.
 */
#ifndef SPLAT_CUDA_H
#define SPLAT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPLAT_CUDA_ABI_VERSION 1

typedef enum splat_status {
  SPLAT_OK = 0,
  SPLAT_ERR_INVALID_ARG = 1,   /* null pointer, bad size, frame > MAX_DIM, ... */
  SPLAT_ERR_OOM = 2,           /* device or pinned-host allocation failed */
  SPLAT_ERR_CAPACITY = 3,      /* one tile holds more (splat, tile) pairs than
                                  the pair buffers can (frames that only need
                                  more pairs in total are drawn in windows) */
  SPLAT_ERR_DEVICE = 4,        /* CUDA error (text in splat_cuda_last_error) */
  SPLAT_ERR_TIMEOUT = 5,       /* a bounded device-side wait gave up */
  SPLAT_ERR_UNSUPPORTED = 6    /* option or precision not available */
} splat_status;

/* Largest output width or height (src/render/mod.rs:31-33). */
#define SPLAT_MAX_DIM 16384u
/* Screen tile edge in pixels (src/render/cpu.rs:34). */
#define SPLAT_TILE 16u

/* Scene parameter storage. */
#define SPLAT_PRECISION_FP32 0u /* activated f32 params + precomputed cov3d */
#define SPLAT_PRECISION_FP16 1u /* f32 positions; f16 scales/rotations/opacity/SH */

/*
 * A scene, as the reference's Scene holds it (activated parameters).
 *
 * FP32 (precision = SPLAT_PRECISION_FP32): positions, opacities, colors,
 * cov3d and, for sh_degree > 0, sh_rest are read; scales/rotations and the
 * f16 fields are ignored.
 *   positions  n*3  world-space means                       (scene.rs:13)
 *   opacities  n    sigmoid-activated, in [0, 1]             (scene.rs:18)
 *   colors     n*3  SH_C0 * f_dc + 0.5                       (scene.rs:20)
 *   cov3d      n*6  xx, xy, xz, yy, yz, zz                   (scene.rs:26)
 *   sh_rest    n*rest*3, rest = (deg+1)^2 - 1, splat-major, coefficient
 *              (3DGS basis order, sh.rs:39-64), then RGB   (scene.rs:23)
 *
 * FP16 (precision = SPLAT_PRECISION_FP16): positions stay f32; scales_f16
 * (n*3, linear, exp-activated), rotations_f16 (n*4 unit quaternion x,y,z,w),
 * opacities_f16 (n) and sh_f16 (n*(rest+1)*3: the base colour first, then the
 * rest coefficients, RGB innermost) are IEEE binary16 bit patterns. The 3D
 * covariance is then formed on the device from scale and rotation.
 */
typedef struct splat_scene_desc {
  uint64_t n;
  uint32_t sh_degree;  /* 0..3 */
  uint32_t precision;  /* SPLAT_PRECISION_* */
  const float* positions;
  const float* opacities;
  const float* colors;
  const float* cov3d;
  const float* sh_rest;
  const uint16_t* scales_f16;
  const uint16_t* rotations_f16;
  const uint16_t* opacities_f16;
  const uint16_t* sh_f16;
} splat_scene_desc;

/* A resolved camera pose (src/camera.rs:161-170): camera space is x right,
 * y down, z forward; fov_y in radians. */
typedef struct splat_view_desc {
  float eye[3];
  float right[3];
  float down[3];
  float forward[3];
  float fov_y;
  float near_plane;
} splat_view_desc;

/* RenderStats (src/render/mod.rs:72-83). For this tiled backend `overlaps`
 * counts the (splat, tile) pairs drawn: the tiles of each splat's pixel bbox
 * that its alpha = 1/255 ellipse reaches (every bbox tile, as the
 * reference's cpu backend pairs them, with SPLAT_OPT_BBOX_PAIRS). Stage times are device times from CUDA events
 * (project = projection + SH + pair emission, sort = radix sort + tile ranges,
 * raster = blend + downsample); total_ms is host wall time of the call. */
typedef struct splat_render_stats {
  uint64_t visible;
  uint64_t overlaps;
  double project_ms;
  double sort_ms;
  double raster_ms;
  double total_ms;
} splat_render_stats;

typedef struct splat_cuda_handle splat_cuda_handle;

/* ABI version of the loaded library (SPLAT_CUDA_ABI_VERSION). */
int splat_cuda_abi_version(void);

/* "cuda" (Renderer::name, src/render/mod.rs:87). */
const char* splat_cuda_backend_name(void);

/* Binds a scene to a new renderer on `device` (a CUDA ordinal) and uploads it
 * once. Replaces CpuTiled::new (src/render/cpu.rs:82-91) and
 * GpuRenderer::new (src/render/gpu.rs:510-707). On failure *out is NULL and
 * the status says why (no global error text is kept for a NULL handle; see
 * splat_cuda_create_error). */
int splat_cuda_create(const splat_scene_desc* scene, int device, splat_cuda_handle** out);

/* Text of the last splat_cuda_create failure on this thread (also of
 * splat_cuda_create_from_splat / _from_ply / splat_cuda_create_learned). */
const char* splat_cuda_create_error(void);

/* A renderer for a scene file's bytes (in host memory), decoded on the
 * device: the reader and Scene::finalize run in one GPU thread per splat
 * and write the renderer's device layout directly (precision
 * SPLAT_PRECISION_FP32 or _FP16). The image equals that of splat_cuda_create
 * on the host-parsed, finalized scene.
 *   _from_splat: the 32-byte .splat records; replaces splat_format::parse
 *                (src/splat_format.rs:18-44) + Scene::finalize
 *                (src/scene.rs:62-94). Sizes not a multiple of 32 are
 *                rejected with the reference's message.
 *   _from_ply:   a 3DGS PLY (ascii, binary_little_endian or
 *                binary_big_endian; x y z, f_dc_* or red green blue,
 *                f_rest_*, opacity, scale_*, rot_*, each optional but x y z,
 *                any scalar type); replaces ply::parse (src/ply.rs:218-379) +
 *                Scene::finalize. The header is parsed on the host (ASCII
 *                bodies are converted to f64 rows there), the records decoded
 *                on the device. Errors follow the reference's messages. */
int splat_cuda_create_from_splat(const void* data, size_t bytes, uint32_t precision, int device,
                                 splat_cuda_handle** out);
int splat_cuda_create_from_ply(const void* data, size_t bytes, uint32_t precision, int device,
                               splat_cuda_handle** out);

/* Renders `view` at width x height over background bg (linear RGB) and writes
 * the u8 RGB frame, row-major, to host memory rgb_out (Frame::pixels,
 * src/render/mod.rs:43-49). With downsample = f > 1 the frame is box-filtered
 * by f on the device exactly as term::downsample does (src/term.rs:74-99):
 * the output is floor(w/f) x floor(h/f) pixels. downsample 0 means 1.
 * out_bytes must be at least floor(w/f)*floor(h/f)*3. width or height 0 gives
 * an empty frame and zeroed stats (src/render/cpu.rs:120-122). width or
 * height above SPLAT_MAX_DIM is rejected (src/render/mod.rs:35-41). Pair
 * buffers grow and the frame is re-rendered when a view needs more (splat,
 * tile) pairs than allocated (the reference's grow-and-retry,
 * src/render/gpu.rs:1040-1056). A view that needs more pairs than the pair
 * limit (SPLAT_OPT_PAIR_LIMIT, default 2^30 - 1) or than device memory
 * holds is drawn in windows of whole tiles whose pairs fit, each with the
 * full projection: the frame is complete and identical to a one-pass frame
 * (the reference's gpu backend keeps the front-most pairs instead,
 * src/render/gpu.rs:1253-1289), `overlaps` counts all its pairs. Blocks
 * until the frame is in rgb_out. Replaces Renderer::render
 * (src/render/mod.rs:89-96). */
int splat_cuda_render(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width, uint32_t height,
                      const float bg[3], uint32_t downsample, uint8_t* rgb_out, size_t out_bytes,
                      splat_render_stats* stats);

/* Rows [row0, row0 + rows) of the width x height frame splat_cuda_render
 * would produce, bit for bit, into rgb_out (rows * width * 3 bytes, row0
 * first): the projection covers the whole frame, the tile binning, sorts and
 * blend only the tile rows that meet the window. One frame split into row
 * windows over several devices (each with the scene) is the frame's
 * tile-ownership split without a record exchange. No downsample. In stats,
 * `visible` counts the splats visible in the whole frame and `overlaps` the
 * window's (splat, tile) pairs. The reference has no counterpart: its
 * backends render whole frames (Renderer::render, src/render/mod.rs:89-96). */
int splat_cuda_render_rows(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width, uint32_t height,
                           const float bg[3], uint32_t row0, uint32_t rows, uint8_t* rgb_out, size_t out_bytes,
                           splat_render_stats* stats);

/*
 * One frame over several devices that each hold a SHARD of the splats (a
 * contiguous run of the scene, shards in scene order), with one exchange of
 * projected splats: tile ownership by row windows. No counterpart in the
 * reference, whose backends render whole frames from the whole scene
 * (Renderer::render, src/render/mod.rs:89-96).
 *
 * 1. Each device projects its shard (handle h, created from the shard's
 *    splats) for the whole width x height frame with
 *    splat_cuda_shard_records. Windows k = 0 .. n_windows - 1 are the pixel
 *    rows [row_bounds[k], row_bounds[k + 1]) (bounds nondecreasing, at most
 *    height; n_windows at most 64). Every visible splat whose pixel bbox
 *    meets a window's rows goes to that window as one record of
 *    SPLAT_RECORD_BYTES bytes; the records are written to DEVICE memory
 *    `send` (16-byte aligned) window after window, each window's records in
 *    scene order, and counts[k] receives window k's count. If the records
 *    do not fit send_capacity (records), nothing is written, counts are
 *    filled in and the call returns SPLAT_ERR_CAPACITY (size the buffer from
 *    them and call again). *visible (may be NULL) receives the shard's
 *    visible splats. Blocks until the records are written.
 * 2. The records of window k are exchanged (an all-to-all: sender r's k-th
 *    run to the owner of window k) and concatenated in shard order.
 * 3. The owner draws its window with splat_cuda_render_records: `records`
 *    holds n_records of them (DEVICE memory on h's device, 16-byte aligned,
 *    in shard order as received; at most 2^32 - 1); rows [row0, row0 +
 *    rows) of the frame go to `out`, host memory or device memory of h's
 *    device (rows * width * 3 bytes). The window equals those rows of
 *    splat_cuda_render of the whole scene, bit for bit, when row0 and rows
 *    are those of a window given to every sender. h may be any handle on
 *    the device (its own scene is not read). Stats: `visible` counts the
 *    records, `overlaps` the window's (splat, tile) pairs. Pair buffers grow
 *    and frames past the pair limit are drawn in windows of tiles, as in
 *    splat_cuda_render. Blocks until the rows are in `out`.
 */
#define SPLAT_RECORD_BYTES 48u
int splat_cuda_shard_records(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width, uint32_t height,
                             uint32_t n_windows, const uint32_t* row_bounds, void* send, uint64_t send_capacity,
                             uint64_t* counts, uint64_t* visible);
int splat_cuda_render_records(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width, uint32_t height,
                              const float bg[3], const void* records, uint64_t n_records, uint32_t row0,
                              uint32_t rows, uint8_t* out, size_t out_bytes, splat_render_stats* stats);

/* As splat_cuda_render, but the frame goes to DEVICE memory dev_out (on the
 * handle's device) and the call only enqueues work on the handle's stream: it
 * does not wait for the GPU. Call splat_cuda_finish before using the stats;
 * it reports whether the frame overflowed the pair buffers, in which case the
 * buffers have been grown and the frame must be enqueued again. */
int splat_cuda_render_device(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width, uint32_t height,
                             const float bg[3], uint32_t downsample, uint8_t* dev_out, size_t out_bytes);

/* Terminal cells (the half-block widget HalfBlockImage, src/term.rs:109-130,
 * with ColorMode::color, src/term.rs:39-72): the frame is rendered and
 * downsampled as by splat_cuda_render, then each cell (x, y) of the
 * floor(w/f) x floor(floor(h/f) / 2) grid gets the pixel pair (x, 2y) over
 * (x, 2y + 1): foreground the top pixel, background the bottom one, as
 *   SPLAT_CELLS_TRUECOLOR  6 bytes: fg r, g, b, bg r, g, b
 *   SPLAT_CELLS_ANSI256    2 bytes: fg, bg xterm-256 indices (rgb_to_ansi256)
 * row-major in host memory cells_out (out_bytes at least cols * rows * 6 or
 * * 2); *cols and *rows receive the grid size (either may be NULL). A frame
 * of odd height drops its last row, as the widget does. */
#define SPLAT_CELLS_TRUECOLOR 0u
#define SPLAT_CELLS_ANSI256 1u
int splat_cuda_render_cells(splat_cuda_handle* h, const splat_view_desc* view, uint32_t width, uint32_t height,
                            const float bg[3], uint32_t downsample, uint32_t mode, uint8_t* cells_out,
                            size_t out_bytes, uint32_t* cols, uint32_t* rows, splat_render_stats* stats);

/* Waits for the frames enqueued by splat_cuda_render_device, fills the stats
 * of the last one and reports whether it overflowed the pair buffers
 * (*regrown = 1: the buffers have been grown; enqueue the frame again). A
 * last frame that needs more pairs than the pair limit (or device memory)
 * allows is drawn again in windows of tiles into its destination before
 * this call returns (*regrown = 0, complete stats). */
int splat_cuda_finish(splat_cuda_handle* h, splat_render_stats* stats, int* regrown);

/* Uses `stream` (a cudaStream_t on the handle's device; NULL restores the
 * handle's own stream) for all later work of this handle. */
int splat_cuda_set_stream(splat_cuda_handle* h, void* stream);
/* The cudaStream_t the handle currently launches on. */
void* splat_cuda_get_stream(splat_cuda_handle* h);

/* Renderer options. */
#define SPLAT_OPT_EXACT_BLEND 1u   /* 1: blend with the reference cpu backend's
                                      exact f32 arithmetic (polynomial exp,
                                      unfused multiply-adds); 0 (default): FMA
                                      and the hardware exp2 */
#define SPLAT_OPT_PAIR_CAPACITY 2u /* set the pair-buffer capacity (pairs) */
#define SPLAT_OPT_STAGE_EVENTS 3u  /* 1 (default): time stages with CUDA events */
#define SPLAT_OPT_DEBUG_CAPTURE 4u /* 1: keep per-splat projections for
                                      splat_cuda_debug_dump (costs n*44 bytes) */
#define SPLAT_OPT_FP64_CONICS 5u   /* read-only: splats of the last completed
                                      frame whose 2D covariance determinant fell
                                      below 1e-6 and was recomputed in FP64
                                      (FP16 scenes; 0 otherwise) */
#define SPLAT_OPT_KERNEL_LAUNCHES 6u /* kernels this handle has launched
                                        (set to reset the count) */
#define SPLAT_OPT_BLEND_CONFIG 7u  /* tile shape and blend threads, packed as
                                      tile_w | tile_h << 8 | threads << 16;
                                      shapes 8x8, 16x16 (default), 32x16 and
                                      128, 256 or 512 (default) threads. The
                                      image does not depend on it; the keys of
                                      splat_cuda_debug_dump use its tiles. */
#define SPLAT_OPT_SCENE_SPLATS 8u    /* read-only: gaussians in the scene */
#define SPLAT_OPT_PAIR_LIMIT 9u      /* largest pair-buffer capacity (pairs; 1024 ..
                                        2^30 - 1, the default); frames that need
                                        more are drawn in windows of tiles. The
                                        reference's test-only max_cap
                                        (src/render/gpu.rs:1273). */
/* Fault injection, for tests of the error paths; nothing faults on the GPU.
 * value = kind | microseconds << 8 (0 clears); each injection fires once.
 *   SPLAT_FAULT_ALLOC      the handle's next device allocation reports out of
 *                          memory without calling the allocator: the call
 *                          returns SPLAT_ERR_OOM and the handle stays usable
 *                          (pair-buffer growth absorbs it by trying a smaller
 *                          capacity).
 *   SPLAT_FAULT_LOST_WAIT  the tensor-core waits of the next frame (learned
 *                          colour) or training call also wait for a completion
 *                          that never arrives, giving up after `microseconds`:
 *                          the call returns SPLAT_ERR_TIMEOUT, the kernel frees
 *                          its tensor memory, a training step is dropped, and
 *                          the next call runs normally. */
#define SPLAT_OPT_INJECT_FAULT 10u
#define SPLAT_OPT_COUNT_EVALS 11u  /* 1: the blend (16x16 tiles, 512 threads, not
                                      exact) also counts its pixel/splat
                                      evaluations; a measurement mode */
#define SPLAT_OPT_BLEND_EVALS 12u  /* read-only: pixel/splat evaluations of the
                                      last completed frame (0 unless counted):
                                      the blend's work after early termination */
#define SPLAT_OPT_BBOX_PAIRS 13u  /* 1: pair each splat with every tile of its
                                      pixel bbox, as the reference's tiled
                                      backends do (src/render/cpu.rs:251-277);
                                      0 (default): a tile whose pixel centres
                                      all lie outside the splat's alpha = 1/255
                                      ellipse gets no pair (its contribution
                                      there is zero: the image is the same,
                                      `overlaps` counts the pairs drawn). The
                                      keys of splat_cuda_debug_dump follow it. */
#define SPLAT_FAULT_ALLOC 1u
#define SPLAT_FAULT_LOST_WAIT 2u
int splat_cuda_set_option(splat_cuda_handle* h, uint32_t option, uint64_t value);
int splat_cuda_get_option(splat_cuda_handle* h, uint32_t option, uint64_t* value);

/*
 * Intermediate buffers of the last completed render, for the oracle checks
 * (the bit-exact key/range gate). Any output pointer may be NULL.
 *   proj      n*8 floats per splat: x, y, ext_x, ext_y, depth, conic a, b, c
 *   visible   n bytes: 1 if the splat survived culling
 *   color     n*3 floats: the clamped view-dependent colour of visible splats
 *   keys      sorted (tile << 32 | depth bits) keys, up to key_capacity
 *   values    sorted splat indices, up to key_capacity
 *   ranges    per tile [begin, end) as 2 u32, tiles_x*tiles_y*2 entries
 *             (range_capacity entries at most)
 *   n_pairs   the pair count
 */
int splat_cuda_debug_dump(splat_cuda_handle* h, float* proj, uint8_t* visible, float* color, uint64_t* keys,
                          uint32_t* values, uint64_t key_capacity, uint32_t* ranges, uint64_t range_capacity,
                          uint64_t* n_pairs);

/*
 * Sorts one tile's pairs in place, for callers that cannot allocate device
 * memory (a host whose device memory belongs to another allocator, or code
 * that must not allocate while it runs). No counterpart in the reference: it
 * is the renderer's long-tile sort with its ping-pong buffer moved into a
 * static device array, so the call allocates nothing.
 *   words   DEVICE pointer to n words (depth bits << 32 | splat index), on the
 *           current device; on return they are ordered by depth, equal depths
 *           by splat index (the order the blend consumes).
 *   n       at most 1048576 (1 << 20) words; more is rejected with
 *           SPLAT_ERR_INVALID_ARG before anything is launched.
 *   stream  cudaStream_t to launch on (NULL: the legacy default stream).
 * The call only enqueues work. Every GPU that loads the library holds the
 * 8 MiB scratch array until the process exits; all calls on a device share
 * it, so calls whose work overlaps on the GPU race and must not be issued.
 * The first call on each device looks the array up (cudaGetSymbolAddress);
 * make that first call before any stream capture. No error text is kept. */
int splat_cuda_sort_tile_noalloc(uint64_t* words, uint32_t n, void* stream);

/* Frees the handle and its device memory. NULL is ignored. */
int splat_cuda_destroy(splat_cuda_handle* h);

/*
 * Batched rendering: many views of uneven resolution over several scenes,
 * each stage of the pipeline one launch over all views, the whole batch
 * recorded once as a CUDA graph and replayed by splat_cuda_batch_run. No
 * counterpart in the reference, whose Renderer draws one view per call
 * (src/render/mod.rs:89-96); every view's image equals what
 * splat_cuda_render draws for it alone.
 *
 * The scenes are handles from splat_cuda_create on one device; they must
 * outlive the batch and are only read. A view's frame goes to DEVICE memory
 * dev_out (floor(width/f) * floor(height/f) * 3 bytes). The batch owns its
 * per-view buffers, its stream and its graph; one thread at a time.
 */
typedef struct splat_cuda_batch splat_cuda_batch;

typedef struct splat_batch_view {
  uint32_t scene;       /* index into the scenes given at creation */
  uint32_t width;       /* 1..16384 */
  uint32_t height;      /* 1..16384 */
  uint32_t downsample;  /* 0 or 1: none; else a factor dividing the tile shape */
  splat_view_desc view;
  float bg[3];
  uint32_t reserved;    /* 0 */
  uint8_t* dev_out;     /* device frame of this view */
} splat_batch_view;

/* Tile shape and threads per CTA of the blend: (8,8), (16,16) or (32,16)
 * tiles with 128, 256 or 512 threads. */
typedef struct splat_blend_config {
  uint32_t tile_w, tile_h, threads;
} splat_blend_config;

typedef struct splat_tune_result {
  splat_blend_config config;
  uint32_t reserved;
  double ms;            /* mean device time of one batch (graph launch) */
} splat_tune_result;

/* Plans the batch with the default configuration (16x16 tiles, 512
 * threads), runs it once to size the pair buffers and records the graph. */
int splat_cuda_batch_create(splat_cuda_handle* const* scenes, uint32_t n_scenes, const splat_batch_view* views,
                            uint32_t n_views, splat_cuda_batch** out);
/* Text describing why the last splat_cuda_batch_create of this thread failed. */
const char* splat_cuda_batch_create_error(void);
/* Re-plans and re-records the batch for another blend configuration. */
int splat_cuda_batch_set_config(splat_cuda_batch* b, const splat_blend_config* config);
int splat_cuda_batch_get_config(const splat_cuda_batch* b, splat_blend_config* config);
/* The tuner: times `reps` graph launches of every supported configuration
 * (after one warm-up launch each), twice over the list, keeps each
 * configuration's faster time and the fastest configuration, and re-records
 * the batch with it. Writes up to `capacity` results (every configuration
 * tried, in the order tried, with its time) and their number to
 * *n_results. */
int splat_cuda_batch_autotune(splat_cuda_batch* b, uint32_t reps, splat_tune_result* results, uint32_t capacity,
                              uint32_t* n_results);
/* Launches the recorded graph on the batch's stream; does not wait. */
int splat_cuda_batch_run(splat_cuda_batch* b);
/* Waits for the launched batches; per_view (n_views entries, may be NULL)
 * gets each view's visible splats and pairs and the device times of the
 * last batch's stages (projection, binning + sorts, blend: the same for
 * every view), total_ms (may be NULL) the device time of the last batch. *regrown = 1 when a batch overflowed the
 * pair buffers: they have been grown and the graph re-recorded; run again. */
int splat_cuda_batch_finish(splat_cuda_batch* b, splat_render_stats* per_view, double* total_ms, int* regrown);
/* Options: SPLAT_OPT_EXACT_BLEND and SPLAT_OPT_KERNEL_LAUNCHES as for a
 * renderer (setting EXACT_BLEND re-records the graph). */
int splat_cuda_batch_set_option(splat_cuda_batch* b, uint32_t option, uint64_t value);
int splat_cuda_batch_get_option(const splat_cuda_batch* b, uint32_t option, uint64_t* value);
/* Uses `stream` (NULL: the batch's own) for later launches of the graph. */
int splat_cuda_batch_set_stream(splat_cuda_batch* b, void* stream);
void* splat_cuda_batch_get_stream(const splat_cuda_batch* b);
/* Text describing the last failure on this batch ("" if none). */
const char* splat_cuda_batch_last_error(const splat_cuda_batch* b);
/* Frees the batch (not its scenes). NULL is ignored. */
int splat_cuda_batch_destroy(splat_cuda_batch* b);

/* Text describing the last failure on this handle ("" if none). */
const char* splat_cuda_last_error(const splat_cuda_handle* h);

/*
 * Learned colour. No counterpart in the reference, which evaluates degree-3
 * SH per splat (src/sh.rs:39-64 via src/render/mod.rs:250-257). Each splat's
 * 48 SH floats are replaced by SPLAT_MLP_LATENT fp16 latents, decoded by one
 * MLP shared by all splats:
 *   x = [latent (16) | unit view direction p - eye (3) | 1 | 0 x 12]
 *   rgb = sigmoid(W3 relu(W2 relu(W1 x) + b2) + b3)
 * with fp16 weights and fp32 accumulation on the tensor cores; b1 is W1's
 * column 19. The view direction is the one the SH colour would be evaluated
 * at (normalize_or_zero(p - eye), src/render/mod.rs:250-252).
 *
 * Parameter vector: SPLAT_MLP_PARAMS values (fp32 masters or fp16 bit
 * patterns), matrices row-major [out][in], at these offsets:
 */
#define SPLAT_MLP_LATENT 16u
#define SPLAT_MLP_W1 0u    /* 64 x 32; inputs 0-15 latent, 16-18 direction,
                              19 the bias b1, 20-31 zero */
#define SPLAT_MLP_W2 2048u /* 64 x 64 */
#define SPLAT_MLP_B2 6144u /* 64 */
#define SPLAT_MLP_W3 6208u /* 16 x 64; rows 0-2 give RGB, rows 3-15 zero */
#define SPLAT_MLP_B3 7232u /* 16; entries 3-15 zero */
#define SPLAT_MLP_PARAMS 7248u

/* A renderer whose colour is the learned MLP's. `geometry` is an FP16 scene
 * (precision SPLAT_PRECISION_FP16; sh_degree and sh_f16 are ignored):
 * positions f32, scales/rotations/opacities f16. latents: n *
 * SPLAT_MLP_LATENT fp16 values, splat-major; mlp_params: SPLAT_MLP_PARAMS
 * fp16 values. 64 bytes per splat are read per frame (against 240 for the
 * FP32 SH3 scene). The handle renders with splat_cuda_render and friends,
 * and in batches (splat_cuda_batch_create) beside SH scenes. */
int splat_cuda_create_learned(const splat_scene_desc* geometry, const uint16_t* latents, const uint16_t* mlp_params,
                              int device, splat_cuda_handle** out);

/*
 * Training of the latents and the MLP on the exact SH colours of an SH scene
 * (a handle from splat_cuda_create, FP32 or FP16 storage), on the scene's
 * device. Targets are the reference's SH colour (src/sh.rs:39-64), clamped to
 * [0, 1] (a sigmoid cannot exceed 1), at `directions` Fibonacci-sphere
 * directions per splat (the construction of src/gen.rs:213-219). An epoch
 * visits every (splat, direction) sample once, in an order shuffled per
 * epoch; a step takes `batch` samples (the last step of an epoch fewer), runs
 * forward and backward on the tensor cores and applies Adam to the MLP and
 * (lazily, rows touched by the step only) to the latents. Loss: mean squared
 * error over samples and channels. The scene handle must outlive the learner.
 */
typedef struct splat_cuda_learner splat_cuda_learner;

typedef struct splat_learn_config {
  uint32_t directions; /* per splat, e.g. 256 */
  uint32_t batch;      /* samples per step: a multiple of 128, <= 2^22 */
  float lr, beta1, beta2, eps; /* Adam, e.g. 1e-3, 0.9, 0.999, 1e-8 */
  uint64_t seed;       /* initial parameters and the shuffles */
} splat_learn_config;

typedef struct splat_learn_stats {
  uint64_t steps;             /* steps since creation or set_params */
  double epochs;              /* the same in epochs */
  double mean_loss;           /* mean of the step losses of this call */
  double last_loss;           /* loss of the last step */
  double ms;                  /* device time of this call */
  uint64_t steps_per_epoch;
  uint64_t samples_per_epoch; /* n * directions */
} splat_learn_stats;

/* Learner options (read-only, splat_cuda_learner_get_option). */
#define SPLAT_LEARN_STEPS_PER_EPOCH 100u
#define SPLAT_LEARN_SHUFFLE_BITS 101u /* the sample shuffle's word width */
#define SPLAT_LEARN_TRAIN_CTAS 102u   /* CTAs of the training kernel */

/* Initial parameters: He-uniform hidden layers, Xavier-uniform output, zero
 * biases; latents a fixed random projection of each splat's colour
 * coefficients. */
int splat_cuda_learner_create(const splat_cuda_handle* sh_scene, const splat_learn_config* config,
                              splat_cuda_learner** out);
const char* splat_cuda_learner_create_error(void);
/* Runs `steps` training steps (blocks until done). */
int splat_cuda_learner_train(splat_cuda_learner* l, uint64_t steps, splat_learn_stats* stats);
/* Replaces the fp32 master parameters (SPLAT_MLP_PARAMS) and/or latents
 * (n * 16; either may be NULL) and resets Adam and the step count. */
int splat_cuda_learner_set_params(splat_cuda_learner* l, const float* params, const float* latents);
/* Copies the current parameters out; any pointer may be NULL. params and
 * latents are the fp32 masters, the _f16 ones the fp16 values the kernels use
 * (what splat_cuda_create_learned takes). */
int splat_cuda_learner_params(splat_cuda_learner* l, float* params, float* latents, uint16_t* params_f16,
                              uint16_t* latents_f16);
/* Checkpoint of the training state: the fp32 parameter and latent masters,
 * their Adam moments, the latent rows' update stamps, the step count (Adam's
 * bias correction and the position in the epoch's shuffle) and the loss
 * record, as one byte blob with a header. A learner for the same scene and
 * configuration (splats, directions, batch, seed, SH degree; checked on
 * load) that loads it trains on from where the saver stopped, step for step.
 * No counterpart in the reference (which renders only). */
size_t splat_cuda_learner_state_bytes(const splat_cuda_learner* l);
int splat_cuda_learner_save_state(splat_cuda_learner* l, void* out, size_t bytes);
int splat_cuda_learner_load_state(splat_cuda_learner* l, const void* data, size_t bytes);
/* One step that also reports its gradient before Adam applies it: d loss /
 * d params (SPLAT_MLP_PARAMS) and d loss / d latents (n * 16, zero for rows
 * the step did not sample); either may be NULL. */
int splat_cuda_learner_step_debug(splat_cuda_learner* l, float* grad_params, float* grad_latents);
/* The learner's unit directions (directions * 3 floats). */
int splat_cuda_learner_directions(const splat_cuda_learner* l, float* dirs);
/* SPLAT_LEARN_* and SPLAT_OPT_KERNEL_LAUNCHES. */
int splat_cuda_learner_get_option(const splat_cuda_learner* l, uint32_t option, uint64_t* value);
/* SPLAT_OPT_INJECT_FAULT with SPLAT_FAULT_LOST_WAIT (a test of the timeout
 * path: the steps of the next train or step_debug call give up on a wait and
 * are dropped; that call returns SPLAT_ERR_TIMEOUT). */
int splat_cuda_learner_set_option(splat_cuda_learner* l, uint32_t option, uint64_t value);
const char* splat_cuda_learner_last_error(const splat_cuda_learner* l);
int splat_cuda_learner_destroy(splat_cuda_learner* l);

/* Forward and backward of the MLP on `count` explicit samples (latents fp16
 * count * 16, unit directions and targets count * 3), with fp32 parameters
 * rounded to fp16 as the learner does: the loss, each sample's output and
 * the gradients of the mean loss. The training kernel's own code path, for
 * checking it against an independent computation. Allocates temporaries. */
int splat_cuda_mlp_gradient(int device, const float* params, const uint16_t* latents, const float* dirs,
                            const float* targets, uint32_t count, float* grad_params, float* grad_latents,
                            float* outputs, double* loss);

#ifdef __cplusplus
}
#endif

#endif /* SPLAT_CUDA_H */
