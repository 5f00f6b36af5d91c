// Terminal cells from a frame on the device: the half-block widget of
// src/term.rs:109-130 (each cell shows the pixel pair (x, 2y) over
// (x, 2y + 1): foreground the top pixel, background the bottom one) with the
// colour mapping of ColorMode::color (src/term.rs:39-45): the RGB triple
// (truecolor) or the nearest xterm-256 colour of rgb_to_ansi256
// (src/term.rs:48-72), in the same integer arithmetic.
#include "common.cuh"

namespace splat {
namespace {

__device__ __forceinline__ uint8_t rgb_to_ansi256(uint32_t r, uint32_t g, uint32_t b) {
  const int levels[6] = {0, 95, 135, 175, 215, 255};
  auto cube_idx = [](int v) -> int { return v < 48 ? 0 : (v < 115 ? 1 : min((v - 35) / 40, 5)); };
  const int ri = cube_idx((int)r), gi = cube_idx((int)g), bi = cube_idx((int)b);
  const int avg = ((int)r + (int)g + (int)b) / 3;
  const int gray_idx = min(max((avg - 3) / 10, 0), 23);
  const int gray = 8 + gray_idx * 10;
  auto sq = [](int d) { return d * d; };
  const int dg = sq(gray - (int)r) + sq(gray - (int)g) + sq(gray - (int)b);
  const int dc = sq(levels[ri] - (int)r) + sq(levels[gi] - (int)g) + sq(levels[bi] - (int)b);
  return dg < dc ? (uint8_t)(232 + gray_idx) : (uint8_t)(16 + 36 * ri + 6 * gi + bi);
}

__global__ void k_cells(const uint8_t* __restrict__ frame, uint32_t w, uint32_t cols, uint32_t rows, uint32_t mode,
                        uint8_t* __restrict__ cells) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cols * rows) return;
  const uint32_t cx = i % cols, cy = i / cols;
  const uint8_t* t = frame + ((size_t)(2 * cy) * w + cx) * 3;
  const uint8_t* b = frame + ((size_t)(2 * cy + 1) * w + cx) * 3;
  if (mode == SPLAT_CELLS_TRUECOLOR) {
    uint8_t* o = cells + (size_t)i * 6;
    o[0] = t[0];
    o[1] = t[1];
    o[2] = t[2];
    o[3] = b[0];
    o[4] = b[1];
    o[5] = b[2];
  } else {
    cells[(size_t)i * 2] = rgb_to_ansi256(t[0], t[1], t[2]);
    cells[(size_t)i * 2 + 1] = rgb_to_ansi256(b[0], b[1], b[2]);
  }
}

}  // namespace

cudaError_t launch_cells(const uint8_t* frame, uint32_t w, uint32_t cols, uint32_t rows, uint32_t mode, uint8_t* cells,
                         cudaStream_t stream, uint32_t* launches) {
  const uint32_t n = cols * rows;
  if (n == 0) return cudaSuccess;
  k_cells<<<(n + 255) / 256, 256, 0, stream>>>(frame, w, cols, rows, mode, cells);
  *launches += 1;
  return cudaGetLastError();
}

}  // namespace splat
