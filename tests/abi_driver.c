/* A C host of the C ABI (include/splat_cuda.h): the calls a Rust or C
 * backend makes, in plain C99. It builds an 8x8x8 lattice scene in memory,
 * renders it at 160x96 through splat_cuda_render and as terminal cells
 * through splat_cuda_render_cells, checks the reference's error behaviour
 * (a frame past the pixel limit is rejected with its message) and writes the
 * frame and the cells to the files given as arguments. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "splat_cuda.h"

#define SIDE 8
#define N (SIDE * SIDE * SIDE)
#define W 160
#define H 96

static int fail(const char* what, int rc, const char* msg) {
  fprintf(stderr, "%s failed: %d %s\n", what, rc, msg ? msg : "");
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s frame.rgb cells.bin\n", argv[0]);
    return 2;
  }
  if (splat_cuda_abi_version() != SPLAT_CUDA_ABI_VERSION) return fail("abi version", 0, "");
  if (strcmp(splat_cuda_backend_name(), "cuda") != 0) return fail("backend name", 0, "");
  static float pos[N * 3], opa[N], col[N * 3], cov[N * 6];
  for (int i = 0; i < N; i++) {
    const int x = i % SIDE, y = (i / SIDE) % SIDE, z = i / (SIDE * SIDE);
    const float s = 0.05f;
    pos[3 * i] = -1.0f + 2.0f * (float)x / (SIDE - 1);
    pos[3 * i + 1] = -1.0f + 2.0f * (float)y / (SIDE - 1);
    pos[3 * i + 2] = -1.0f + 2.0f * (float)z / (SIDE - 1);
    opa[i] = 0.9f;
    col[3 * i] = (float)x / (SIDE - 1);
    col[3 * i + 1] = (float)y / (SIDE - 1);
    col[3 * i + 2] = (float)z / (SIDE - 1);
    cov[6 * i] = s * s;  /* identity rotation: diag(s^2) */
    cov[6 * i + 1] = 0.0f;
    cov[6 * i + 2] = 0.0f;
    cov[6 * i + 3] = s * s;
    cov[6 * i + 4] = 0.0f;
    cov[6 * i + 5] = s * s;
  }
  splat_scene_desc d;
  memset(&d, 0, sizeof d);
  d.n = N;
  d.sh_degree = 0;
  d.precision = SPLAT_PRECISION_FP32;
  d.positions = pos;
  d.opacities = opa;
  d.colors = col;
  d.cov3d = cov;
  splat_cuda_handle* h = NULL;
  int rc = splat_cuda_create(&d, 0, &h);
  if (rc != SPLAT_OK) return fail("create", rc, splat_cuda_create_error());
  splat_view_desc v;
  memset(&v, 0, sizeof v);
  v.eye[2] = -4.0f;
  v.right[0] = 1.0f;
  v.down[1] = 1.0f;
  v.forward[2] = 1.0f;
  v.fov_y = 50.0f * 3.14159265f / 180.0f;
  v.near_plane = 0.05f;
  const float bg[3] = {0.1f, 0.1f, 0.1f};
  static unsigned char frame[W * H * 3];
  splat_render_stats st;
  rc = splat_cuda_render(h, &v, W, H, bg, 1, frame, sizeof frame, &st);
  if (rc != SPLAT_OK) return fail("render", rc, splat_cuda_last_error(h));
  if (st.visible != N || st.overlaps == 0) return fail("stats", 0, "");
  rc = splat_cuda_render(h, &v, 20000, H, bg, 1, frame, sizeof frame, &st);
  if (rc != SPLAT_ERR_INVALID_ARG || !strstr(splat_cuda_last_error(h), "pixel limit"))
    return fail("pixel limit", rc, splat_cuda_last_error(h));
  rc = splat_cuda_render(h, &v, W, H, bg, 1, frame, sizeof frame, &st);
  if (rc != SPLAT_OK) return fail("render again", rc, splat_cuda_last_error(h));
  static unsigned char cells[W * (H / 2) * 2];
  uint32_t cols = 0, rows = 0;
  rc = splat_cuda_render_cells(h, &v, W, H, bg, 1, SPLAT_CELLS_ANSI256, cells, sizeof cells, &cols, &rows, NULL);
  if (rc != SPLAT_OK || cols != W || rows != H / 2) return fail("cells", rc, splat_cuda_last_error(h));
  FILE* f = fopen(argv[1], "wb");
  if (!f || fwrite(frame, 1, sizeof frame, f) != sizeof frame) return fail("write frame", 0, argv[1]);
  fclose(f);
  f = fopen(argv[2], "wb");
  if (!f || fwrite(cells, 1, sizeof cells, f) != sizeof cells) return fail("write cells", 0, argv[2]);
  fclose(f);
  splat_cuda_destroy(h);
  printf("ok visible %llu pairs %llu\n", (unsigned long long)st.visible, (unsigned long long)st.overlaps);
  return 0;
}
