// Kernel (d): per-tile front-to-back blend with the terminal box-filter
// downsample fused in.
//
// One CTA per 16x16 tile, one pixel per thread, over the tile's pairs in
// depth order (sorted per tile by the binning stage); each warp covers an 8x4 block
// of the tile so a splat whose pixel bbox misses the block is skipped by the
// whole warp. The tile's depth-sorted splat list is walked in batches of 256:
// the CTA gathers the batch's 48-byte records into shared memory (one per
// thread, coalesced index loads, the next batch's gather in flight while the
// current one blends), storing each splat's bbox as a row/column bit mask so
// the per-pixel bbox test is one AND and one compare; then every pixel blends
// the batch front to back. A pixel stops once its transmittance drops below T_MIN; the CTA stops
// when a block vote finds no live pixel (the reference stops a tile when all
// its row masks are empty, src/render/cpu.rs:693-702).
//
// Per pixel and splat the arithmetic is that of raster_tile
// (src/render/cpu.rs:638-703): power = (-a/2 dx^2 + -c/2 dy^2) + (-b dy) dx
// inside the splat's pixel bbox, alpha = min(opacity * exp(power), 0.99),
// masked by power <= 0 and alpha >= 1/255, C += colour * alpha * T,
// T *= 1 - alpha. EXACT = true evaluates it with the reference's x86 f32
// semantics (unfused multiply-adds, the polynomial exp_neg of
// src/render/simd.rs:315-331), which reproduces the cpu backend's image bit
// for bit; EXACT = false uses FMA and the hardware exp2 (the default).
// The result is quantised with to_u8 (src/render/mod.rs:282-285) and, for a
// downsample factor f dividing 16, averaged over f x f blocks in shared
// memory with term::downsample's truncating integer division
// (src/term.rs:74-99); other factors go through a full-resolution scratch
// frame and k_downsample.
#include "common.cuh"

namespace splat {
namespace {

constexpr float kLog2e = 1.44269504088896340736f;

// src/render/simd.rs:315-331 with the portable F4's unfused mul_add.
__device__ __forceinline__ float exp_neg_exact(float xin) {
  const float C1 = 0.6933594f;
  const float C2 = -2.1219444e-4f;
  const float x = fmaxf(xin, -87.0f);
  const float n = rintf(__fmul_rn(x, kLog2e));
  const float f = __fsub_rn(__fsub_rn(x, __fmul_rn(n, C1)), __fmul_rn(n, C2));
  float p = 1.9875691e-4f;
  p = __fadd_rn(1.3981999e-3f, __fmul_rn(p, f));
  p = __fadd_rn(8.333452e-3f, __fmul_rn(p, f));
  p = __fadd_rn(4.1665796e-2f, __fmul_rn(p, f));
  p = __fadd_rn(1.6666665e-1f, __fmul_rn(p, f));
  p = __fadd_rn(0.5f, __fmul_rn(p, f));
  const float f2 = __fmul_rn(f, f);
  const float r = __fadd_rn(__fadd_rn(f, 1.0f), __fmul_rn(p, f2));
  return __fmul_rn(r, __int_as_float(((int)n + 127) << 23));
}

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// to_u8 (src/render/mod.rs:282-285)
__device__ __forceinline__ uint32_t to_u8(float v) {
  const float c = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);  // f32::clamp; NaN passes
  const float q = __fadd_rn(__fmul_rn(c, 255.0f), 0.5f);
  if (!(q > 0.0f)) return 0u;
  if (q >= 255.0f) return 255u;
  return (uint32_t)q;
}

// One splat's contribution test at this pixel: returns alpha, or 0 when the
// splat does not contribute (outside the bbox, power > 0, alpha < 1/255).
template <bool EXACT>
__device__ __forceinline__ float splat_alpha(uint32_t m, uint32_t mybits, const float4& a, const float4& b,
                                             float fx05, float gbase, float lanef, float rowc, float lxf, float lyf) {
  float pw, alpha;
  if (EXACT) {
    const float cx0 = __fsub_rn(fx05, a.x);
    const float dx = __fadd_rn(lanef, __fadd_rn(gbase, cx0));
    const float qx = __fmul_rn(__fmul_rn(dx, dx), a.z);
    const float dy = __fsub_rn(rowc, a.y);
    const float qy = __fmul_rn(__fmul_rn(b.x, dy), dy);
    const float bdy = __fmul_rn(a.w, dy);
    pw = __fadd_rn(__fadd_rn(qx, qy), __fmul_rn(bdy, dx));
    alpha = fminf(__fmul_rn(exp_neg_exact(pw), b.y), kAlphaMax);
  } else {
    const float dx = lxf - a.x;
    const float dy = lyf - a.y;
    pw = fmaf(dx, fmaf(a.z, dx, a.w * dy), (b.x * dy) * dy);
    alpha = fminf(ex2_approx(pw) * b.y, kAlphaMax);
  }
  // A pixel outside the splat's bbox is at least half a pixel beyond the
  // ellipse on which opacity * exp(power) = 1/255 (the bbox is the k-sigma
  // extent rounded outwards and pixels are sampled at their centres), so the
  // alpha test alone excludes it in the default path; the exact path also
  // tests the bbox, as the reference does.
  const bool on = (pw <= 0.0f) && (alpha >= kAlphaMin) && (!EXACT || (m & mybits) == mybits);
  return on ? alpha : 0.0f;
}

template <bool EXACT>
__device__ __forceinline__ void accumulate(float alpha, const float4& b, float blue, float& T, float& cr, float& cg,
                                           float& cb) {
  if (EXACT) {
    const float w = __fmul_rn(alpha, T);
    cr = __fadd_rn(cr, __fmul_rn(b.z, w));
    cg = __fadd_rn(cg, __fmul_rn(b.w, w));
    cb = __fadd_rn(cb, __fmul_rn(blue, w));
    T = __fmul_rn(T, __fsub_rn(1.0f, alpha));
  } else {
    const float w = alpha * T;
    cr = fmaf(b.z, w, cr);
    cg = fmaf(b.w, w, cg);
    cb = fmaf(blue, w, cb);
    T = T - w;
  }
}

template <bool EXACT>
__global__ void __launch_bounds__(256) k_blend(FrameParams fp, const Record* __restrict__ rec,
                                               const uint64_t* __restrict__ pairs, const uint2* __restrict__ ranges,
                                               uint8_t* __restrict__ out, uint8_t* __restrict__ full) {
  // Per batch entry: the splat's pixel bbox clipped to this tile as a bit
  // mask (columns in bits 0-15, rows in bits 16-31), its geometry and colour.
  // The default path stores the centre relative to the tile's first pixel
  // centre and the conic pre-scaled by log2(e) for exp2. Each warp then lists
  // the entries whose bbox meets its 8x4 block and walks only those, two at a
  // time (the second splat's alpha is computed while the first one's is being
  // accumulated).
  __shared__ float4 s_a[256];  // x, y, -a/2, -b
  __shared__ float4 s_b[256];  // -c/2, opacity, red, green
  __shared__ uint32_t s_mask[256];
  __shared__ float s_c[256];  // blue
  __shared__ uint8_t s_list[8][256];
  __shared__ uint32_t s_px[256];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t tile = blockIdx.x;
  const uint32_t tx = tile % fp.tiles_x, ty = tile / fp.tiles_x;
  const uint32_t ox = tx * kTile, oy = ty * kTile;
  const uint32_t wx = (warp & 1) * 8, wy = (warp >> 1) * 4;
  const uint32_t lx = wx + (lane & 7), ly = wy + (lane >> 3);
  const uint32_t px = ox + lx, py = oy + ly;
  const bool inside = px < fp.w && py < fp.h;
  const uint32_t mybits = (1u << lx) | (1u << (16 + ly));
  const uint32_t wxbits = 0xFFu << wx, wybits = 0xFu << (16 + wy);
  const uint2 range = ranges[tile];
  const uint32_t begin = range.x, n = range.y > range.x ? range.y - range.x : 0u;
  auto splat_at = [&](uint32_t p) -> uint32_t { return (uint32_t)pairs[begin + p]; };

  // EXACT: dx = lane + ((g*4) + ((ox + 0.5) - x)), dy = ((oy + ly) + 0.5) - y
  // in the reference's association (src/render/cpu.rs:658-671).
  const float fx05 = __fadd_rn((float)ox, 0.5f);
  const float gbase = (float)(lx & ~3u), lanef = (float)(lx & 3u);
  const float rowc = __fadd_rn(__fadd_rn((float)oy, (float)ly), 0.5f);
  const float lxf = (float)lx, lyf = (float)ly;
  const float ox05 = (float)ox + 0.5f, oy05 = (float)oy + 0.5f;

  float T = 1.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
  bool done = !inside;

  // The next batch's record is gathered into registers while the current
  // batch is blended.
  Record nr;
  bool has = false;
  if ((uint32_t)tid < n) {
    nr = rec[splat_at(tid)];
    has = true;
  }
  for (uint32_t start = 0; start < n; start += 256) {
    if (has) {
      const uint32_t bx = __float_as_uint(nr.r2.y), by = __float_as_uint(nr.r2.z);
      const int x0 = min(max((int)(bx & 0xFFFFu) - (int)ox, 0), 16), x1 = min(max((int)(bx >> 16) - (int)ox, 0), 16);
      const int y0 = min(max((int)(by & 0xFFFFu) - (int)oy, 0), 16), y1 = min(max((int)(by >> 16) - (int)oy, 0), 16);
      const uint32_t xb = ((1u << x1) - 1u) & ~((1u << x0) - 1u);
      const uint32_t yb = ((1u << y1) - 1u) & ~((1u << y0) - 1u);
      s_mask[tid] = xb | (yb << 16);
      float4 a = nr.r0, b = nr.r1;
      if (!EXACT) {
        a.x -= ox05;
        a.y -= oy05;
        a.z *= kLog2e;
        a.w *= kLog2e;
        b.x *= kLog2e;
      }
      s_a[tid] = a;
      s_b[tid] = b;
      s_c[tid] = nr.r2.x;
    }
    __syncthreads();
    const uint32_t nxt = start + 256 + tid;
    has = nxt < n;
    if (has) nr = rec[splat_at(nxt)];
    const uint32_t cnt = min(256u, n - start);
    // This warp's list of batch entries whose bbox meets its block.
    uint32_t len = 0;
    if (__any_sync(0xffffffffu, !done)) {
      for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
        const uint32_t e = c0 + lane;
        const uint32_t m = e < cnt ? s_mask[e] : 0u;
        const bool hit = (m & wxbits) && (m & wybits);
        const uint32_t bal = __ballot_sync(0xffffffffu, hit);
        if (hit) s_list[warp][len + __popc(bal & ((1u << lane) - 1u))] = (uint8_t)e;
        len += __popc(bal);
      }
      __syncwarp();
    }
    if (!done) {
      uint32_t k = 0;
      for (; k + 1 < len; k += 2) {
        const uint32_t j0 = s_list[warp][k], j1 = s_list[warp][k + 1];
        const float4 a0 = s_a[j0], b0 = s_b[j0];
        const float4 a1 = s_a[j1], b1 = s_b[j1];
        const float al0 = splat_alpha<EXACT>(s_mask[j0], mybits, a0, b0, fx05, gbase, lanef, rowc, lxf, lyf);
        const float al1 = splat_alpha<EXACT>(s_mask[j1], mybits, a1, b1, fx05, gbase, lanef, rowc, lxf, lyf);
        if (al0 > 0.0f) {
          accumulate<EXACT>(al0, b0, s_c[j0], T, cr, cg, cb);
          if (T < kTMin) {
            done = true;
            break;
          }
        }
        if (al1 > 0.0f) {
          accumulate<EXACT>(al1, b1, s_c[j1], T, cr, cg, cb);
          if (T < kTMin) {
            done = true;
            break;
          }
        }
      }
      if (!done && k < len) {
        const uint32_t j0 = s_list[warp][k];
        const float4 a0 = s_a[j0], b0 = s_b[j0];
        const float al0 = splat_alpha<EXACT>(s_mask[j0], mybits, a0, b0, fx05, gbase, lanef, rowc, lxf, lyf);
        if (al0 > 0.0f) {
          accumulate<EXACT>(al0, b0, s_c[j0], T, cr, cg, cb);
          if (T < kTMin) done = true;
        }
      }
    }
    if (__syncthreads_count(!done) == 0) break;
  }

  // C + T * bg, quantised (the reference adds unfused: c + (t * bg)).
  const uint32_t qr = to_u8(__fadd_rn(cr, __fmul_rn(T, fp.bg[0])));
  const uint32_t qg = to_u8(__fadd_rn(cg, __fmul_rn(T, fp.bg[1])));
  const uint32_t qb = to_u8(__fadd_rn(cb, __fmul_rn(T, fp.bg[2])));
  const uint32_t f = fp.downsample;
  if (f == 1) {
    if (inside) {
      uint8_t* o = out + ((size_t)py * fp.w + px) * 3;
      o[0] = (uint8_t)qr;
      o[1] = (uint8_t)qg;
      o[2] = (uint8_t)qb;
    }
    return;
  }
  if (kTile % f != 0) {  // factor 3 etc.: full-resolution scratch, then k_downsample
    if (inside) {
      uint8_t* o = full + ((size_t)py * fp.w + px) * 3;
      o[0] = (uint8_t)qr;
      o[1] = (uint8_t)qg;
      o[2] = (uint8_t)qb;
    }
    return;
  }
  s_px[ly * kTile + lx] = qr | (qg << 8) | (qb << 16);
  __syncthreads();
  const uint32_t per = kTile / f;  // output pixels per tile edge
  if ((uint32_t)tid < per * per) {
    const uint32_t bxl = tid % per, byl = tid / per;
    const uint32_t obx = ox / f + bxl, oby = oy / f + byl;
    if (obx < fp.out_w && oby < fp.out_h) {
      uint32_t acc[3] = {0u, 0u, 0u};
      for (uint32_t sy = 0; sy < f; sy++)
        for (uint32_t sx = 0; sx < f; sx++) {
          const uint32_t p = s_px[(byl * f + sy) * kTile + bxl * f + sx];
          acc[0] += p & 255u;
          acc[1] += (p >> 8) & 255u;
          acc[2] += (p >> 16) & 255u;
        }
      const uint32_t nn = f * f;
      uint8_t* o = out + ((size_t)oby * fp.out_w + obx) * 3;
      o[0] = (uint8_t)(acc[0] / nn);
      o[1] = (uint8_t)(acc[1] / nn);
      o[2] = (uint8_t)(acc[2] / nn);
    }
  }
}

// term::downsample (src/term.rs:74-99) for factors that do not divide the tile.
__global__ void k_downsample(FrameParams fp, const uint8_t* __restrict__ full, uint8_t* __restrict__ out) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= fp.out_w || y >= fp.out_h) return;
  const uint32_t f = fp.downsample;
  uint32_t acc[3] = {0u, 0u, 0u};
  for (uint32_t sy = 0; sy < f; sy++) {
    const uint8_t* row = full + ((size_t)(y * f + sy) * fp.w + x * f) * 3;
    for (uint32_t sx = 0; sx < f; sx++) {
      acc[0] += row[3 * sx];
      acc[1] += row[3 * sx + 1];
      acc[2] += row[3 * sx + 2];
    }
  }
  const uint32_t nn = f * f;
  uint8_t* o = out + ((size_t)y * fp.out_w + x) * 3;
  o[0] = (uint8_t)(acc[0] / nn);
  o[1] = (uint8_t)(acc[1] / nn);
  o[2] = (uint8_t)(acc[2] / nn);
}

}  // namespace

cudaError_t launch_blend(const FrameParams& fp, const Record* rec, const uint64_t* pairs, const uint2* ranges,
                         bool exact, uint8_t* out, uint8_t* full_scratch, cudaStream_t stream, uint32_t* launches) {
  const unsigned tiles = fp.tiles_x * fp.tiles_y;
  if (tiles == 0) return cudaSuccess;
  if (exact)
    k_blend<true><<<tiles, 256, 0, stream>>>(fp, rec, pairs, ranges, out, full_scratch);
  else
    k_blend<false><<<tiles, 256, 0, stream>>>(fp, rec, pairs, ranges, out, full_scratch);
  *launches += 1;
  if (fp.downsample > 1 && kTile % fp.downsample != 0 && fp.out_w > 0 && fp.out_h > 0) {
    dim3 grid((fp.out_w + 127) / 128, fp.out_h);
    k_downsample<<<grid, 128, 0, stream>>>(fp, full_scratch, out);
    *launches += 1;
  }
  return cudaGetLastError();
}

}  // namespace splat
