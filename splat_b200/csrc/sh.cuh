// Spherical-harmonics colour, shared by the projection (project.cu) and the
// learned-colour trainer's targets (mlp.cu): `sh::eval_rest` of the reference
// (src/sh.rs:39-64), operation by operation. Compiled with --fmad=false (the
// projection) every value equals the reference's unfused x86 f32 result.
#pragma once

namespace splat {
namespace sh {

// src/sh.rs:5-22
constexpr float kShC1 = 0.4886025f;
constexpr float kShC2_0 = 1.0925485f, kShC2_1 = -1.0925485f, kShC2_2 = 0.31539157f, kShC2_3 = -1.0925485f,
                kShC2_4 = 0.54627424f;
constexpr float kShC3_0 = -0.5900436f, kShC3_1 = 2.8906114f, kShC3_2 = -0.4570458f, kShC3_3 = 0.37317633f,
                kShC3_4 = -0.4570458f, kShC3_5 = 1.4453057f, kShC3_6 = -0.5900436f;

// sh::eval_rest added to c; R(coef, ch) loads rest coefficient `coef`,
// channel `ch` of the splat.
template <int DEG, class Load>
__device__ __forceinline__ void eval_sh(Load&& R, float x, float y, float z, float c[3]) {
  if constexpr (DEG >= 1) {
    float r[3];
#pragma unroll
    for (int ch = 0; ch < 3; ch++) {
      float v = kShC1 * (((-y) * R(0, ch) + z * R(1, ch)) - x * R(2, ch));
      r[ch] = v;
    }
    if constexpr (DEG >= 2) {
      float xx = x * x, yy = y * y, zz = z * z;
      float xy = x * y, yz = y * z, xz = x * z;
      float b3 = kShC2_0 * xy, b4 = kShC2_1 * yz, b5 = kShC2_2 * ((2.0f * zz - xx) - yy), b6 = kShC2_3 * xz,
            b7 = kShC2_4 * (xx - yy);
#pragma unroll
      for (int ch = 0; ch < 3; ch++) {
        float s = b3 * R(3, ch);
        s = s + b4 * R(4, ch);
        s = s + b5 * R(5, ch);
        s = s + b6 * R(6, ch);
        s = s + b7 * R(7, ch);
        r[ch] = r[ch] + s;
      }
      if constexpr (DEG >= 3) {
        float b8 = (kShC3_0 * y) * (3.0f * xx - yy);
        float b9 = (kShC3_1 * xy) * z;
        float b10 = (kShC3_2 * y) * ((4.0f * zz - xx) - yy);
        float b11 = (kShC3_3 * z) * ((2.0f * zz - 3.0f * xx) - 3.0f * yy);
        float b12 = (kShC3_4 * x) * ((4.0f * zz - xx) - yy);
        float b13 = (kShC3_5 * z) * (xx - yy);
        float b14 = (kShC3_6 * x) * (xx - 3.0f * yy);
#pragma unroll
        for (int ch = 0; ch < 3; ch++) {
          float u = b8 * R(8, ch);
          u = u + b9 * R(9, ch);
          u = u + b10 * R(10, ch);
          u = u + b11 * R(11, ch);
          u = u + b12 * R(12, ch);
          u = u + b13 * R(13, ch);
          u = u + b14 * R(14, ch);
          r[ch] = r[ch] + u;
        }
      }
    }
#pragma unroll
    for (int ch = 0; ch < 3; ch++) c[ch] = c[ch] + r[ch];
  }
}

}  // namespace sh
}  // namespace splat
