// Scene::finalize's activation steps on the device, shared by the FP16
// projection (project.cu) and the device-side scene decoders (decode.cu).
// Operation order is glam's (SSE2 Quat::length, Mat3 products), so with
// --fmad=false every result equals the reference's f32 value.
#pragma once

namespace splat {

// Quaternion normalisation (src/scene.rs:164-171): q / |q| when |q| is finite
// and > 1e-12, else the identity; glam's SSE2 Quat::length sums
// (x^2 + z^2) + (y^2 + w^2).
template <class T>
__device__ __forceinline__ void normalize_quat(T& qx, T& qy, T& qz, T& qw) {
  const T len = sqrt((qx * qx + qz * qz) + (qy * qy + qw * qw));
  if (isfinite(len) && len > T(1e-12)) {
    qx = qx / len;
    qy = qy / len;
    qz = qz / len;
    qw = qw / len;
  } else {
    qx = qy = qz = T(0);
    qw = T(1);
  }
}

// covariance (src/scene.rs:261-270): R S S^T R^T in glam's Mat3 operation
// order, from a unit quaternion; upper triangle xx, xy, xz, yy, yz, zz.
template <class T>
__device__ __forceinline__ void covariance_rs(const T s[3], T qx, T qy, T qz, T qw, T c[6]) {
  const T x2 = qx + qx, y2 = qy + qy, z2 = qz + qz;
  const T xx = qx * x2, xy = qx * y2, xz = qx * z2, yy = qy * y2, yz = qy * z2, zz = qz * z2;
  const T wx = qw * x2, wy = qw * y2, wz = qw * z2;
  const T r[3][3] = {{T(1) - (yy + zz), xy + wz, xz - wy},   // column 0
                     {xy - wz, T(1) - (xx + zz), yz + wx},   // column 1
                     {xz + wy, yz - wx, T(1) - (xx + yy)}};  // column 2
  T m[3][3];  // columns of R * diag(s): c0*v.x + c1*v.y + c2*v.z with v = (s0,0,0), ...
  for (int j = 0; j < 3; j++)
    for (int k = 0; k < 3; k++) {
      const T v0 = j == 0 ? s[0] : T(0), v1 = j == 1 ? s[1] : T(0), v2 = j == 2 ? s[2] : T(0);
      m[j][k] = (r[0][k] * v0 + r[1][k] * v1) + r[2][k] * v2;
    }
  T o[3][3];  // columns of m * m^T; column j of m^T is row j of m
  for (int j = 0; j < 3; j++)
    for (int k = 0; k < 3; k++) o[j][k] = (m[0][k] * m[0][j] + m[1][k] * m[1][j]) + m[2][k] * m[2][j];
  c[0] = o[0][0];
  c[1] = o[1][0];
  c[2] = o[2][0];
  c[3] = o[1][1];
  c[4] = o[2][1];
  c[5] = o[2][2];
}

// Scene::finalize + covariance of one splat: the quaternion normalised, then
// R S S^T R^T.
template <class T>
__device__ __forceinline__ void covariance_from(const T s[3], T qx, T qy, T qz, T qw, T c[6]) {
  normalize_quat(qx, qy, qz, qw);
  covariance_rs(s, qx, qy, qz, qw, c);
}

}  // namespace splat
