// project_common.cuh -- per-gaussian helpers shared by the projection kernel
// and the backward parameter chain: rotation, 3D covariance, the projection
// Jacobian and the SH basis. Which rounding they get depends on the including
// file: project.cu compiles them without contraction (the projection must
// round like the reference); param_grads.cu lets them fuse (gradients).
#pragma once

#include "common.cuh"

namespace pxs {
namespace {

__device__ __forceinline__ float dot3(float a0, float b0, float a1, float b1, float a2, float b2) {
  return a0 * b0 + (a1 * b1 + a2 * b2);
}

// Correctly rounded single-precision exp.
__device__ __forceinline__ float exp_cr(float x) { return __double2float_rn(exp((double)x)); }

// x86 cvttss2si semantics (what (int)floor(v) gives the reference): values
// outside the int range, and NaN, become INT_MIN.
__device__ __forceinline__ int float_to_int_x86(float v) {
  if (!(v > -2147483904.0f && v < 2147483648.0f)) return INT32_MIN;
  return (int)v;
}

// Quaternion::normalized then toRotationMatrix; R row-major (SplatRaster.cpp:78-80).
__device__ __forceinline__ void rotation_of(float w, float x, float y, float z, float R[9],
                                            float qn[4]) {
  const float sq = (x * x + z * z) + (y * y + w * w);
  if (sq > 0.f) {
    const float norm = sqrtf(sq);
    w = w / norm;
    x = x / norm;
    y = y / norm;
    z = z / norm;
  }
  qn[0] = w;
  qn[1] = x;
  qn[2] = y;
  qn[3] = z;
  const float tx = 2.f * x, ty = 2.f * y, tz = 2.f * z;
  const float twx = tx * w, twy = ty * w, twz = tz * w;
  const float txx = tx * x, txy = ty * x, txz = tz * x;
  const float tyy = ty * y, tyz = tz * y, tzz = tz * z;
  R[0] = 1.f - (tyy + tzz);
  R[1] = txy - twz;
  R[2] = txz + twy;
  R[3] = txy + twz;
  R[4] = 1.f - (txx + tzz);
  R[5] = tyz - twx;
  R[6] = txz - twy;
  R[7] = tyz + twx;
  R[8] = 1.f - (txx + tyy);
}

// covariance3d (SplatRaster.cpp:82-87): M = R diag(s); Sigma = M M^T.
__device__ __forceinline__ void covariance(const float R[9], const float s[3], float Sigma[9],
                                           float M[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) M[i * 3 + j] = R[i * 3 + j] * s[j];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      Sigma[i * 3 + j] = dot3(M[i * 3 + 0], M[j * 3 + 0], M[i * 3 + 1], M[j * 3 + 1],
                              M[i * 3 + 2], M[j * 3 + 2]);
}

// projectionJacobian (SplatRaster.cpp:91-102) times W: T = J W (2x3).
__device__ __forceinline__ void jacobian_times_w(const float p[3], const pxs_camera& cam,
                                                 float J[6], float T[6]) {
  const float z = p[2];
  const float limit_x = cam.tan_half_x * kFrustumSlack;
  const float limit_y = cam.tan_half_y * kFrustumSlack;
  float ux = p[0] / z, uy = p[1] / z;
  ux = ux < -limit_x ? -limit_x : (limit_x < ux ? limit_x : ux);
  uy = uy < -limit_y ? -limit_y : (limit_y < uy ? limit_y : uy);
  const float x = ux * z, y = uy * z;
  J[0] = cam.fx / z;
  J[1] = 0.f;
  J[2] = -cam.fx * x / (z * z);
  J[3] = 0.f;
  J[4] = cam.fy / z;
  J[5] = -cam.fy * y / (z * z);
  const float* W = cam.R;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      T[i * 3 + j] = dot3(J[i * 3 + 0], W[0 * 3 + j], J[i * 3 + 1], W[1 * 3 + j], J[i * 3 + 2],
                          W[2 * 3 + j]);
}

// shBasis (SplatRaster.cpp:29-52).
__device__ __forceinline__ int sh_basis(int degree, float x, float y, float z, float* basis) {
  if (degree < 1) return 0;
  const float C1 = 0.4886025119029199f;
  basis[0] = -C1 * y;
  basis[1] = C1 * z;
  basis[2] = -C1 * x;
  if (degree < 2) return 3;
  const float xx = x * x, yy = y * y, zz = z * z;
  const float xy = x * y, yz = y * z, xz = x * z;
  basis[3] = 1.0925484305920792f * xy;
  basis[4] = -1.0925484305920792f * yz;
  basis[5] = 0.31539156525252005f * (2.f * zz - xx - yy);
  basis[6] = -1.0925484305920792f * xz;
  basis[7] = 0.5462742152960396f * (xx - yy);
  if (degree < 3) return 8;
  basis[8] = -0.5900435899266435f * y * (3.f * xx - yy);
  basis[9] = 2.890611442640554f * xy * z;
  basis[10] = -0.4570457994644658f * y * (4.f * zz - xx - yy);
  basis[11] = 0.3731763325901154f * z * (2.f * zz - 3.f * xx - 3.f * yy);
  basis[12] = -0.4570457994644658f * x * (4.f * zz - xx - yy);
  basis[13] = 1.445305721320277f * z * (xx - yy);
  basis[14] = -0.5900435899266435f * x * (xx - 3.f * yy);
  return 15;
}

// shBasisJacobian (SplatRaster.cpp:55-76): jac[b][axis].
__device__ __forceinline__ void sh_basis_jacobian(int count, float x, float y, float z,
                                                  float jac[15][3]) {
  if (count < 1) return;
  const float C1 = 0.4886025119029199f;
  jac[0][0] = 0.f; jac[0][1] = -C1; jac[0][2] = 0.f;
  jac[1][0] = 0.f; jac[1][1] = 0.f; jac[1][2] = C1;
  jac[2][0] = -C1; jac[2][1] = 0.f; jac[2][2] = 0.f;
  if (count < 8) return;
  const float xx = x * x, yy = y * y, zz = z * z;
#define SETJ(b, cc, a0, a1, a2) \
  jac[b][0] = (cc) * (a0);      \
  jac[b][1] = (cc) * (a1);      \
  jac[b][2] = (cc) * (a2)
  SETJ(3, 1.0925484305920792f, y, x, 0.f);
  SETJ(4, -1.0925484305920792f, 0.f, z, y);
  SETJ(5, 0.31539156525252005f, -2.f * x, -2.f * y, 4.f * z);
  SETJ(6, -1.0925484305920792f, z, 0.f, x);
  SETJ(7, 0.5462742152960396f, 2.f * x, -2.f * y, 0.f);
  if (count < 15) return;
  SETJ(8, -0.5900435899266435f, 6.f * x * y, 3.f * xx - 3.f * yy, 0.f);
  SETJ(9, 2.890611442640554f, y * z, x * z, x * y);
  SETJ(10, -0.4570457994644658f, -2.f * x * y, 4.f * zz - xx - 3.f * yy, 8.f * y * z);
  SETJ(11, 0.3731763325901154f, -6.f * x * z, -6.f * y * z, 6.f * zz - 3.f * xx - 3.f * yy);
  SETJ(12, -0.4570457994644658f, 4.f * zz - 3.f * xx - yy, -2.f * x * y, 8.f * x * z);
  SETJ(13, 1.445305721320277f, 2.f * x * z, -2.f * y * z, xx - yy);
  SETJ(14, -0.5900435899266435f, 3.f * xx - 3.f * yy, -6.f * x * y, 0.f);
#undef SETJ
}

// Shared per-gaussian state, view independent.
struct GaussianState {
  float pos[3];
  float R[9];
  float qn[4];
  float s[3];
  float Sigma[9];
  float M[9];
  float opacity;
};

__device__ __forceinline__ void load_state(const float* __restrict__ params, int64_t N, int g,
                                           GaussianState& st) {
#pragma unroll
  for (int a = 0; a < 3; ++a) st.pos[a] = params[(int64_t)(PXS_C_POSITION + a) * N + g];
  const float w = params[(int64_t)(PXS_C_ROTATION + 0) * N + g];
  const float x = params[(int64_t)(PXS_C_ROTATION + 1) * N + g];
  const float y = params[(int64_t)(PXS_C_ROTATION + 2) * N + g];
  const float z = params[(int64_t)(PXS_C_ROTATION + 3) * N + g];
  rotation_of(w, x, y, z, st.R, st.qn);
#pragma unroll
  for (int a = 0; a < 3; ++a) st.s[a] = exp_cr(params[(int64_t)(PXS_C_LOG_SCALE + a) * N + g]);
  covariance(st.R, st.s, st.Sigma, st.M);
  // gaussianOpacity (GaussianCloud.h:81-83)
  st.opacity = 1.0f / (1.0f + exp_cr(-params[(int64_t)PXS_C_OPACITY * N + g]));
}

}  // namespace
}  // namespace pxs
