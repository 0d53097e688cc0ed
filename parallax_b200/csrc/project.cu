// project.cu -- EWA projection with SH colour, and the backward parameter chain.
//
// Compiled with -fmad=false: every product and sum rounds separately, in the
// order the reference's own compiled code evaluates it (scalar C++ left to
// right; Eigen's fixed-size products per coefficient as x0 + (x1 + x2); float
// 4-vector reductions as (x0 + x2) + (x1 + x3)). With IEEE division and square
// root this reproduces the reference's projection bit for bit except where
// glibc's expf is not correctly rounded: exp here is the correctly rounded
// value (computed in double and rounded once).
#include "common.cuh"
#include "kernels.h"

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

// One thread per gaussian, looping over the views of the batch so the
// parameters are read once (projectSplats, SplatRaster.cpp:201-258).
__global__ void __launch_bounds__(256)
    k_project(const float* __restrict__ params, int N, int S, int64_t slot_stride,
              const ViewDesc* __restrict__ views, int n_views, ProjectedSoA out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= slot_stride) return;
  if (g >= N) {
    for (int v = 0; v < n_views; ++v) {
      const int64_t slot = v * slot_stride + g;
      out.depth_key[slot] = kCulledKey;
      out.tile_count[slot] = 0;
    }
    return;
  }
  GaussianState st;
  load_state(params, N, g, st);
  const float dc0 = params[(int64_t)(PXS_C_DC + 0) * N + g];
  const float dc1 = params[(int64_t)(PXS_C_DC + 1) * N + g];
  const float dc2 = params[(int64_t)(PXS_C_DC + 2) * N + g];

  for (int v = 0; v < n_views; ++v) {
    const int64_t slot = v * slot_stride + g;
    const ViewDesc& vd = views[v];
    const pxs_camera& cam = vd.cam;
    float p[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
      p[i] = dot3(cam.R[i * 3 + 0], st.pos[0], cam.R[i * 3 + 1], st.pos[1], cam.R[i * 3 + 2],
                  st.pos[2]) +
             cam.t[i];
    bool visible = !(p[2] < 0.01f);
    float cov[4], det = 0.f;
    if (visible) {
      float J[6], T[6], TS[6];
      jacobian_times_w(p, cam, J, T);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          TS[i * 3 + j] = dot3(T[i * 3 + 0], st.Sigma[0 * 3 + j], T[i * 3 + 1],
                               st.Sigma[1 * 3 + j], T[i * 3 + 2], st.Sigma[2 * 3 + j]);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
          cov[i * 2 + j] = dot3(TS[i * 3 + 0], T[j * 3 + 0], TS[i * 3 + 1], T[j * 3 + 1],
                                TS[i * 3 + 2], T[j * 3 + 2]);
      cov[0] += vd.screen_dilation;
      cov[3] += vd.screen_dilation;
      det = cov[0] * cov[3] - cov[1] * cov[2];
      visible = !(det <= 1e-12f);
    }
    float mean_x = 0.f, mean_y = 0.f, radius = 0.f;
    if (visible) {
      mean_x = cam.fx * p[0] / p[2] + cam.cx;
      mean_y = cam.fy * p[1] / p[2] + cam.cy;
      const float mid = 0.5f * (cov[0] + cov[3]);
      const float under = mid * mid - det;
      const float spread = sqrtf(0.f < under ? under : 0.f);
      const float major = mid + spread;
      radius = 3.f * sqrtf(major < 1e-6f ? 1e-6f : major);
      if (mean_x + radius < 0.f || mean_x - radius >= (float)cam.width ||
          mean_y + radius < 0.f || mean_y - radius >= (float)cam.height)
        visible = false;
      else if (st.opacity < vd.min_alpha)
        visible = false;
    }
    if (!visible) {
      out.depth_key[slot] = kCulledKey;
      out.tile_count[slot] = 0;
      continue;
    }
    // evaluateSh (SplatRaster.cpp:179-199) along the unit camera->gaussian direction
    float off[3] = {st.pos[0] - cam.center[0], st.pos[1] - cam.center[1],
                    st.pos[2] - cam.center[2]};
    const float sq = off[0] * off[0] + (off[1] * off[1] + off[2] * off[2]);
    float d[3] = {off[0], off[1], off[2]};
    if (sq > 0.f) {
      const float norm = sqrtf(sq);
      d[0] = off[0] / norm;
      d[1] = off[1] / norm;
      d[2] = off[2] / norm;
    }
    float color[3] = {0.5f + kShC0 * dc0, 0.5f + kShC0 * dc1, 0.5f + kShC0 * dc2};
    float basis[15];
    const int count = sh_basis(vd.sh_degree, d[0], d[1], d[2], basis);
    const int usable = count < S ? count : S;
    for (int c = 0; c < 3; ++c) {
      float sum = 0.f;
      for (int k = 0; k < usable; ++k)
        sum += basis[k] * params[(int64_t)(PXS_C_SH_REST + c * S + k) * N + g];
      color[c] += sum;
    }
    uint32_t flags = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (color[c] < 0.f) {
        flags |= 1u << c;
        color[c] = 0.f;
      }
    }
    const float conic_a = cov[3] / det, conic_b = -cov[1] / det, conic_c = cov[0] / det;
    out.xy[slot] = make_float2(mean_x, mean_y);
    out.conic_op[slot] = make_float4(conic_a, conic_b, conic_c, st.opacity);
    out.color[slot] = make_float4(color[0], color[1], color[2], __uint_as_float(flags));
    out.depth_key[slot] = __float_as_uint(p[2]);
    if (out.debug_cov != nullptr)
      out.debug_cov[slot] = make_float4(cov[0], cov[1], cov[3], radius);
    // tileRange (SplatRaster.cpp:121-126)
    const int x0 = max(0, float_to_int_x86(floorf((mean_x - radius) / 16.f)));
    const int x1 = min(vd.tiles_x - 1, float_to_int_x86(floorf((mean_x + radius) / 16.f)));
    const int y0 = max(0, float_to_int_x86(floorf((mean_y - radius) / 16.f)));
    const int y1 = min(vd.tiles_y - 1, float_to_int_x86(floorf((mean_y + radius) / 16.f)));
    const int tiles = (x1 >= x0 && y1 >= y0) ? (x1 - x0 + 1) * (y1 - y0 + 1) : 0;
    out.rect[slot] = make_uint2((uint32_t)(x0 & 0xFFFF) | ((uint32_t)(x1 & 0xFFFF) << 16),
                                (uint32_t)(y0 & 0xFFFF) | ((uint32_t)(y1 & 0xFFFF) << 16));
    out.tile_count[slot] = tiles;
  }
}

// Screen-space accumulators back to the gaussian's parameters
// (SplatRaster.cpp:437-575), summed over the views of the batch and ADDED into
// grads. Also visible_count += 1 and screen_gradient += sum |dmean| for every
// projected slot (SplatRaster.cpp:451-453).
template <int S>
__global__ void __launch_bounds__(128)
    k_param_grads(const float* __restrict__ params, int N, int64_t slot_stride,
                  const ViewDesc* __restrict__ views, int n_views, const uint32_t* depth_key,
                  const float4* __restrict__ conic_op, const float4* __restrict__ color,
                  const ScreenGrad* __restrict__ screen, float* __restrict__ grads,
                  float* __restrict__ screen_gradient, int32_t* __restrict__ visible_count) {
  constexpr int P = 14 + 3 * S;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N) return;
  int visible = 0;
  float screen_sum = 0.f;
  bool any = false;
  float acc[P];
#pragma unroll
  for (int c = 0; c < P; ++c) acc[c] = 0.f;
  bool have_state = false;
  GaussianState st;

  for (int v = 0; v < n_views; ++v) {
    const int64_t slot = v * slot_stride + g;
    if (depth_key[slot] == kCulledKey) continue;
    const ScreenGrad sg = screen[slot];
    visible += 1;
    screen_sum += sg.dmean_abs;
    if (sg.touched == 0.f) continue;
    if (!have_state) {
      load_state(params, N, g, st);
      have_state = true;
    }
    any = true;
    const ViewDesc& vd = views[v];
    const pxs_camera& cam = vd.cam;
    const float4 co = conic_op[slot];
    const float4 col = color[slot];
    const uint32_t clamped = __float_as_uint(col.w);
    // opacity: alpha = sigmoid(logit) * G
    const float opacity = co.w;
    acc[PXS_C_OPACITY] += sg.dopacity * opacity * (1.f - opacity);
    // colour: through the SH clamp into the coefficients and the direction
    float dcol[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      dcol[c] = sg.dcolor[c];
      if (clamped & (1u << c)) dcol[c] = 0.f;
      acc[PXS_C_DC + c] += kShC0 * dcol[c];
    }
    float ddir[3] = {0.f, 0.f, 0.f};
    const int degree = vd.sh_degree;
    const float off[3] = {st.pos[0] - cam.center[0], st.pos[1] - cam.center[1],
                          st.pos[2] - cam.center[2]};
    const float distance = sqrtf(off[0] * off[0] + (off[1] * off[1] + off[2] * off[2]));
    if constexpr (S > 0) {
      if (degree >= 1 && distance > 1e-9f) {
        const float dir[3] = {off[0] / distance, off[1] / distance, off[2] / distance};
        float basis[15];
        float jac[15][3];
        const int basis_count = sh_basis(degree, dir[0], dir[1], dir[2], basis);
        const int usable = basis_count < S ? basis_count : S;
        sh_basis_jacobian(basis_count, dir[0], dir[1], dir[2], jac);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (dcol[c] == 0.f) continue;
#pragma unroll
          for (int b = 0; b < S; ++b) {
            if (b < usable) {
              acc[PXS_C_SH_REST + c * S + b] += basis[b] * dcol[c];
              const float k = params[(int64_t)(PXS_C_SH_REST + c * S + b) * N + g] * dcol[c];
              ddir[0] += jac[b][0] * k;
              ddir[1] += jac[b][1] * k;
              ddir[2] += jac[b][2] * k;
            }
          }
        }
      }
    }
    // mean: pixels = f * x / z + c
    float p[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
      p[i] = dot3(cam.R[i * 3 + 0], st.pos[0], cam.R[i * 3 + 1], st.pos[1], cam.R[i * 3 + 2],
                  st.pos[2]) +
             cam.t[i];
    const float z = p[2];
    const float fx = cam.fx, fy = cam.fy;
    const float dmx = sg.dmean[0], dmy = sg.dmean[1];
    float dp[3] = {fx / z * dmx, fy / z * dmy, -(fx * p[0] * dmx + fy * p[1] * dmy) / (z * z)};
    // conic -> 2D covariance: -(A D A), D the symmetric gradient
    const float A[4] = {co.x, co.y, co.y, co.z};
    const float Dm[4] = {sg.dconic[0], 0.5f * sg.dconic[1], 0.5f * sg.dconic[1], sg.dconic[2]};
    float AD[4], dcov2[4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) AD[i * 2 + j] = A[i * 2 + 0] * Dm[0 * 2 + j] + A[i * 2 + 1] * Dm[1 * 2 + j];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
        dcov2[i * 2 + j] = -(AD[i * 2 + 0] * A[0 * 2 + j] + AD[i * 2 + 1] * A[1 * 2 + j]);
    // 2D covariance -> 3D covariance and the projection Jacobian
    float J[6], T[6];
    jacobian_times_w(p, cam, J, T);
    float TtD[6], dcov3[9];  // T^T dcov2 (3x2), then (3x3)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) TtD[i * 2 + j] = T[0 * 3 + i] * dcov2[0 * 2 + j] + T[1 * 3 + i] * dcov2[1 * 2 + j];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) dcov3[i * 3 + j] = TtD[i * 2 + 0] * T[0 * 3 + j] + TtD[i * 2 + 1] * T[1 * 3 + j];
    float D2T[6], dT[6], dJ[6];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        D2T[i * 3 + j] = (2.f * dcov2[i * 2 + 0]) * T[0 * 3 + j] + (2.f * dcov2[i * 2 + 1]) * T[1 * 3 + j];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        dT[i * 3 + j] = dot3(D2T[i * 3 + 0], st.Sigma[0 * 3 + j], D2T[i * 3 + 1], st.Sigma[1 * 3 + j],
                             D2T[i * 3 + 2], st.Sigma[2 * 3 + j]);
    const float* W = cam.R;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)  // dJ = dT W^T
        dJ[i * 3 + j] = dot3(dT[i * 3 + 0], W[j * 3 + 0], dT[i * 3 + 1], W[j * 3 + 1],
                             dT[i * 3 + 2], W[j * 3 + 2]);
    const float lim_x = cam.tan_half_x * kFrustumSlack, lim_y = cam.tan_half_y * kFrustumSlack;
    const bool clamped_x = fabsf(p[0] / z) > lim_x;
    const bool clamped_y = fabsf(p[1] / z) > lim_y;
    const float jx = clamped_x ? copysignf(lim_x, p[0]) * z : p[0];
    const float jy = clamped_y ? copysignf(lim_y, p[1]) * z : p[1];
    if (!clamped_x) dp[0] += dJ[2] * (-fx / (z * z));
    if (!clamped_y) dp[1] += dJ[5] * (-fy / (z * z));
    const float dz_x = (clamped_x ? 1.f : 2.f) * fx * jx / (z * z * z);
    const float dz_y = (clamped_y ? 1.f : 2.f) * fy * jy / (z * z * z);
    dp[2] += dJ[0] * (-fx / (z * z)) + dJ[4] * (-fy / (z * z)) + dJ[2] * dz_x + dJ[5] * dz_y;
    float dpos[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)  // W^T dp
      dpos[i] = dot3(W[0 * 3 + i], dp[0], W[1 * 3 + i], dp[1], W[2 * 3 + i], dp[2]);
    const float ddir_sq = ddir[0] * ddir[0] + (ddir[1] * ddir[1] + ddir[2] * ddir[2]);
    if (distance > 1e-9f && ddir_sq > 0.f) {
      const float dir[3] = {off[0] / distance, off[1] / distance, off[2] / distance};
      const float dd = dot3(dir[0], ddir[0], dir[1], ddir[1], dir[2], ddir[2]);
#pragma unroll
      for (int i = 0; i < 3; ++i) dpos[i] += (ddir[i] - dir[i] * dd) / distance;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[PXS_C_POSITION + i] += dpos[i];
    // Sigma = (R S)(R S)^T -> scale and rotation
    float sym2[9], dM[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) sym2[i * 3 + j] = 2.f * (0.5f * (dcov3[i * 3 + j] + dcov3[j * 3 + i]));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        dM[i * 3 + j] = dot3(sym2[i * 3 + 0], st.M[0 * 3 + j], sym2[i * 3 + 1], st.M[1 * 3 + j],
                             sym2[i * 3 + 2], st.M[2 * 3 + j]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {  // (R^T dM)(a, a) * s_a
      const float dS = dot3(st.R[0 * 3 + a], dM[0 * 3 + a], st.R[1 * 3 + a], dM[1 * 3 + a],
                            st.R[2 * 3 + a], dM[2 * 3 + a]);
      acc[PXS_C_LOG_SCALE + a] += dS * st.s[a];
    }
    float dR[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) dR[r * 3 + c] = dM[r * 3 + c] * st.s[c];
    const float qw0 = params[(int64_t)(PXS_C_ROTATION + 0) * N + g];
    const float qx0 = params[(int64_t)(PXS_C_ROTATION + 1) * N + g];
    const float qy0 = params[(int64_t)(PXS_C_ROTATION + 2) * N + g];
    const float qz0 = params[(int64_t)(PXS_C_ROTATION + 3) * N + g];
    float raw_norm = sqrtf((qx0 * qx0 + qz0 * qz0) + (qy0 * qy0 + qw0 * qw0));
    raw_norm = raw_norm < 1e-12f ? 1e-12f : raw_norm;
    const float qw = st.qn[0], qx = st.qn[1], qy = st.qn[2], qz = st.qn[3];
#define DR(r, c) dR[(r)*3 + (c)]
    float dq[4];
    dq[0] = 0.f + 2.f * (-qz * DR(0, 1) + qy * DR(0, 2) + qz * DR(1, 0) - qx * DR(1, 2) -
                         qy * DR(2, 0) + qx * DR(2, 1));
    dq[1] = 0.f + 2.f * (qy * DR(0, 1) + qz * DR(0, 2) + qy * DR(1, 0) - 2.f * qx * DR(1, 1) -
                         qw * DR(1, 2) + qz * DR(2, 0) + qw * DR(2, 1) - 2.f * qx * DR(2, 2));
    dq[2] = 0.f + 2.f * (-2.f * qy * DR(0, 0) + qx * DR(0, 1) + qw * DR(0, 2) + qx * DR(1, 0) +
                         qz * DR(1, 2) - qw * DR(2, 0) + qz * DR(2, 1) - 2.f * qy * DR(2, 2));
    dq[3] = 0.f + 2.f * (-2.f * qz * DR(0, 0) - qw * DR(0, 1) + qx * DR(0, 2) + qw * DR(1, 0) -
                         2.f * qz * DR(1, 1) + qy * DR(1, 2) + qx * DR(2, 0) + qy * DR(2, 1));
#undef DR
    const float unit[4] = {qw, qx, qy, qz};
    const float ud = (unit[0] * dq[0] + unit[2] * dq[2]) + (unit[1] * dq[1] + unit[3] * dq[3]);
#pragma unroll
    for (int a = 0; a < 4; ++a) acc[PXS_C_ROTATION + a] += (dq[a] - unit[a] * ud) / raw_norm;
  }
  if (visible) {
    visible_count[g] += visible;
    screen_gradient[g] += screen_sum;
  }
  if (any) {
#pragma unroll
    for (int c = 0; c < P; ++c) grads[(int64_t)c * N + g] += acc[c];
  }
}

void launch_project(const float* params, int N, int S, int64_t slot_stride,
                    const ViewDesc* views, int n_views, const ProjectedSoA& out,
                    cudaStream_t stream) {
  const int threads = 256;
  const int blocks = (int)((slot_stride + threads - 1) / threads);
  if (blocks > 0) {
    count_launch();
    k_project<<<blocks, threads, 0, stream>>>(params, N, S, slot_stride, views, n_views, out);
  }
}

void launch_param_grads(const float* params, int N, int S, int64_t slot_stride,
                        const ViewDesc* views, int n_views, const uint32_t* depth_key,
                        const float4* conic_op, const float4* color, const ScreenGrad* screen,
                        float* grads, float* screen_gradient, int32_t* visible_count,
                        cudaStream_t stream) {
  const int threads = 128;
  const int blocks = (N + threads - 1) / threads;
  if (blocks == 0) return;
#define LAUNCH(SS)                                                                          \
  count_launch();                                                                   \
  k_param_grads<SS><<<blocks, threads, 0, stream>>>(params, N, slot_stride, views, n_views, \
                                                    depth_key, conic_op, color, screen,     \
                                                    grads, screen_gradient, visible_count)
  switch (S) {
    case 0: LAUNCH(0); break;
    case 3: LAUNCH(3); break;
    case 8: LAUNCH(8); break;
    default: LAUNCH(15); break;
  }
#undef LAUNCH
}

}  // namespace pxs
