// param_grads.cu -- the backward parameter chain: per-(view, gaussian)
// screen-space gradients back to each gaussian's parameters.
//
// rasterizeSplatsBackward, parameter pass (SplatRaster.cpp:435-575). One
// thread per gaussian loops over the batch's views that render it (every
// view for one cloud; its scene's views for a batch of several scenes),
// keeping the parameter gradients in registers, and adds them into the
// gradient array once. The
// chain is gradient arithmetic, compiled with fused multiply-adds.
#include "common.cuh"
#include "kernels.h"
#include "project_common.cuh"

namespace pxs {
namespace {

constexpr int kParamThreads = 128;

// sum_b w[b] * grad(basis_b)(x, y, z) for the first `count` basis functions
// (shBasisJacobian, SplatRaster.cpp:55-76, contracted with w band by band, so
// the 15 x 3 Jacobian is never held).
__device__ __forceinline__ void sh_gradient_dot(int count, float x, float y, float z,
                                                const float w[15], float d[3]) {
  if (count < 1) return;
  const float C1 = 0.4886025119029199f;
  d[0] += -C1 * w[2];
  d[1] += -C1 * w[0];
  d[2] += C1 * w[1];
  if (count < 8) return;
  const float xx = x * x, yy = y * y, zz = z * z;
  float k = 1.0925484305920792f * w[3];
  d[0] += k * y; d[1] += k * x;
  k = -1.0925484305920792f * w[4];
  d[1] += k * z; d[2] += k * y;
  k = 0.31539156525252005f * w[5];
  d[0] += k * (-2.f * x); d[1] += k * (-2.f * y); d[2] += k * (4.f * z);
  k = -1.0925484305920792f * w[6];
  d[0] += k * z; d[2] += k * x;
  k = 0.5462742152960396f * w[7];
  d[0] += k * (2.f * x); d[1] += k * (-2.f * y);
  if (count < 15) return;
  k = -0.5900435899266435f * w[8];
  d[0] += k * (6.f * x * y); d[1] += k * (3.f * xx - 3.f * yy);
  k = 2.890611442640554f * w[9];
  d[0] += k * (y * z); d[1] += k * (x * z); d[2] += k * (x * y);
  k = -0.4570457994644658f * w[10];
  d[0] += k * (-2.f * x * y); d[1] += k * (4.f * zz - xx - 3.f * yy); d[2] += k * (8.f * y * z);
  k = 0.3731763325901154f * w[11];
  d[0] += k * (-6.f * x * z); d[1] += k * (-6.f * y * z); d[2] += k * (6.f * zz - 3.f * xx - 3.f * yy);
  k = -0.4570457994644658f * w[12];
  d[0] += k * (4.f * zz - 3.f * xx - yy); d[1] += k * (-2.f * x * y); d[2] += k * (8.f * x * z);
  k = 1.445305721320277f * w[13];
  d[0] += k * (2.f * x * z); d[1] += k * (-2.f * y * z); d[2] += k * (xx - yy);
  k = -0.5900435899266435f * w[14];
  d[0] += k * (3.f * xx - 3.f * yy); d[1] += k * (-6.f * x * y);
}

// The rotation matrix of a unit quaternion (Quaternion::toRotationMatrix).
__device__ __forceinline__ void rotation_from_unit(const float q[4], float R[9]) {
  const float w = q[0], x = q[1], y = q[2], z = q[3];
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


// Block-wide exclusive scan of one int per thread of a kParamThreads block;
// the total goes to *total.
__device__ __forceinline__ int block_exclusive_scan_int(int v, int* s_warp, int* total) {
  const int lane = lane_id(), w = warp_id();
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int n = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += n;
  }
  if (lane == 31) s_warp[w] = x;
  __syncthreads();
  int before = 0, all = 0;
#pragma unroll
  for (int k = 0; k < kParamThreads / 32; ++k) {
    const int s = s_warp[k];
    if (k < w) before += s;
    all += s;
  }
  __syncthreads();  // s_warp is reused by the next scan
  *total = all;
  return before + x - v;
}

}  // namespace

// Per-entry results in shared memory (one column per entry): the 14
// gradients of position, log-scale, rotation, opacity and dc, then the `S`
// usable SH basis values (0 past them) and the clamp-masked colour gradient,
// from which the entry's SH-rest gradients basis[b] * dcol[c] follow.
template <int S>
struct EntryLayout {
  static constexpr int kBasis0 = PXS_C_SH_REST;
  static constexpr int kRows = PXS_C_SH_REST + S + 3;
};

// The parameter chain's shared memory (76 KB at SH degree 3).
template <int S>
struct ParamSmem {
  static constexpr int kRest = 3 * S > 0 ? 3 * S : 1;
  float coef[kRest][kParamThreads];  // sh_rest, channel-major
  float grad[kRest][kParamThreads];
  float acc[PXS_C_SH_REST][kParamThreads];
  float state[11][kParamThreads];  // position, unit quaternion, scales, raw norm
  float res[EntryLayout<S>::kRows][kParamThreads];
  uint32_t mask[kParamThreads];
  int off[kParamThreads];
  int warp[kParamThreads / 32];
};

// The chain of one touched (gaussian, view) slot (SplatRaster.cpp:455-575):
// the gaussian's state (position, unit quaternion, its raw norm, scales), its
// SH-rest coefficients `coef` (column of a [3S][kParamThreads] array) and the
// slot's screen accumulators, projection and colour into the column `out`.
template <int S>
__device__ __forceinline__ void entry_chain(const float pos[3], const float qn[4], const float sc[3],
                                            float raw_norm, const float* coef,
                                            const ViewDesc& vd, const ScreenGrad& sg,
                                            const float4 co, const float4 col, float* out) {
  constexpr int kBasis0 = EntryLayout<S>::kBasis0;
  if constexpr (S > 0) {
#pragma unroll
    for (int b = 0; b < S; ++b) out[(kBasis0 + b) * kParamThreads] = 0.f;
  }
  float Rg[9], Mg[9], Sigma[9];
  rotation_from_unit(qn, Rg);
  covariance(Rg, sc, Sigma, Mg);
  const pxs_camera& cam = vd.cam;
  const uint32_t clamped = __float_as_uint(col.w);
  // opacity: alpha = sigmoid(logit) * G
  const float opacity = co.w;
  out[PXS_C_OPACITY * kParamThreads] = sg.dopacity * opacity * (1.f - opacity);
  // colour: through the SH clamp into the coefficients and the direction
  float dcol[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    dcol[c] = sg.dcolor[c];
    if (clamped & (1u << c)) dcol[c] = 0.f;
    out[(PXS_C_DC + c) * kParamThreads] = kShC0 * dcol[c];
    out[(kBasis0 + S + c) * kParamThreads] = dcol[c];
  }
  float ddir[3] = {0.f, 0.f, 0.f};
  const int degree = vd.sh_degree;
  const float off[3] = {pos[0] - cam.center[0], pos[1] - cam.center[1],
                        pos[2] - cam.center[2]};
  const float distance = sqrtf(off[0] * off[0] + (off[1] * off[1] + off[2] * off[2]));
  if constexpr (S > 0) {
    if (degree >= 1 && distance > 1e-9f) {
      const float dir[3] = {off[0] / distance, off[1] / distance, off[2] / distance};
      float basis[15];
      const int basis_count = sh_basis(degree, dir[0], dir[1], dir[2], basis);
      const int usable = basis_count < S ? basis_count : S;
      // w_b = sum_c sh[c][b] dcol[c]; d(colour)/d(direction) . dcol = sum_b w_b grad(basis_b)
      float w[15];
#pragma unroll
      for (int b = 0; b < 15; ++b) w[b] = 0.f;
#pragma unroll
      for (int b = 0; b < S; ++b) {
        if (b < usable) {
          float wb = 0.f;
#pragma unroll
          for (int c = 0; c < 3; ++c) wb += coef[(c * S + b) * kParamThreads] * dcol[c];
          w[b] = wb;
          out[(kBasis0 + b) * kParamThreads] = basis[b];
        }
      }
      sh_gradient_dot(usable, dir[0], dir[1], dir[2], w, ddir);
    }
  }
  // mean: pixels = f * x / z + c
  float p[3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
    p[i] = dot3(cam.R[i * 3 + 0], pos[0], cam.R[i * 3 + 1], pos[1], cam.R[i * 3 + 2],
                pos[2]) +
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
      dT[i * 3 + j] = dot3(D2T[i * 3 + 0], Sigma[0 * 3 + j], D2T[i * 3 + 1], Sigma[1 * 3 + j],
                           D2T[i * 3 + 2], Sigma[2 * 3 + j]);
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
  for (int i = 0; i < 3; ++i) out[(PXS_C_POSITION + i) * kParamThreads] = dpos[i];
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
      dM[i * 3 + j] = dot3(sym2[i * 3 + 0], Mg[0 * 3 + j], sym2[i * 3 + 1], Mg[1 * 3 + j],
                           sym2[i * 3 + 2], Mg[2 * 3 + j]);
#pragma unroll
  for (int a = 0; a < 3; ++a) {  // (R^T dM)(a, a) * s_a
    const float dS = dot3(Rg[0 * 3 + a], dM[0 * 3 + a], Rg[1 * 3 + a], dM[1 * 3 + a],
                          Rg[2 * 3 + a], dM[2 * 3 + a]);
    out[(PXS_C_LOG_SCALE + a) * kParamThreads] = dS * sc[a];
  }
  float dR[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) dR[r * 3 + c] = dM[r * 3 + c] * sc[c];
  const float qw = qn[0], qx = qn[1], qy = qn[2], qz = qn[3];
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
  for (int a = 0; a < 4; ++a) out[(PXS_C_ROTATION + a) * kParamThreads] = (dq[a] - unit[a] * ud) / raw_norm;
}

// Screen-space accumulators back to the gaussian's parameters
// (SplatRaster.cpp:437-575), summed over the views of the batch and ADDED into
// grads. Also visible_count += 1 and screen_gradient += sum |dmean| for every
// projected slot (SplatRaster.cpp:451-453).
//
// Only slots some pixel reached past the alpha cap ("touched") have a
// gradient, and in depth-culled scenes they are a small share of the visible
// slots. So a CTA of kParamThreads gaussians first scans its slots, 32 views
// at a time (visible counts, and a bitmask of the touched views per
// gaussian), compacts the touched (gaussian, view) entries by a block scan,
// runs the chain on them with every lane busy, one entry per thread, and then
// each thread folds its own gaussian's entries into its sums in view order
// (deterministic: no atomics). The SH-rest coefficients and sums live in
// shared memory.
template <int S>
__global__ void __launch_bounds__(kParamThreads, 3)
    k_param_grads(const float* __restrict__ params, int N, int64_t slot_stride,
                  const ViewDesc* __restrict__ views, int n_views, const uint32_t* depth_key,
                  const float4* __restrict__ conic_op, const float4* __restrict__ color,
                  const ScreenGrad* __restrict__ screen, float* __restrict__ grads,
                  float* __restrict__ screen_gradient, int32_t* __restrict__ visible_count) {
  constexpr int T = kParamThreads;
  constexpr int kBasis0 = EntryLayout<S>::kBasis0;
  extern __shared__ __align__(16) unsigned char param_smem[];
  ParamSmem<S>& sm = *reinterpret_cast<ParamSmem<S>*>(param_smem);
  auto& s_coef = sm.coef;
  auto& s_grad = sm.grad;
  auto& s_acc = sm.acc;
  auto& s_state = sm.state;
  auto& s_res = sm.res;
  auto& s_mask = sm.mask;
  auto& s_off = sm.off;
  auto& s_warp = sm.warp;
  const int t = threadIdx.x;
  const int g = blockIdx.x * T + t;
  const bool live = g < N;  // no early return: the block synchronises below
  if (live) {
#pragma unroll
    for (int j = 0; j < PXS_C_SH_REST; ++j) s_acc[j][t] = 0.f;
  }
  int visible = 0;
  float screen_sum = 0.f;
  bool have_state = false;

  for (int vg = 0; vg < n_views; vg += 32) {
    // scan: every slot's accumulators exist (cleared each step), so the key
    // and the accumulators' last four floats are read together
    uint32_t mask = 0u;
    if (live) {
      const int vend = min(n_views, vg + 32);
      // eight views' reads in flight at once, then their bookkeeping in view order
      for (int v0 = vg; v0 < vend; v0 += 8) {
        uint32_t key[8];
        float4 tail[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          key[j] = kCulledKey;
          const int v = v0 + j;
          if (v < vend) {
            const int local = g - views[v].gauss_offset;  // this gaussian's slot in view v
            if (local >= 0 && local < views[v].gauss_count) {
              const int64_t slot = v * slot_stride + local;
              key[j] = depth_key[slot];
              tail[j] = reinterpret_cast<const float4*>(screen + slot)[2];
            }
          }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          if (key[j] == kCulledKey) continue;
          visible += 1;
          screen_sum += tail[j].y;  // dmean_abs
          if (tail[j].z != 0.f) mask |= 1u << (v0 + j - vg);  // touched
        }
      }
      if (mask != 0u && !have_state) {
        // the first touched slot: the gaussian's state, its SH-rest
        // coefficients and cleared SH-rest sums
        if constexpr (S > 0) {
          float coef[3 * S];
#pragma unroll
          for (int j = 0; j < 3 * S; ++j) coef[j] = params[(int64_t)(PXS_C_SH_REST + j) * N + g];
#pragma unroll
          for (int j = 0; j < 3 * S; ++j) {
            s_coef[j][t] = coef[j];
            s_grad[j][t] = 0.f;
          }
        }
        GaussianState st;
        load_state(params, N, g, st);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          s_state[a][t] = st.pos[a];
          s_state[7 + a][t] = st.s[a];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) s_state[3 + a][t] = st.qn[a];
        const float qw0 = params[(int64_t)(PXS_C_ROTATION + 0) * N + g];
        const float qx0 = params[(int64_t)(PXS_C_ROTATION + 1) * N + g];
        const float qy0 = params[(int64_t)(PXS_C_ROTATION + 2) * N + g];
        const float qz0 = params[(int64_t)(PXS_C_ROTATION + 3) * N + g];
        float raw_norm = sqrtf((qx0 * qx0 + qz0 * qz0) + (qy0 * qy0 + qw0 * qw0));
        s_state[10][t] = raw_norm < 1e-12f ? 1e-12f : raw_norm;
        have_state = true;
      }
    }
    const int count = __popc(mask);
    s_mask[t] = mask;
    int total = 0;
    const int off = block_exclusive_scan_int(count, s_warp, &total);
    s_off[t] = off;
    __syncthreads();
    for (int c0 = 0; c0 < total; c0 += T) {
      const int i = c0 + t;
      if (i < total) {
        // the entry's gaussian: the last thread whose first entry is at or
        // before i (an empty thread shares its offset with the next one)
        int lo = 0, hi = T - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s_off[mid] <= i) lo = mid;
          else hi = mid - 1;
        }
        const int owner = lo;
        uint32_t m = s_mask[owner];
        for (int k = i - s_off[owner]; k > 0; --k) m &= m - 1u;  // its k-th touched view
        const int v = vg + __ffs(m) - 1;
        const ViewDesc& vd = views[v];
        const int go = blockIdx.x * T + owner;
        const int64_t slot = v * slot_stride + (go - vd.gauss_offset);
        const ScreenGrad sg = screen[slot];
        const float4 co = conic_op[slot];
        const float4 col = color[slot];
        const float pos[3] = {s_state[0][owner], s_state[1][owner], s_state[2][owner]};
        const float qn[4] = {s_state[3][owner], s_state[4][owner], s_state[5][owner],
                             s_state[6][owner]};
        const float sc[3] = {s_state[7][owner], s_state[8][owner], s_state[9][owner]};
        entry_chain<S>(pos, qn, sc, s_state[10][owner], &s_coef[0][owner], vd, sg, co, col,
                       &s_res[0][t]);
      }
      __syncthreads();
      // each gaussian adds its entries of this chunk, in view order
      const int e0 = max(off, c0), e1 = min(off + count, c0 + T);
      for (int e = e0; e < e1; ++e) {
        const int col = e - c0;
#pragma unroll
        for (int j = 0; j < PXS_C_SH_REST; ++j) s_acc[j][t] += s_res[j][col];
        if constexpr (S > 0) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float dcol = s_res[kBasis0 + S + c][col];
#pragma unroll
            for (int b = 0; b < S; ++b) s_grad[c * S + b][t] += s_res[kBasis0 + b][col] * dcol;
          }
        }
      }
      __syncthreads();
    }
  }
  if (!live) return;
  if (visible) {
    visible_count[g] += visible;
    screen_gradient[g] += screen_sum;
  }
  if (have_state) {
    // read-modify-write in groups whose reads are all issued before the writes
    float old[PXS_C_SH_REST];
#pragma unroll
    for (int c = 0; c < PXS_C_SH_REST; ++c) old[c] = grads[(int64_t)c * N + g];
#pragma unroll
    for (int c = 0; c < PXS_C_SH_REST; ++c) grads[(int64_t)c * N + g] = old[c] + s_acc[c][t];
    if constexpr (S > 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float rest[S];
#pragma unroll
        for (int b = 0; b < S; ++b) rest[b] = grads[(int64_t)(PXS_C_SH_REST + c * S + b) * N + g];
#pragma unroll
        for (int b = 0; b < S; ++b)
          grads[(int64_t)(PXS_C_SH_REST + c * S + b) * N + g] = rest[b] + s_grad[c * S + b][t];
      }
    }
  }
}

void configure_param_grads_kernel() {
  cudaFuncSetAttribute(k_param_grads<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(ParamSmem<0>));
  cudaFuncSetAttribute(k_param_grads<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(ParamSmem<3>));
  cudaFuncSetAttribute(k_param_grads<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(ParamSmem<8>));
  cudaFuncSetAttribute(k_param_grads<15>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(ParamSmem<15>));
}

void launch_param_grads(const float* params, int N, int S, int64_t slot_stride,
                        const ViewDesc* views, int n_views, const uint32_t* depth_key,
                        const float4* conic_op, const float4* color, const ScreenGrad* screen,
                        float* grads, float* screen_gradient, int32_t* visible_count,
                        cudaStream_t stream) {
  const int threads = kParamThreads;
  const int blocks = (N + threads - 1) / threads;
  if (blocks == 0) return;
#define LAUNCH(SS)                                                                      \
  count_launch();                                                                       \
  k_param_grads<SS><<<blocks, threads, sizeof(ParamSmem<SS>), stream>>>(                \
      params, N, slot_stride, views, n_views, depth_key, conic_op, color, screen, grads, \
      screen_gradient, visible_count)
  switch (S) {
    case 0: LAUNCH(0); break;
    case 3: LAUNCH(3); break;
    case 8: LAUNCH(8); break;
    default: LAUNCH(15); break;
  }
#undef LAUNCH
}


}  // namespace pxs
