// project.cu -- EWA projection with SH colour.
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
#include "project_common.cuh"

namespace pxs {


constexpr int kProjectThreads = 256;

// One thread per slot index i, looping over the views of the batch: view v's
// slot i holds gaussian gauss_offset + i of that view's range. Views of one
// cloud share the gaussian, so its parameters are read once; a batch of
// several scenes reads each scene's gaussian when the scene changes
// (projectSplats, SplatRaster.cpp:201-258). The gaussian's S SH-rest
// coefficients per channel are read together into this thread's column of
// shared memory and serve every view.
template <int S>
__global__ void __launch_bounds__(kProjectThreads, 3)
    k_project(const float* __restrict__ params, int N, int64_t slot_stride,
              const ViewDesc* __restrict__ views, int n_views, ProjectedSoA out) {
  constexpr int kRest = 3 * S > 0 ? 3 * S : 1;
  __shared__ float s_sh[kRest][kProjectThreads];
  const int t = threadIdx.x;
  const int i = blockIdx.x * blockDim.x + t;
  if (i >= slot_stride) return;
  GaussianState st;
  int g = -1;  // the gaussian whose state is loaded
  float dc0 = 0.f, dc1 = 0.f, dc2 = 0.f;

  for (int v = 0; v < n_views; ++v) {
    const int64_t slot = v * slot_stride + i;
    const ViewDesc& vd = views[v];
    if (i >= vd.gauss_count) {
      out.depth_key[slot] = kCulledKey;
      out.tile_count[slot] = 0;
      continue;
    }
    if (vd.gauss_offset + i != g) {
      g = vd.gauss_offset + i;
      if constexpr (S > 0) {
        float sh[3 * S];
#pragma unroll
        for (int j = 0; j < 3 * S; ++j) sh[j] = params[(int64_t)(PXS_C_SH_REST + j) * N + g];
#pragma unroll
        for (int j = 0; j < 3 * S; ++j) s_sh[j][t] = sh[j];
      }
      load_state(params, N, g, st);
      dc0 = params[(int64_t)(PXS_C_DC + 0) * N + g];
      dc1 = params[(int64_t)(PXS_C_DC + 1) * N + g];
      dc2 = params[(int64_t)(PXS_C_DC + 2) * N + g];
    }
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
#pragma unroll
      for (int k = 0; k < S; ++k)
        if (k < usable) sum += basis[k] * s_sh[c * S + k][t];
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

void launch_project(const float* params, int N, int S, int64_t slot_stride,
                    const ViewDesc* views, int n_views, const ProjectedSoA& out,
                    cudaStream_t stream) {
  const int threads = kProjectThreads;
  const int blocks = (int)((slot_stride + threads - 1) / threads);
  if (blocks <= 0) return;
  count_launch();
  switch (S) {
    case 0:
      k_project<0><<<blocks, threads, 0, stream>>>(params, N, slot_stride, views, n_views, out);
      break;
    case 3:
      k_project<3><<<blocks, threads, 0, stream>>>(params, N, slot_stride, views, n_views, out);
      break;
    case 8:
      k_project<8><<<blocks, threads, 0, stream>>>(params, N, slot_stride, views, n_views, out);
      break;
    default:
      k_project<15><<<blocks, threads, 0, stream>>>(params, N, slot_stride, views, n_views, out);
      break;
  }
}

}  // namespace pxs
