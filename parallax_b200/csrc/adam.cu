// adam.cu -- the optimiser step, fused with clearing the gradients and with
// folding this step's densification statistics into the running totals.
//
// applyGradients (SplatTrainer.cpp:218-256) with adamDelta (:56-65), one
// thread per gaussian so the quaternion can be renormalised in registers.
// Compiled with -fmad=false: with IEEE division and square root the update is
// bit-identical to the reference's for identical gradients.
#include <type_traits>

#include "common.cuh"
#include "kernels.h"

namespace pxs {

__device__ __forceinline__ float adam_delta(float& m, float& v, float g, float lr, float b1,
                                            float b2, float eps, float c1, float c2) {
  m = b1 * m + (1.f - b1) * g;
  v = b2 * v + (1.f - b2) * g * g;
  const float m_hat = m / c1;
  const float v_hat = v / c2;
  return -lr * m_hat / (sqrtf(v_hat) + eps);
}

__global__ void __launch_bounds__(256, 4)
    k_adam(float* __restrict__ params, float* __restrict__ grads, float* __restrict__ m,
           float* __restrict__ v, int N, int S, const StepScalars* __restrict__ scalars,
           int zero_grads, float* __restrict__ screen_gradient,
           int32_t* __restrict__ visible_count, float* __restrict__ acc_gradient,
           int32_t* __restrict__ acc_views, const int32_t* __restrict__ skip,
           const float* __restrict__ position_scale) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N) return;
  // a step whose tile pairs overflowed is redone by the host: leave the state alone
  if (skip != nullptr && *skip != 0) return;
  const StepScalars& s = *scalars;
  const int64_t n = N;
  const int P = 14 + 3 * S;
  // positionLearningRate (SplatTrainer.cpp:200-208) ends with "* extent": with
  // several scenes lr[0] holds the rest and each gaussian its scene's extent
  const float lr_position = position_scale != nullptr ? s.lr[0] * position_scale[g] : s.lr[0];
  // channels [c0, c0 + K) with learning rate lr(c): every load of the group
  // is issued before its first store, so K channels' loads are in flight at once
  auto update = [&](auto K, int c0, auto lr_of) {
    constexpr int k = decltype(K)::value;
    float pp[k], gg[k], mm[k], vv[k];
#pragma unroll
    for (int j = 0; j < k; ++j) {
      const int64_t i = (int64_t)(c0 + j) * n + g;
      pp[j] = params[i];
      gg[j] = grads[i];
      mm[j] = m[i];
      vv[j] = v[i];
    }
#pragma unroll
    for (int j = 0; j < k; ++j) {
      const int64_t i = (int64_t)(c0 + j) * n + g;
      params[i] = pp[j] + adam_delta(mm[j], vv[j], gg[j], lr_of(c0 + j), s.beta1, s.beta2,
                                     s.epsilon, s.correction1, s.correction2);
      m[i] = mm[j];
      v[i] = vv[j];
      if (zero_grads) grads[i] = 0.f;
    }
  };
  using Six = std::integral_constant<int, 6>;
  using Four = std::integral_constant<int, 4>;
  using One = std::integral_constant<int, 1>;
  // position and log-scale, then opacity and dc, then the SH rest
  update(Six{}, 0, [&](int c) { return c < 3 ? lr_position : s.lr[1]; });
  update(Four{}, PXS_C_OPACITY, [&](int c) { return c == PXS_C_OPACITY ? s.lr[3] : s.lr[4]; });
  int c = PXS_C_SH_REST;
  for (; c + 4 <= P; c += 4) update(Four{}, c, [&](int) { return s.lr[5]; });
  for (; c < P; ++c) update(One{}, c, [&](int) { return s.lr[5]; });
  float q[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int64_t i = (int64_t)(PXS_C_ROTATION + a) * n + g;
    float mm = m[i], vv = v[i];
    q[a] = params[i] + adam_delta(mm, vv, grads[i], s.lr[2], s.beta1, s.beta2, s.epsilon,
                                  s.correction1, s.correction2);
    m[i] = mm;
    v[i] = vv;
    if (zero_grads) grads[i] = 0.f;
  }
  // Quaternion::norm / normalize over (x, y, z, w) storage (SplatTrainer.cpp:247-248)
  const float sq = (q[1] * q[1] + q[3] * q[3]) + (q[2] * q[2] + q[0] * q[0]);
  const float norm = sqrtf(sq);
  if (norm > 1e-6f) {
#pragma unroll
    for (int a = 0; a < 4; ++a) q[a] = q[a] / norm;
  } else {
    q[0] = 1.f;
    q[1] = q[2] = q[3] = 0.f;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) params[(int64_t)(PXS_C_ROTATION + a) * n + g] = q[a];
  // accumulateStatistics (SplatTrainer.cpp:258-263), then this step's stats clear
  if (screen_gradient != nullptr) {
    if (acc_gradient != nullptr) {
      acc_gradient[g] += screen_gradient[g];
      acc_views[g] += visible_count[g];
    }
    if (zero_grads) {
      screen_gradient[g] = 0.f;
      visible_count[g] = 0;
    }
  }
}

void launch_adam(float* params, float* grads, float* m, float* v, int N, int S,
                 const StepScalars* scalars, int zero_grads, float* screen_gradient,
                 int32_t* visible_count, float* acc_gradient, int32_t* acc_views,
                 cudaStream_t stream, const float* position_scale) {
  if (N <= 0) return;
  count_launch();
  k_adam<<<(N + 255) / 256, 256, 0, stream>>>(params, grads, m, v, N, S, scalars, zero_grads,
                                              screen_gradient, visible_count, acc_gradient,
                                              acc_views, nullptr, position_scale);
}

void launch_adam_checked(float* params, float* grads, float* m, float* v, int N, int S,
                         const StepScalars* scalars, float* screen_gradient,
                         int32_t* visible_count, float* acc_gradient, int32_t* acc_views,
                         const int32_t* skip, cudaStream_t stream,
                         const float* position_scale) {
  if (N <= 0) return;
  count_launch();
  k_adam<<<(N + 255) / 256, 256, 0, stream>>>(params, grads, m, v, N, S, scalars, 1,
                                              screen_gradient, visible_count, acc_gradient,
                                              acc_views, skip, position_scale);
}

// resetOpacity (SplatTrainer.cpp:301-309): cap the logit, clear its moments.
__global__ void k_reset_opacity(float* __restrict__ params, float* __restrict__ m,
                                float* __restrict__ v, int N, float ceiling) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N) return;
  const int64_t i = (int64_t)PXS_C_OPACITY * N + g;
  const float x = params[i];
  params[i] = ceiling < x ? ceiling : x;  // std::min(x, ceiling)
  m[i] = 0.f;
  v[i] = 0.f;
}

void launch_reset_opacity(float* params, float* m, float* v, int N, float ceiling,
                          cudaStream_t stream) {
  if (N > 0) {
    count_launch();
    k_reset_opacity<<<(N + 255) / 256, 256, 0, stream>>>(params, m, v, N, ceiling);
  }
}

}  // namespace pxs

namespace pxs {

// The data-parallel reduction block's small parts (see pxs_trainer_accumulate):
// the visible counts as floats (exact for counts below 2^24) and the loss tail
// (mean loss x views, views), so one collective sums everything.
__global__ void k_pack_reduction(const int32_t* __restrict__ visible, float* __restrict__ visible_f,
                                 int N, const float* __restrict__ loss_mean, int n_views,
                                 float* __restrict__ tail) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < N) visible_f[g] = (float)visible[g];
  if (g == 0) {
    tail[0] = loss_mean[0] * (float)n_views;
    tail[1] = (float)n_views;
  }
}

__global__ void k_unpack_visible(const float* __restrict__ visible_f,
                                 int32_t* __restrict__ visible, int N) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < N) visible[g] = (int32_t)rintf(visible_f[g]);
}

void launch_pack_reduction(const int32_t* visible, float* visible_f, int N,
                           const float* loss_mean, int n_views, float* tail,
                           cudaStream_t stream) {
  count_launch();
  k_pack_reduction<<<(std::max(N, 1) + 255) / 256, 256, 0, stream>>>(visible, visible_f, N,
                                                                     loss_mean, n_views, tail);
}

void launch_unpack_visible(const float* visible_f, int32_t* visible, int N, cudaStream_t stream) {
  if (N <= 0) return;
  count_launch();
  k_unpack_visible<<<(N + 255) / 256, 256, 0, stream>>>(visible_f, visible, N);
}

}  // namespace pxs
