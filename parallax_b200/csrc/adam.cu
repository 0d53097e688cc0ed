// adam.cu -- the optimiser step, fused with clearing the gradients and with
// folding this step's densification statistics into the running totals.
//
// applyGradients (SplatTrainer.cpp:218-256) with adamDelta (:56-65), one
// thread per gaussian so the quaternion can be renormalised in registers.
// Compiled with -fmad=false: with IEEE division and square root the update is
// bit-identical to the reference's for identical gradients.
#include <tuple>
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

// Adam as an elementwise pass over (task, group of four gaussians), for N a
// multiple of 4 (every component row then starts on a 16-byte boundary): a
// thread updates one parameter row of four consecutive gaussians with 16-byte
// loads and stores. Task t < 6 is row t (position, log-scale); task 6 is the
// four rotation rows together, so the quaternion is renormalised in
// registers; tasks 7.. are rows 10.. (opacity, dc, sh_rest); with statistics
// the last task folds this step's densify statistics into the running totals.
// Element by element the arithmetic of k_adam, so the results are the same
// bits; many small independent threads keep enough loads in flight to stream
// the eight P x N arrays at close to the memory bandwidth.
__device__ __forceinline__ void ld4(const float* base, int64_t row, int64_t n, int g4,
                                    float (&x)[4]) {
  const float4 t = reinterpret_cast<const float4*>(base + row * n)[g4];
  x[0] = t.x;
  x[1] = t.y;
  x[2] = t.z;
  x[3] = t.w;
}
__device__ __forceinline__ void st4(float* base, int64_t row, int64_t n, int g4,
                                    const float (&x)[4]) {
  reinterpret_cast<float4*>(base + row * n)[g4] = make_float4(x[0], x[1], x[2], x[3]);
}

__global__ void __launch_bounds__(256)
    k_adam_rows(float* __restrict__ params, float* __restrict__ grads, float* __restrict__ m,
                float* __restrict__ v, int N, int S, const StepScalars* __restrict__ scalars,
                int zero_grads, float* __restrict__ screen_gradient,
                int32_t* __restrict__ visible_count, float* __restrict__ acc_gradient,
                int32_t* __restrict__ acc_views, const int32_t* __restrict__ skip,
                const float* __restrict__ position_scale) {
  const int g4 = blockIdx.x * blockDim.x + threadIdx.x;
  if (g4 >= N / 4) return;
  if (skip != nullptr && *skip != 0) return;
  const StepScalars& s = *scalars;
  const int64_t n = N;
  const int P = 14 + 3 * S;
  const int task = blockIdx.y;
  const float zero[4] = {0.f, 0.f, 0.f, 0.f};
  if (task == 6) {
    float q[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      float pp[4], gg[4], mm[4], vv[4];
      ld4(params, PXS_C_ROTATION + a, n, g4, pp);
      ld4(grads, PXS_C_ROTATION + a, n, g4, gg);
      ld4(m, PXS_C_ROTATION + a, n, g4, mm);
      ld4(v, PXS_C_ROTATION + a, n, g4, vv);
#pragma unroll
      for (int e = 0; e < 4; ++e)
        q[a][e] = pp[e] + adam_delta(mm[e], vv[e], gg[e], s.lr[2], s.beta1, s.beta2, s.epsilon,
                                     s.correction1, s.correction2);
      st4(m, PXS_C_ROTATION + a, n, g4, mm);
      st4(v, PXS_C_ROTATION + a, n, g4, vv);
      if (zero_grads) st4(grads, PXS_C_ROTATION + a, n, g4, zero);
    }
    // Quaternion::norm / normalize over (x, y, z, w) storage (SplatTrainer.cpp:247-248)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float w = q[0][e], x = q[1][e], y = q[2][e], z = q[3][e];
      const float sq = (x * x + z * z) + (y * y + w * w);
      const float norm = sqrtf(sq);
      if (norm > 1e-6f) {
#pragma unroll
        for (int a = 0; a < 4; ++a) q[a][e] = q[a][e] / norm;
      } else {
        q[0][e] = 1.f;
        q[1][e] = q[2][e] = q[3][e] = 0.f;
      }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) st4(params, PXS_C_ROTATION + a, n, g4, q[a]);
    return;
  }
  const int row = task < 6 ? task : task + 3;  // tasks 7.. are rows 10..
  if (row < P) {
    float lr[4];
    if (row < 3) {
      float ps[4] = {1.f, 1.f, 1.f, 1.f};
      if (position_scale != nullptr) ld4(position_scale, 0, n, g4, ps);
#pragma unroll
      for (int e = 0; e < 4; ++e) lr[e] = position_scale != nullptr ? s.lr[0] * ps[e] : s.lr[0];
    } else {
      const float r = row < PXS_C_ROTATION ? s.lr[1]
                      : row == PXS_C_OPACITY ? s.lr[3]
                      : row < PXS_C_SH_REST  ? s.lr[4]
                                             : s.lr[5];
#pragma unroll
      for (int e = 0; e < 4; ++e) lr[e] = r;
    }
    float pp[4], gg[4], mm[4], vv[4];
    ld4(params, row, n, g4, pp);
    ld4(grads, row, n, g4, gg);
    ld4(m, row, n, g4, mm);
    ld4(v, row, n, g4, vv);
#pragma unroll
    for (int e = 0; e < 4; ++e)
      pp[e] += adam_delta(mm[e], vv[e], gg[e], lr[e], s.beta1, s.beta2, s.epsilon,
                          s.correction1, s.correction2);
    st4(params, row, n, g4, pp);
    st4(m, row, n, g4, mm);
    st4(v, row, n, g4, vv);
    if (zero_grads) st4(grads, row, n, g4, zero);
    return;
  }
  // accumulateStatistics (SplatTrainer.cpp:258-263), then this step's stats clear
  if (screen_gradient != nullptr) {
    float4* sg = reinterpret_cast<float4*>(screen_gradient);
    int4* vc = reinterpret_cast<int4*>(visible_count);
    if (acc_gradient != nullptr) {
      float4 a4 = reinterpret_cast<float4*>(acc_gradient)[g4];
      const float4 b = sg[g4];
      a4.x += b.x;
      a4.y += b.y;
      a4.z += b.z;
      a4.w += b.w;
      reinterpret_cast<float4*>(acc_gradient)[g4] = a4;
      int4 av = reinterpret_cast<int4*>(acc_views)[g4];
      const int4 bv = vc[g4];
      av.x += bv.x;
      av.y += bv.y;
      av.z += bv.z;
      av.w += bv.w;
      reinterpret_cast<int4*>(acc_views)[g4] = av;
    }
    if (zero_grads) {
      sg[g4] = make_float4(0.f, 0.f, 0.f, 0.f);
      vc[g4] = make_int4(0, 0, 0, 0);
    }
  }
}

// The elementwise form where every row (and every statistics array) is
// 16-byte aligned, else one gaussian per thread.
template <typename... A>
void launch_adam_kernel(int N, const float* params, const float* grads, const float* screen,
                        const int32_t* visible, const float* acc_gradient,
                        const int32_t* acc_views, const float* position_scale,
                        cudaStream_t stream, A... args) {
  auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  const bool wide = N % 4 == 0 && aligned(params) && aligned(grads) &&
                    (screen == nullptr || (aligned(screen) && aligned(visible))) &&
                    (acc_gradient == nullptr || (aligned(acc_gradient) && aligned(acc_views))) &&
                    (position_scale == nullptr || aligned(position_scale));
  count_launch();
  if (wide) {
    // tasks: rows 0-5, the rotation rows, rows 10..P-1, the statistics
    const int S = std::get<5>(std::make_tuple(args...));
    const int tasks = 6 + 1 + (14 + 3 * S - 10) + (screen != nullptr ? 1 : 0);
    k_adam_rows<<<dim3((N / 4 + 255) / 256, tasks), 256, 0, stream>>>(args...);
  } else {
    k_adam<<<(N + 255) / 256, 256, 0, stream>>>(args...);
  }
}

void launch_adam(float* params, float* grads, float* m, float* v, int N, int S,
                 const StepScalars* scalars, int zero_grads, float* screen_gradient,
                 int32_t* visible_count, float* acc_gradient, int32_t* acc_views,
                 cudaStream_t stream, const float* position_scale) {
  if (N <= 0) return;
  launch_adam_kernel(N, params, grads, screen_gradient, visible_count, acc_gradient, acc_views,
                     position_scale, stream, params, grads, m, v, N, S, scalars, zero_grads,
                     screen_gradient, visible_count, acc_gradient, acc_views,
                     static_cast<const int32_t*>(nullptr), position_scale);
}

void launch_adam_checked(float* params, float* grads, float* m, float* v, int N, int S,
                         const StepScalars* scalars, float* screen_gradient,
                         int32_t* visible_count, float* acc_gradient, int32_t* acc_views,
                         const int32_t* skip, cudaStream_t stream,
                         const float* position_scale) {
  if (N <= 0) return;
  launch_adam_kernel(N, params, grads, screen_gradient, visible_count, acc_gradient, acc_views,
                     position_scale, stream, params, grads, m, v, N, S, scalars, 1,
                     screen_gradient, visible_count, acc_gradient, acc_views, skip,
                     position_scale);
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
