/*
 * pxo.c -- CPU oracle instantiations (test infrastructure; see pxo.h).
 *
 * Compile with IEEE single-precision semantics and no contraction
 * (-O2 -ffp-contract=off, no -ffast-math): the f32 functions then reproduce
 * the reference's own IEEE build bit for bit.
 */
#include "pxo.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)

/* ----------------------------------------------------------- float build */
#define REAL float
#define SFX(n) CAT(n, _f32)
#define C(x) CAT(x, f)
#define EXPR expf
#define SQRTR sqrtf
#define FLOORR floorf
#define FABSR fabsf
#define COPYSIGNR copysignf
#define SPLAT pxs_projected_splat
#include "pxo_impl.h"
#undef REAL
#undef SFX
#undef C
#undef EXPR
#undef SQRTR
#undef FLOORR
#undef FABSR
#undef COPYSIGNR
#undef SPLAT

/* ---------------------------------------------------------- double build */
#define REAL double
#define SFX(n) CAT(n, _f64)
#define C(x) x
#define EXPR exp
#define SQRTR sqrt
#define FLOORR floor
#define FABSR fabs
#define COPYSIGNR copysign
#define SPLAT pxo_splat_f64
#include "pxo_impl.h"
#undef REAL
#undef SFX
#undef C
#undef EXPR
#undef SQRTR
#undef FLOORR
#undef FABSR
#undef COPYSIGNR
#undef SPLAT

/* ------------------------------------------------------ public wrappers */

void pxo_evaluate_sh_f32(const float* params, int32_t n, int32_t g, int32_t rest_per_channel,
                         int32_t degree, const float direction[3], float color[3],
                         uint32_t* clamped) {
  evaluate_sh_internal_f32(params, n, g, rest_per_channel, degree, direction, color, clamped);
}

int32_t pxo_project_f32(const float* params, int32_t n, int32_t rest_per_channel,
                        int32_t cloud_sh_degree, const pxs_camera* camera,
                        const pxs_raster_options* options, pxs_projected_splat* out) {
  return project_internal_f32(params, n, rest_per_channel, cloud_sh_degree, camera, options,
                              out);
}

int64_t pxo_build_tiles_f32(const pxs_projected_splat* projected, int32_t count, int32_t width,
                            int32_t height, int32_t* offsets, int32_t* entries,
                            int64_t capacity) {
  return build_tiles_internal_f32(projected, count, width, height, offsets, entries, capacity);
}

void pxo_rasterize_f32(const pxs_projected_splat* projected, int32_t count,
                       const pxs_camera* camera, const pxs_raster_options* options, float* rgb,
                       float* transmittance) {
  rasterize_internal_f32(projected, count, camera, options, rgb, transmittance);
}

float pxo_mean_ssim_f32(const float* rendered, const float* target, int32_t width,
                        int32_t height, float* d_rendered) {
  return mean_ssim_internal_f32(rendered, target, width, height, d_rendered);
}

float pxo_photometric_loss_f32(const float* rendered, const float* target, int32_t width,
                               int32_t height, float ssim_weight, float* dL_drgb) {
  return photometric_loss_internal_f32(rendered, target, width, height, ssim_weight, dL_drgb);
}

void pxo_backward_f32(const float* params, int32_t n, int32_t rest_per_channel,
                      int32_t cloud_sh_degree, const pxs_camera* camera,
                      const pxs_raster_options* options, const pxs_projected_splat* projected,
                      int32_t count, const float* rgb, const float* dL_drgb, float* grads,
                      float* screen_gradient, int32_t* visible_count) {
  (void)rgb;
  backward_internal_f32(params, n, rest_per_channel, cloud_sh_degree, camera, options,
                        projected, count, dL_drgb, grads, screen_gradient, visible_count);
}

float pxo_render_and_accumulate_f32(const float* params, int32_t n, int32_t rest_per_channel,
                                    int32_t cloud_sh_degree, const pxs_camera* camera,
                                    const pxs_raster_options* options, const float* target,
                                    float ssim_weight, float* grads, float* screen_gradient,
                                    int32_t* visible_count) {
  pxs_projected_splat* projected =
      (pxs_projected_splat*)malloc(sizeof(pxs_projected_splat) * (size_t)(n > 0 ? n : 1));
  const int32_t count =
      project_internal_f32(params, n, rest_per_channel, cloud_sh_degree, camera, options,
                           projected);
  const size_t pixels = (size_t)camera->width * (size_t)camera->height;
  float* rgb = (float*)malloc(sizeof(float) * (pixels * 3 + 1));
  float* dL = (float*)malloc(sizeof(float) * (pixels * 3 + 1));
  rasterize_internal_f32(projected, count, camera, options, rgb, NULL);
  const float loss = photometric_loss_internal_f32(rgb, target, camera->width, camera->height,
                                                   ssim_weight, dL);
  backward_internal_f32(params, n, rest_per_channel, cloud_sh_degree, camera, options,
                        projected, count, dL, grads, screen_gradient, visible_count);
  free(dL);
  free(rgb);
  free(projected);
  return loss;
}

int32_t pxo_project_f64(const double* params, int32_t n, int32_t rest_per_channel,
                        int32_t cloud_sh_degree, const pxs_camera* camera,
                        const pxs_raster_options* options, pxo_splat_f64* out) {
  return project_internal_f64(params, n, rest_per_channel, cloud_sh_degree, camera, options,
                              out);
}

void pxo_rasterize_f64(const pxo_splat_f64* projected, int32_t count, const pxs_camera* camera,
                       const pxs_raster_options* options, double* rgb, double* transmittance) {
  rasterize_internal_f64(projected, count, camera, options, rgb, transmittance);
}

double pxo_mean_ssim_f64(const double* rendered, const double* target, int32_t width,
                         int32_t height, double* d_rendered) {
  return mean_ssim_internal_f64(rendered, target, width, height, d_rendered);
}

double pxo_photometric_loss_f64(const double* rendered, const double* target, int32_t width,
                                int32_t height, double ssim_weight, double* dL_drgb) {
  return photometric_loss_internal_f64(rendered, target, width, height, ssim_weight, dL_drgb);
}

void pxo_backward_f64(const double* params, int32_t n, int32_t rest_per_channel,
                      int32_t cloud_sh_degree, const pxs_camera* camera,
                      const pxs_raster_options* options, const pxo_splat_f64* projected,
                      int32_t count, const double* rgb, const double* dL_drgb, double* grads,
                      double* screen_gradient, int32_t* visible_count) {
  (void)rgb;
  backward_internal_f64(params, n, rest_per_channel, cloud_sh_degree, camera, options,
                        projected, count, dL_drgb, grads, screen_gradient, visible_count);
}

void pxo_render_f64(const double* params, int32_t n, int32_t rest_per_channel,
                    int32_t cloud_sh_degree, const pxs_camera* camera,
                    const pxs_raster_options* options, double* rgb) {
  pxo_splat_f64* projected =
      (pxo_splat_f64*)malloc(sizeof(pxo_splat_f64) * (size_t)(n > 0 ? n : 1));
  const int32_t count = project_internal_f64(params, n, rest_per_channel, cloud_sh_degree,
                                             camera, options, projected);
  rasterize_internal_f64(projected, count, camera, options, rgb, NULL);
  free(projected);
}

double pxo_objective_f64(const double* params, int32_t n, int32_t rest_per_channel,
                         int32_t cloud_sh_degree, const pxs_camera* camera,
                         const pxs_raster_options* options, const double* target,
                         double ssim_weight) {
  const size_t values = (size_t)camera->width * (size_t)camera->height * 3;
  double* rgb = (double*)malloc(sizeof(double) * (values + 1));
  pxo_render_f64(params, n, rest_per_channel, cloud_sh_degree, camera, options, rgb);
  double result = 0.0;
  if (ssim_weight < 0.0) {
    for (size_t i = 0; i < values; ++i) result += target[i] * rgb[i];
  } else {
    result = photometric_loss_internal_f64(rgb, target, camera->width, camera->height,
                                           ssim_weight, NULL);
  }
  free(rgb);
  return result;
}

/* ------------------------------------------------------------------ Adam */

/* adamDelta (SplatTrainer.cpp:56-65). */
static float adam_delta(float* m, float* v, float g, float lr, float b1, float b2, float eps,
                        float c1, float c2) {
  *m = b1 * *m + (1.f - b1) * g;
  *v = b2 * *v + (1.f - b2) * g * g;
  const float m_hat = *m / c1;
  const float v_hat = *v / c2;
  return -lr * m_hat / (sqrtf(v_hat) + eps);
}

/* applyGradients (SplatTrainer.cpp:218-256). */
void pxo_adam_f32(float* params, const float* grads, float* m, float* v, int32_t n,
                  int32_t rest_per_channel, const float lr[6], float beta1, float beta2,
                  float epsilon, float correction1, float correction2) {
  const size_t N = (size_t)n;
#define IDX(c, g) ((size_t)(c) * N + (size_t)(g))
#define STEP(c, g, rate)                                                                     \
  params[IDX(c, g)] += adam_delta(&m[IDX(c, g)], &v[IDX(c, g)], grads[IDX(c, g)], (rate), \
                                  beta1, beta2, epsilon, correction1, correction2)
  for (int32_t g = 0; g < n; ++g) {
    for (int a = 0; a < 3; ++a) {
      STEP(0 + a, g, lr[0]);
      STEP(3 + a, g, lr[1]);
      STEP(11 + a, g, lr[4]);
    }
    STEP(10, g, lr[3]);
    for (int a = 0; a < 4; ++a) STEP(6 + a, g, lr[2]);
    /* Quaternion::norm / normalize over (x, y, z, w) storage (SplatTrainer.cpp:247-248) */
    const float w = params[IDX(6, g)], x = params[IDX(7, g)], y = params[IDX(8, g)],
                z = params[IDX(9, g)];
    const float sq = (x * x + z * z) + (y * y + w * w);
    if (sqrtf(sq) > 1e-6f) {
      const float norm = sqrtf(sq);
      params[IDX(6, g)] = w / norm;
      params[IDX(7, g)] = x / norm;
      params[IDX(8, g)] = y / norm;
      params[IDX(9, g)] = z / norm;
    } else {
      params[IDX(6, g)] = 1.f;
      params[IDX(7, g)] = 0.f;
      params[IDX(8, g)] = 0.f;
      params[IDX(9, g)] = 0.f;
    }
    for (int k = 0; k < 3 * rest_per_channel; ++k) STEP(14 + k, g, lr[5]);
  }
#undef STEP
#undef IDX
}

/* ------------------------------------------------------------- densify */

/* nextNormal (SplatDensify.cpp:11-24). */
static uint32_t xorshift32(uint32_t* state) {
  uint32_t x = *state;
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  *state = x == 0u ? 1u : x;
  return *state;
}

float pxo_next_normal(uint32_t* state) {
  float u1 = (float)xorshift32(state) / 4294967296.f;
  if (u1 < 1e-7f) u1 = 1e-7f;
  const float u2 = (float)xorshift32(state) / 4294967296.f;
  return sqrtf(-2.f * logf(u1)) * cosf(2.f * 3.14159265358979f * u2);
}

static float opacity_of(float logit) { return 1.0f / (1.0f + expf(-logit)); }

static float largest_scale(const float* params, size_t N, size_t g) {
  float best = expf(params[3 * N + g]);
  for (int a = 1; a < 3; ++a) {
    const float s = expf(params[(3 + a) * N + g]);
    if (s > best) best = s;
  }
  return best;
}

/* densifyAndPrune (SplatDensify.cpp:28-109). `params` has room for
 * config->max_gaussians gaussians laid out with stride max_gaussians on
 * output; on input the stride is n. */
int32_t pxo_densify_and_prune(float* params, int32_t n, int32_t rest_per_channel,
                              const float* screen_gradient, const int32_t* visible_count,
                              const pxs_train_config* config, float extent, int32_t iteration,
                              uint32_t* rng_state, int32_t* source, int32_t* cloned,
                              int32_t* split, int32_t* pruned) {
  const int P = 14 + 3 * rest_per_channel;
  const size_t N = (size_t)n;
  *cloned = *split = *pruned = 0;
  if (n == 0) return 0;
  const float size_threshold = config->percent_dense * extent;
  char* keep = (char*)malloc(N);
  memset(keep, 1, N);
  /* additions: at most 2 per gaussian */
  float* add = (float*)malloc(sizeof(float) * (size_t)P * (2 * N + 1));
  size_t n_add = 0;
  const int has_room = n < config->max_gaussians;
  if (has_room) {
    for (size_t g = 0; g < N; ++g) {
      const int views = visible_count[g];
      if (views <= 0) continue;
      const float mean_gradient = screen_gradient[g] / (float)views;
      if (mean_gradient < config->densify_grad_threshold) continue;
      const float largest = largest_scale(params, N, g);
      if (largest <= size_threshold) {
        for (int c = 0; c < P; ++c) add[n_add * (size_t)P + (size_t)c] = params[c * N + g];
        ++n_add;
        ++*cloned;
      } else {
        float scale[3], q[4], qn[4], R[9];
        for (int a = 0; a < 3; ++a) scale[a] = expf(params[(3 + a) * N + g]);
        for (int a = 0; a < 4; ++a) q[a] = params[(6 + a) * N + g];
        quat_normalized_f32(q, qn);
        quat_to_matrix_f32(qn, R);
        const float log_div = logf(config->split_scale_divider);
        for (int child = 0; child < 2; ++child) {
          /* The compiled reference draws the three normals of
           * Vec3f(n()*sx, n()*sy, n()*sz) last argument first. */
          const float nz = pxo_next_normal(rng_state);
          const float ny = pxo_next_normal(rng_state);
          const float nx = pxo_next_normal(rng_state);
          const float sample[3] = {nx * scale[0], ny * scale[1], nz * scale[2]};
          float* dst = &add[n_add * (size_t)P];
          for (int c = 0; c < P; ++c) dst[c] = params[c * N + g];
          for (int i = 0; i < 3; ++i) {
            dst[i] = params[i * N + g] + (R[i * 3 + 0] * sample[0] +
                                          (R[i * 3 + 1] * sample[1] + R[i * 3 + 2] * sample[2]));
          }
          for (int a = 0; a < 3; ++a) dst[3 + a] = params[(3 + a) * N + g] - log_div;
          ++n_add;
        }
        keep[g] = 0;
        ++*split;
      }
    }
  }
  const int prune_oversized = iteration > config->opacity_reset_interval;
  const float max_scale = config->prune_scale_fraction * extent;
  const int cap = config->max_gaussians;
  float* out = (float*)malloc(sizeof(float) * (size_t)P * (N + n_add + 1));
  size_t count = 0;
  for (size_t g = 0; g < N; ++g) {
    if (!keep[g]) continue;
    const int prunable = opacity_of(params[10 * N + g]) < config->prune_opacity ||
                         (prune_oversized && largest_scale(params, N, g) > max_scale);
    if (prunable) {
      ++*pruned;
      continue;
    }
    for (int c = 0; c < P; ++c) out[count * (size_t)P + (size_t)c] = params[c * N + g];
    source[count] = (int32_t)g;
    ++count;
  }
  for (size_t a = 0; a < n_add; ++a) {
    if ((int)count >= cap) break;
    const float* src = &add[a * (size_t)P];
    float ls = expf(src[3]);
    for (int k = 1; k < 3; ++k) {
      const float s = expf(src[3 + k]);
      if (s > ls) ls = s;
    }
    const int prunable = opacity_of(src[10]) < config->prune_opacity ||
                         (prune_oversized && ls > max_scale);
    if (prunable) {
      ++*pruned;
      continue;
    }
    memcpy(&out[count * (size_t)P], src, sizeof(float) * (size_t)P);
    source[count] = -1;
    ++count;
  }
  /* back to component-major with stride `count` */
  for (int c = 0; c < P; ++c)
    for (size_t g = 0; g < count; ++g) params[(size_t)c * count + g] = out[g * (size_t)P + (size_t)c];
  free(out);
  free(add);
  free(keep);
  return (int32_t)count;
}
