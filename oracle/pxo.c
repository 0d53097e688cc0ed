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

/* ---------------------------------------------- per-pixel decision margins
 *
 * The compositing loop of rasterizeSplats (SplatRaster.cpp:285-303) makes
 * four threshold decisions per evaluated entry: power > 0 (skip), the cap of
 * alpha at 0.99, alpha < min_alpha (skip) and, after the multiply,
 * T < transmittance_cutoff (stop). Two implementations whose inputs differ in
 * the last bit (glibc's expf is not correctly rounded everywhere; sums round
 * in a different order) can take a decision the other way and change a pixel
 * by far more than their rounding. For every pixel this walks the list in the
 * given order, exactly as the compositing loop does, and reports:
 *   margin[p] the least relative distance of any decision quantity from its
 *             threshold (|power| against the size of its terms; alpha against
 *             min_alpha and 0.99; T against the cutoff), computed in double;
 *   kind[p]   which decision that was: 1 power, 2 alpha floor, 3 cap,
 *             4 cutoff (0 when the pixel evaluated nothing);
 *   tie[p]    1 when a contributing entry shares its depth (bit-equal) with
 *             another entry that would also contribute at the pixel, so their
 *             order, the sort's tie-break, decides the result.
 * Test infrastructure: the parity tests use it to show that every value off
 * by more than the tolerance is a branch flip or a depth tie. */
void pxo_pixel_decisions_f32(const pxs_projected_splat* projected, int32_t count,
                             const pxs_camera* cam, const pxs_raster_options* opt,
                             float* margin, int32_t* kind, int32_t* tie) {
  const int width = cam->width, height = cam->height;
  const size_t pixels = (size_t)width * (size_t)height;
  if (pixels == 0) return;
  const int cols = (width + 15) / 16, rows = (height + 15) / 16;
  const int tiles = cols * rows;
  int32_t* offsets = (int32_t*)malloc(sizeof(int32_t) * (size_t)(tiles + 1));
  int64_t total = build_tiles_internal_f32(projected, count, width, height, offsets, NULL, 0);
  int32_t* entries = (int32_t*)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
  build_tiles_internal_f32(projected, count, width, height, offsets, entries, total);
  const double floor_ = opt->min_alpha, cutoff = opt->transmittance_cutoff;
  for (int ty = 0; ty < rows; ++ty) {
    for (int tx = 0; tx < cols; ++tx) {
      const int tile = ty * cols + tx;
      const int begin = offsets[tile], end = offsets[tile + 1];
      const int y_end = height < (ty + 1) * 16 ? height : (ty + 1) * 16;
      const int x_end = width < (tx + 1) * 16 ? width : (tx + 1) * 16;
      for (int y = ty * 16; y < y_end; ++y) {
        for (int x = tx * 16; x < x_end; ++x) {
          const size_t pixel = (size_t)y * (size_t)width + (size_t)x;
          const float px = (float)x + 0.5f, py = (float)y + 0.5f;
          float T = 1.0f;
          double best = INFINITY;
          int best_kind = 0, tied = 0;
          for (int e = begin; e < end; ++e) {
            const pxs_projected_splat* s = &projected[entries[e]];
            const float dx = px - s->mean[0], dy = py - s->mean[1];
            const float power =
                -0.5f * (s->conic[0] * dx * dx + s->conic[2] * dy * dy) - s->conic[1] * dx * dy;
            const double size = 0.5 * fabs((double)s->conic[0] * dx * dx) +
                                0.5 * fabs((double)s->conic[2] * dy * dy) +
                                fabs((double)s->conic[1] * dx * dy) + 1e-30;
            const double m_power = fabs((double)power) / size;
            if (m_power < best) { best = m_power; best_kind = 1; }
            if (power > 0.0f) continue;
            const float raw = s->opacity * expf(power);
            const double m_cap = fabs((double)raw - 0.99) / 0.99;
            if (m_cap < best) { best = m_cap; best_kind = 3; }
            const float alpha = raw < 0.99f ? raw : 0.99f;
            const double m_floor = fabs((double)alpha - floor_) / floor_;
            if (m_floor < best) { best = m_floor; best_kind = 2; }
            if (alpha < opt->min_alpha) continue;
            /* a contributing entry with another entry of its depth that would
             * also pass both alpha tests here: their order is the tie-break,
             * whichever of them the walk reaches first (the other may lie past
             * the cutoff) */
            if (!tied) {
              for (int dir = -1; dir <= 1 && !tied; dir += 2) {
                for (int f = e + dir; f >= begin && f < end; f += dir) {
                  const pxs_projected_splat* o = &projected[entries[f]];
                  if (memcmp(&o->depth, &s->depth, sizeof(float)) != 0) break;
                  const float ox = px - o->mean[0], oy = py - o->mean[1];
                  const float op = -0.5f * (o->conic[0] * ox * ox + o->conic[2] * oy * oy) -
                                   o->conic[1] * ox * oy;
                  if (op > 0.0f) continue;
                  const float oraw = o->opacity * expf(op);
                  if ((oraw < 0.99f ? oraw : 0.99f) >= opt->min_alpha) {
                    tied = 1;
                    break;
                  }
                }
              }
            }
            T *= 1.0f - alpha;
            const double m_cut = fabs((double)T - cutoff) / cutoff;
            if (m_cut < best) { best = m_cut; best_kind = 4; }
            if (T < opt->transmittance_cutoff) break;
          }
          if (margin) margin[pixel] = best_kind ? (float)best : INFINITY;
          if (kind) kind[pixel] = best_kind;
          if (tie) tie[pixel] = tied;
        }
      }
    }
  }
  free(entries);
  free(offsets);
}
