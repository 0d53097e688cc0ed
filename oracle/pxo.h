/*
 * pxo.h -- CPU oracle for the splat training path (test infrastructure).
 *
 * A plain-C restatement of the reference's CPU splat maths
 * (engine/native/cpp/src/splat/SplatRaster.cpp, SplatTrainer.cpp,
 * SplatDensify.cpp), used only by the tests, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline leg to check the CUDA path. It is never linked into
 * the product library.
 *
 * Two instantiations share one source (pxo_impl.h):
 *   *_f32  single precision, evaluated in the reference's operation order
 *          (including Eigen's association of small fixed-size products), so
 *          that with IEEE evaluation it reproduces the reference bit for bit;
 *   *_f64  the same equations in double precision, for finite differences.
 *
 * Parity of the f32 instantiation is pinned against the reference itself,
 * compiled from its own sources into oracle/_ref/ (see oracle/Makefile), and
 * against the golden fixtures under tests/golden/.
 */
#ifndef PXO_H
#define PXO_H

#include <stdint.h>

#include "pxs.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Projected splat with REAL = double fields (the f64 instantiation). */
typedef struct pxo_splat_f64 {
  int32_t index;
  double mean[2];
  double cov2d[3];
  double conic[3];
  double depth;
  double radius;
  double color[3];
  double opacity;
  uint32_t clamped;
} pxo_splat_f64;

/* ---- single precision (bit-level restatement) ---- */

void pxo_evaluate_sh_f32(const float* params, int32_t n, int32_t g, int32_t rest_per_channel,
                         int32_t degree, const float direction[3], float color[3],
                         uint32_t* clamped);
int32_t pxo_project_f32(const float* params, int32_t n, int32_t rest_per_channel,
                        int32_t cloud_sh_degree, const pxs_camera* camera,
                        const pxs_raster_options* options, pxs_projected_splat* out);
/* Tile lists over `projected` (indices into `projected`), SplatRaster.cpp:114-151.
 * Returns the pair count; writes at most `capacity` entries. */
int64_t pxo_build_tiles_f32(const pxs_projected_splat* projected, int32_t count, int32_t width,
                            int32_t height, int32_t* offsets, int32_t* entries,
                            int64_t capacity);
void pxo_rasterize_f32(const pxs_projected_splat* projected, int32_t count,
                       const pxs_camera* camera, const pxs_raster_options* options, float* rgb,
                       float* transmittance);
float pxo_mean_ssim_f32(const float* rendered, const float* target, int32_t width,
                        int32_t height, float* d_rendered);
float pxo_photometric_loss_f32(const float* rendered, const float* target, int32_t width,
                               int32_t height, float ssim_weight, float* dL_drgb);
/* Adds into grads (P x n), screen_gradient (n) and visible_count (n). */
void pxo_backward_f32(const float* params, int32_t n, int32_t rest_per_channel,
                      int32_t cloud_sh_degree, const pxs_camera* camera,
                      const pxs_raster_options* options, const pxs_projected_splat* projected,
                      int32_t count, const float* rgb, const float* dL_drgb, float* grads,
                      float* screen_gradient, int32_t* visible_count);
/* project + rasterise + loss + backward; returns the loss. */
float pxo_render_and_accumulate_f32(const float* params, int32_t n, int32_t rest_per_channel,
                                    int32_t cloud_sh_degree, const pxs_camera* camera,
                                    const pxs_raster_options* options, const float* target,
                                    float ssim_weight, float* grads, float* screen_gradient,
                                    int32_t* visible_count);
/* One Adam step (SplatTrainer.cpp:56-65, :218-256); lr[6] per group. */
void pxo_adam_f32(float* params, const float* grads, float* m, float* v, int32_t n,
                  int32_t rest_per_channel, const float lr[6], float beta1, float beta2,
                  float epsilon, float correction1, float correction2);

/* ---- double precision (finite differences) ---- */

int32_t pxo_project_f64(const double* params, int32_t n, int32_t rest_per_channel,
                        int32_t cloud_sh_degree, const pxs_camera* camera,
                        const pxs_raster_options* options, pxo_splat_f64* out);
void pxo_rasterize_f64(const pxo_splat_f64* projected, int32_t count, const pxs_camera* camera,
                       const pxs_raster_options* options, double* rgb, double* transmittance);
double pxo_mean_ssim_f64(const double* rendered, const double* target, int32_t width,
                         int32_t height, double* d_rendered);
double pxo_photometric_loss_f64(const double* rendered, const double* target, int32_t width,
                                int32_t height, double ssim_weight, double* dL_drgb);
void pxo_backward_f64(const double* params, int32_t n, int32_t rest_per_channel,
                      int32_t cloud_sh_degree, const pxs_camera* camera,
                      const pxs_raster_options* options, const pxo_splat_f64* projected,
                      int32_t count, const double* rgb, const double* dL_drgb, double* grads,
                      double* screen_gradient, int32_t* visible_count);
/* Renders into rgb (width*height*3) in double precision. */
void pxo_render_f64(const double* params, int32_t n, int32_t rest_per_channel,
                    int32_t cloud_sh_degree, const pxs_camera* camera,
                    const pxs_raster_options* options, double* rgb);
/* Loss of a double-precision render against `target`: ssim_weight >= 0 gives
 * the photometric loss; ssim_weight < 0 gives the linear functional
 * sum(weights * rgb) used by the reference's gradient check
 * (SplatRasterTest.cpp:99-112), with `target` holding the weights. */
double pxo_objective_f64(const double* params, int32_t n, int32_t rest_per_channel,
                         int32_t cloud_sh_degree, const pxs_camera* camera,
                         const pxs_raster_options* options, const double* target,
                         double ssim_weight);

/* ---- densification (SplatDensify.cpp:11-109), single precision ---- */

/* `params` has room for max_gaussians; returns the new count. `source` gets
 * the old index or -1 per new gaussian. */
int32_t pxo_densify_and_prune(float* params, int32_t n, int32_t rest_per_channel,
                              const float* screen_gradient, const int32_t* visible_count,
                              const pxs_train_config* config, float extent, int32_t iteration,
                              uint32_t* rng_state, int32_t* source, int32_t* cloned,
                              int32_t* split, int32_t* pruned);
/* One Box-Muller normal from the reference's xorshift32 (SplatDensify.cpp:11-24). */
float pxo_next_normal(uint32_t* state);

/* Per-pixel decision margins of the compositing loop in the given list order
 * (least relative distance of power, alpha and T from their thresholds, which
 * decision it was, and whether two contributing entries share a depth); see
 * pxo.c. */
void pxo_pixel_decisions_f32(const pxs_projected_splat* projected, int32_t count,
                             const pxs_camera* cam, const pxs_raster_options* opt,
                             float* margin, int32_t* kind, int32_t* tie);

#ifdef __cplusplus
}
#endif

#endif /* PXO_H */
