// ref_api.cpp -- extern "C" entry points onto the reference's own CPU splat
// code (test infrastructure).
//
// oracle/Makefile compiles this file together with the reference's sources,
// where they lie (engine/native/cpp/src/splat/{SplatRaster,SplatTrainer,
// SplatDensify,GaussianCloud}.cpp and src/io/ImageIo.cpp), into
// oracle/_ref/libpxref_ieee.so (IEEE arithmetic, the parity oracle) and
// oracle/_ref/libpxref_fast.so (the reference's own -O3 -ffast-math flags,
// the timed CPU baseline). Nothing here computes anything itself: it only
// converts between the component-major float arrays of pxs.h and the
// reference's GaussianCloud / SplatView / SplatGradients types and calls the
// reference's public functions.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "parallax/io/ImageIo.h"
#include "parallax/splat/SplatDensify.h"
#include "parallax/splat/SplatRaster.h"
#include "parallax/splat/SplatTrainer.h"
#include "parallax/testing/SyntheticScene.h"
#include "pxs.h"

#ifdef PXREF_SHIM
#include <algorithm>
#include <chrono>
#include <limits>
#include <stdexcept>

#include "CudaSplatTrainer.h"
#endif

using namespace parallax;

namespace {

GaussianCloud toCloud(const float* params, int n, int rest, int sh_degree) {
  GaussianCloud cloud;
  cloud.sh_degree = sh_degree;
  cloud.gaussians.resize(static_cast<size_t>(n));
  const size_t N = static_cast<size_t>(n);
  for (size_t g = 0; g < N; ++g) {
    Gaussian& G = cloud.gaussians[g];
    G.position = Vec3f(params[0 * N + g], params[1 * N + g], params[2 * N + g]);
    G.log_scale = Vec3f(params[3 * N + g], params[4 * N + g], params[5 * N + g]);
    G.rotation = Eigen::Quaternionf(params[6 * N + g], params[7 * N + g], params[8 * N + g],
                                    params[9 * N + g]);
    G.opacity_logit = params[10 * N + g];
    for (int c = 0; c < 3; ++c) G.dc[c] = params[(11 + c) * N + g];
    G.sh_rest.resize(static_cast<size_t>(3 * rest));
    for (int k = 0; k < 3 * rest; ++k) G.sh_rest[k] = params[(14 + k) * N + g];
  }
  return cloud;
}

int fromCloud(const GaussianCloud& cloud, int rest, float* params, int capacity) {
  const int n = static_cast<int>(cloud.size());
  if (n > capacity) return -n;
  const size_t N = static_cast<size_t>(n);
  for (size_t g = 0; g < N; ++g) {
    const Gaussian& G = cloud.gaussians[g];
    for (int a = 0; a < 3; ++a) {
      params[(0 + a) * N + g] = G.position[a];
      params[(3 + a) * N + g] = G.log_scale[a];
      params[(11 + a) * N + g] = G.dc[a];
    }
    params[6 * N + g] = G.rotation.w();
    params[7 * N + g] = G.rotation.x();
    params[8 * N + g] = G.rotation.y();
    params[9 * N + g] = G.rotation.z();
    params[10 * N + g] = G.opacity_logit;
    for (int k = 0; k < 3 * rest; ++k) params[(14 + k) * N + g] = G.sh_rest[k];
  }
  return n;
}

SplatView toView(const double* K, int width, int height, const double* R, const double* t) {
  SplatView view;
  view.intrinsics.fx = K[0];
  view.intrinsics.fy = K[1];
  view.intrinsics.cx = K[2];
  view.intrinsics.cy = K[3];
  view.intrinsics.width = width;
  view.intrinsics.height = height;
  Mat3 rot;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) rot(r, c) = R[r * 3 + c];
  view.camera_from_world = Pose(rot, Vec3(t[0], t[1], t[2]));
  return view;
}

RasterOptions toOptions(const pxs_raster_options* o) {
  RasterOptions options;
  if (o == nullptr) return options;
  for (int c = 0; c < 3; ++c) options.background[c] = o->background[c];
  options.sh_degree = o->sh_degree;
  options.min_alpha = o->min_alpha;
  options.transmittance_cutoff = o->transmittance_cutoff;
  options.screen_dilation = o->screen_dilation;
  return options;
}

SplatTrainingConfig toConfig(const pxs_train_config* c) {
  SplatTrainingConfig config;
  config.iterations = c->iterations;
  config.position_lr_initial = c->position_lr_initial;
  config.position_lr_final = c->position_lr_final;
  config.dc_lr = c->dc_lr;
  config.sh_rest_lr_divider = c->sh_rest_lr_divider;
  config.opacity_lr = c->opacity_lr;
  config.scale_lr = c->scale_lr;
  config.rotation_lr = c->rotation_lr;
  config.adam_beta1 = c->adam_beta1;
  config.adam_beta2 = c->adam_beta2;
  config.adam_epsilon = c->adam_epsilon;
  config.ssim_weight = c->ssim_weight;
  config.sh_degree = c->sh_degree;
  config.sh_increase_interval = c->sh_increase_interval;
  config.densify_from_iteration = c->densify_from_iteration;
  config.densify_until_iteration = c->densify_until_iteration;
  config.densify_interval = c->densify_interval;
  config.densify_grad_threshold = c->densify_grad_threshold;
  config.percent_dense = c->percent_dense;
  config.split_scale_divider = c->split_scale_divider;
  config.opacity_reset_interval = c->opacity_reset_interval;
  config.opacity_reset_value = c->opacity_reset_value;
  config.prune_opacity = c->prune_opacity;
  config.prune_scale_fraction = c->prune_scale_fraction;
  config.max_gaussians = c->max_gaussians;
  config.seed = c->seed;
  return config;
}

void toProjected(const ProjectedSplat& s, pxs_projected_splat* o) {
  o->index = s.index;
  o->mean[0] = s.mean.x();
  o->mean[1] = s.mean.y();
  for (int i = 0; i < 3; ++i) {
    o->cov2d[i] = s.cov2d[i];
    o->conic[i] = s.conic[i];
    o->color[i] = s.color[i];
  }
  o->depth = s.depth;
  o->radius = s.radius;
  o->opacity = s.opacity;
  o->clamped = (s.color_clamped[0] ? 1u : 0u) | (s.color_clamped[1] ? 2u : 0u) |
               (s.color_clamped[2] ? 4u : 0u);
}

ProjectedSplat fromProjected(const pxs_projected_splat& o) {
  ProjectedSplat s;
  s.index = o.index;
  s.mean = Vec2f(o.mean[0], o.mean[1]);
  s.cov2d = Vec3f(o.cov2d[0], o.cov2d[1], o.cov2d[2]);
  s.conic = Vec3f(o.conic[0], o.conic[1], o.conic[2]);
  s.depth = o.depth;
  s.radius = o.radius;
  for (int i = 0; i < 3; ++i) {
    s.color[i] = o.color[i];
    s.color_clamped[i] = (o.clamped >> i) & 1u;
  }
  s.opacity = o.opacity;
  return s;
}

void addGradients(const SplatGradients& g, int rest, float* grads, float* screen, int32_t* visible) {
  const size_t N = g.position.size();
  for (size_t i = 0; i < N; ++i) {
    for (int a = 0; a < 3; ++a) {
      grads[(0 + a) * N + i] += g.position[i][a];
      grads[(3 + a) * N + i] += g.log_scale[i][a];
      grads[(11 + a) * N + i] += g.dc[i][a];
    }
    for (int a = 0; a < 4; ++a) grads[(6 + a) * N + i] += g.rotation[i][a];
    grads[10 * N + i] += g.opacity_logit[i];
    for (int k = 0; k < 3 * rest; ++k)
      grads[(14 + k) * N + i] += g.sh_rest[i * static_cast<size_t>(3 * rest) + k];
    screen[i] += g.screen_gradient[i];
    visible[i] += g.visible_count[i];
  }
}

std::vector<SplatTrainingView> toViews(int n_views, const double* K, const int32_t* sizes,
                                       const double* R, const double* t,
                                       const float* const* images) {
  std::vector<SplatTrainingView> views;
  for (int v = 0; v < n_views; ++v) {
    SplatTrainingView tv;
    tv.view = toView(K + 4 * v, sizes[2 * v], sizes[2 * v + 1], R + 9 * v, t + 3 * v);
    const size_t values = static_cast<size_t>(sizes[2 * v]) * sizes[2 * v + 1] * 3;
    tv.image.assign(images[v], images[v] + values);
    views.push_back(std::move(tv));
  }
  return views;
}

struct RefTrainer {
  std::unique_ptr<SplatTrainer> trainer;
  int rest = 0;
};

// A SplatBackend that renders, scores and differentiates a whole batch of
// views per training step instead of the one view the trainer hands it. Each
// view runs the reference's own CpuSplatBackend::renderAndAccumulate
// (SplatTrainer.cpp:104-113) on its own host thread into its own
// SplatGradients; the per-view gradients are then added in view order, which
// is what the additive SplatGradients contract (SplatRaster.h:133-137) gives a
// caller accumulating several views before one optimiser step. The trainer's
// own applyGradients (SplatTrainer.cpp:218-256) then takes the Adam step.
class BatchCpuBackend final : public SplatBackend {
 public:
  BatchCpuBackend(const std::vector<SplatTrainingView>* views, int threads)
      : views_(views), threads_(std::max(1, threads)) {}

  void setBatch(const int32_t* ids, int count) { batch_.assign(ids, ids + count); }

  std::string name() const override { return "cpu-batch"; }

  SplatImage render(const GaussianCloud& cloud, const SplatView& view,
                    const RasterOptions& options) override {
    return renderSplats(cloud, view, options);
  }

  float renderAndAccumulate(const GaussianCloud& cloud, const SplatView&,
                            const RasterOptions& options, const std::vector<float>&,
                            float ssim_weight, SplatGradients* gradients) override {
    const size_t count = batch_.size();
    const int stride = gradients->sh_rest_stride;
    per_view_.resize(count);
    losses_.assign(count, 0.f);
    std::vector<std::thread> pool;
    const int workers = static_cast<int>(std::min<size_t>(count, static_cast<size_t>(threads_)));
    for (int w = 0; w < workers; ++w) {
      pool.emplace_back([&, w] {
        std::unique_ptr<SplatBackend> cpu = makeCpuSplatBackend();
        for (size_t i = static_cast<size_t>(w); i < count; i += static_cast<size_t>(workers)) {
          const SplatTrainingView& v = (*views_)[static_cast<size_t>(batch_[i])];
          per_view_[i].resize(cloud.size(), stride);
          losses_[i] = cpu->renderAndAccumulate(cloud, v.view, options, v.image, ssim_weight,
                                                &per_view_[i]);
        }
      });
    }
    for (std::thread& t : pool) t.join();
    pool.clear();
    // gradients += sum over views, in view order, split by gaussian ranges
    const size_t n = cloud.size();
    const size_t chunk = (n + static_cast<size_t>(threads_) - 1) / static_cast<size_t>(threads_);
    for (int w = 0; w < threads_; ++w) {
      const size_t lo = std::min(n, static_cast<size_t>(w) * chunk);
      const size_t hi = std::min(n, lo + chunk);
      pool.emplace_back([&, lo, hi] {
        for (size_t i = 0; i < count; ++i) {
          const SplatGradients& g = per_view_[i];
          for (size_t k = lo; k < hi; ++k) {
            gradients->position[k] += g.position[k];
            gradients->log_scale[k] += g.log_scale[k];
            gradients->rotation[k] += g.rotation[k];
            gradients->opacity_logit[k] += g.opacity_logit[k];
            for (int c = 0; c < 3; ++c) gradients->dc[k][c] += g.dc[k][c];
            for (int r = 0; r < stride; ++r)
              gradients->sh_rest[k * static_cast<size_t>(stride) + static_cast<size_t>(r)] +=
                  g.sh_rest[k * static_cast<size_t>(stride) + static_cast<size_t>(r)];
            gradients->screen_gradient[k] += g.screen_gradient[k];
            gradients->visible_count[k] += g.visible_count[k];
          }
        }
      });
    }
    for (std::thread& t : pool) t.join();
    float sum = 0.f;
    for (float l : losses_) sum += l;
    return count ? sum / static_cast<float>(count) : 0.f;
  }

 private:
  const std::vector<SplatTrainingView>* views_;
  int threads_;
  std::vector<int32_t> batch_;
  std::vector<SplatGradients> per_view_;
  std::vector<float> losses_;
};

struct RefBatchTrainer {
  std::vector<SplatTrainingView> views;
  BatchCpuBackend* backend = nullptr;  // owned by trainer
  std::unique_ptr<SplatTrainer> trainer;
  int rest = 0;
};

}  // namespace

extern "C" {

void ref_camera(const double* K, int width, int height, const double* R, const double* t,
                pxs_camera* out) {
  // The float values projectSplats derives from a SplatView (SplatRaster.cpp:206-212).
  const SplatView view = toView(K, width, height, R, t);
  const Eigen::Matrix3f W = view.camera_from_world.R.cast<float>();
  const Vec3f tf = view.camera_from_world.t.cast<float>();
  const Vec3f center = view.camera_from_world.center().cast<float>();
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out->R[r * 3 + c] = W(r, c);
  for (int i = 0; i < 3; ++i) {
    out->t[i] = tf[i];
    out->center[i] = center[i];
  }
  const CameraIntrinsics& k = view.intrinsics;
  out->fx = static_cast<float>(k.fx);
  out->fy = static_cast<float>(k.fy);
  out->cx = static_cast<float>(k.cx);
  out->cy = static_cast<float>(k.cy);
  out->tan_half_x = static_cast<float>(0.5 * k.width / k.fx);
  out->tan_half_y = static_cast<float>(0.5 * k.height / k.fy);
  out->width = width;
  out->height = height;
}

int ref_project(const float* params, int n, int rest, int cloud_sh, const double* K, int width,
                int height, const double* R, const double* t, const pxs_raster_options* opt,
                pxs_projected_splat* out) {
  const GaussianCloud cloud = toCloud(params, n, rest, cloud_sh);
  const std::vector<ProjectedSplat> p =
      projectSplats(cloud, toView(K, width, height, R, t), toOptions(opt));
  for (size_t i = 0; i < p.size(); ++i) toProjected(p[i], &out[i]);
  return static_cast<int>(p.size());
}

void ref_rasterize(const pxs_projected_splat* projected, int count, const double* K, int width,
                   int height, const double* R, const double* t, const pxs_raster_options* opt,
                   float* rgb, float* transmittance) {
  std::vector<ProjectedSplat> p;
  p.reserve(static_cast<size_t>(count));
  for (int i = 0; i < count; ++i) p.push_back(fromProjected(projected[i]));
  const SplatImage image = rasterizeSplats(p, toView(K, width, height, R, t), toOptions(opt));
  std::memcpy(rgb, image.rgb.data(), image.rgb.size() * sizeof(float));
  if (transmittance != nullptr) {
    std::memcpy(transmittance, image.transmittance.data(),
                image.transmittance.size() * sizeof(float));
  }
}

void ref_render(const float* params, int n, int rest, int cloud_sh, const double* K, int width,
                int height, const double* R, const double* t, const pxs_raster_options* opt,
                float* rgb, float* transmittance) {
  const GaussianCloud cloud = toCloud(params, n, rest, cloud_sh);
  const SplatImage image =
      renderSplats(cloud, toView(K, width, height, R, t), toOptions(opt));
  std::memcpy(rgb, image.rgb.data(), image.rgb.size() * sizeof(float));
  if (transmittance != nullptr) {
    std::memcpy(transmittance, image.transmittance.data(),
                image.transmittance.size() * sizeof(float));
  }
}

float ref_photometric_loss(const float* rendered, const float* target, int width, int height,
                           float ssim_weight, float* dL_drgb) {
  SplatImage image;
  image.width = width;
  image.height = height;
  const size_t values = static_cast<size_t>(width) * height * 3;
  image.rgb.assign(rendered, rendered + values);
  image.transmittance.assign(values / 3, 0.f);
  std::vector<float> tgt(target, target + values);
  std::vector<float> grad;
  const float loss = photometricLoss(image, tgt, ssim_weight, dL_drgb ? &grad : nullptr);
  if (dL_drgb != nullptr) std::memcpy(dL_drgb, grad.data(), values * sizeof(float));
  return loss;
}

float ref_mean_ssim(const float* rendered, const float* target, int width, int height,
                    float* d_rendered) {
  const size_t values = static_cast<size_t>(width) * height * 3;
  std::vector<float> a(rendered, rendered + values), b(target, target + values), d;
  const float ssim = meanSsim(a, b, width, height, d_rendered ? &d : nullptr);
  if (d_rendered != nullptr) std::memcpy(d_rendered, d.data(), values * sizeof(float));
  return ssim;
}

// rasterizeSplatsBackward after the reference's own projection and forward.
void ref_backward(const float* params, int n, int rest, int cloud_sh, const double* K,
                  int width, int height, const double* R, const double* t,
                  const pxs_raster_options* opt, const float* dL_drgb, float* grads,
                  float* screen, int32_t* visible) {
  const GaussianCloud cloud = toCloud(params, n, rest, cloud_sh);
  const SplatView view = toView(K, width, height, R, t);
  const RasterOptions options = toOptions(opt);
  const std::vector<ProjectedSplat> p = projectSplats(cloud, view, options);
  const SplatImage image = rasterizeSplats(p, view, options);
  const size_t values = static_cast<size_t>(width) * height * 3;
  std::vector<float> dL(dL_drgb, dL_drgb + values);
  SplatGradients g;
  g.resize(cloud.size(), 3 * rest);
  rasterizeSplatsBackward(cloud, view, options, p, image, dL, &g);
  addGradients(g, rest, grads, screen, visible);
}

// CpuSplatBackend::renderAndAccumulate (SplatTrainer.cpp:104-113).
float ref_render_and_accumulate(const float* params, int n, int rest, int cloud_sh,
                                const double* K, int width, int height, const double* R,
                                const double* t, const pxs_raster_options* opt,
                                const float* target, float ssim_weight, float* grads,
                                float* screen, int32_t* visible) {
  const GaussianCloud cloud = toCloud(params, n, rest, cloud_sh);
  const SplatView view = toView(K, width, height, R, t);
  const size_t values = static_cast<size_t>(width) * height * 3;
  std::vector<float> tgt(target, target + values);
  SplatGradients g;
  g.resize(cloud.size(), 3 * rest);
  std::unique_ptr<SplatBackend> backend = makeCpuSplatBackend();
  const float loss =
      backend->renderAndAccumulate(cloud, view, toOptions(opt), tgt, ssim_weight, &g);
  addGradients(g, rest, grads, screen, visible);
  return loss;
}

// renderAndAccumulate's chain (SplatTrainer.cpp:104-113) on a projected list
// the caller supplies, in the caller's order: rasterizeSplats, photometricLoss,
// rasterizeSplatsBackward. projectSplats orders equal depths with the unstable
// std::sort (SplatRaster.cpp:260-261); the parity tests pass its own output
// re-sorted with equal depths by gaussian index, which gives the reference's
// arithmetic under a specified tie order. `rgb` (may be null) gets the image.
float ref_render_and_accumulate_projected(const float* params, int n, int rest, int cloud_sh,
                                          const double* K, int width, int height,
                                          const double* R, const double* t,
                                          const pxs_raster_options* opt,
                                          const pxs_projected_splat* projected, int count,
                                          const float* target, float ssim_weight, float* rgb,
                                          float* grads, float* screen, int32_t* visible) {
  const GaussianCloud cloud = toCloud(params, n, rest, cloud_sh);
  const SplatView view = toView(K, width, height, R, t);
  const RasterOptions options = toOptions(opt);
  std::vector<ProjectedSplat> p;
  p.reserve(static_cast<size_t>(count));
  for (int i = 0; i < count; ++i) p.push_back(fromProjected(projected[i]));
  const SplatImage image = rasterizeSplats(p, view, options);
  const size_t values = static_cast<size_t>(width) * height * 3;
  if (rgb != nullptr) std::memcpy(rgb, image.rgb.data(), values * sizeof(float));
  std::vector<float> tgt(target, target + values), dL;
  const float loss = photometricLoss(image, tgt, ssim_weight, &dL);
  SplatGradients g;
  g.resize(cloud.size(), 3 * rest);
  rasterizeSplatsBackward(cloud, view, options, p, image, dL, &g);
  addGradients(g, rest, grads, screen, visible);
  return loss;
}

// densifyAndPrune (SplatDensify.cpp:28-109). `params` has room for
// config->max_gaussians gaussians; output stride is the new count.
int ref_densify(float* params, int n, int rest, const float* screen, const int32_t* visible,
                const pxs_train_config* config, float extent, int iteration, uint32_t* rng,
                int32_t* source, int32_t* cloned, int32_t* split, int32_t* pruned) {
  GaussianCloud cloud = toCloud(params, n, rest, 3);
  SplatDensifyStats stats;
  stats.screen_gradient.assign(screen, screen + n);
  stats.visible_count.assign(visible, visible + n);
  const SplatDensifyResult r =
      densifyAndPrune(&cloud, stats, toConfig(config), extent, iteration, rng);
  for (size_t i = 0; i < r.source_index.size(); ++i) source[i] = r.source_index[i];
  *cloned = r.cloned;
  *split = r.split;
  *pruned = r.pruned;
  return fromCloud(cloud, rest, params, config->max_gaussians);
}

// ------------------------------------------------------------- the trainer

void* ref_trainer_create(const float* params, int n, int rest, int cloud_sh, int n_views,
                         const double* K, const int32_t* sizes, const double* R,
                         const double* t, const float* const* images,
                         const pxs_train_config* config) {
  auto* holder = new RefTrainer;
  holder->rest = rest;
  holder->trainer = std::make_unique<SplatTrainer>(
      toCloud(params, n, rest, cloud_sh), toViews(n_views, K, sizes, R, t, images),
      toConfig(config));
  return holder;
}

void ref_trainer_destroy(void* handle) { delete static_cast<RefTrainer*>(handle); }

// ------------------------------------------- the batched reference trainer
//
// The reference's SplatTrainer (its schedule and its Adam, applyGradients) with
// BatchCpuBackend: each step renders, scores and differentiates the views set
// by ref_batch_trainer_step on up to `threads` host threads, adds their
// gradients, and takes one Adam step. This is the reference's CPU code for a
// many-views-per-step training step.
void* ref_batch_trainer_create(const float* params, int n, int rest, int cloud_sh,
                               int n_views, const double* K, const int32_t* sizes,
                               const double* R, const double* t, const float* const* images,
                               const pxs_train_config* config, int threads) {
  auto* holder = new RefBatchTrainer;
  holder->rest = rest;
  holder->views = toViews(n_views, K, sizes, R, t, images);
  auto backend = std::make_unique<BatchCpuBackend>(&holder->views, threads);
  holder->backend = backend.get();
  // The trainer gets every camera (its scene extent, cameraExtent, comes from
  // them) without the images; the view it picks each step is ignored by the
  // backend, which renders the batch.
  std::vector<SplatTrainingView> cameras;
  for (const SplatTrainingView& v : holder->views) {
    SplatTrainingView c;
    c.view = v.view;
    cameras.push_back(std::move(c));
  }
  holder->trainer = std::make_unique<SplatTrainer>(toCloud(params, n, rest, cloud_sh),
                                                   std::move(cameras), toConfig(config),
                                                   std::move(backend));
  return holder;
}

// One training step over the `count` views `ids`; returns the trainer's
// step() result and the mean loss over the batch.
int ref_batch_trainer_step(void* handle, int count, const int32_t* ids, float* loss) {
  auto* h = static_cast<RefBatchTrainer*>(handle);
  h->backend->setBatch(ids, count);
  const bool stepped = h->trainer->step();
  if (loss != nullptr) *loss = h->trainer->lastLoss();
  return stepped ? 1 : 0;
}

int ref_batch_trainer_download(void* handle, float* params, int capacity) {
  auto* h = static_cast<RefBatchTrainer*>(handle);
  return fromCloud(h->trainer->cloud(), h->rest, params, capacity);
}

void ref_batch_trainer_destroy(void* handle) { delete static_cast<RefBatchTrainer*>(handle); }

// The benchmark clouds drawn with the reference's own generator,
// parallax::testing::Rng (SyntheticScene.h:80-107): per gaussian, in this
// order, position U[-1,1]^3, log sigma log_scale_mean + 0.5 N(0,1) per axis, a
// quaternion normalise(N(0,1)^4) (w, x, y, z), opacity logit N(0,1), dc from an
// RGB value 0.5 + 0.1 N(0,1) per channel, sh_rest 0.1 N(0,1). Component-major
// output like every array of pxs.h.
int ref_synthetic_cloud(uint64_t seed, int count, int rest, float log_scale_mean,
                        float* params) {
  if (count < 0 || params == nullptr) return -1;
  parallax::testing::Rng rng(seed);
  const size_t N = static_cast<size_t>(count);
  const double c0 = 0.28209479177387814;
  for (size_t g = 0; g < N; ++g) {
    for (int a = 0; a < 3; ++a) params[(0 + a) * N + g] = static_cast<float>(rng.uniform(-1.0, 1.0));
    for (int a = 0; a < 3; ++a)
      params[(3 + a) * N + g] = static_cast<float>(log_scale_mean + 0.5 * rng.normal());
    double q[4], norm = 0.0;
    for (double& v : q) {
      v = rng.normal();
      norm += v * v;
    }
    norm = std::sqrt(norm);
    if (norm < 1e-9) {
      q[0] = 1.0;
      q[1] = q[2] = q[3] = 0.0;
      norm = 1.0;
    }
    for (int a = 0; a < 4; ++a) params[(6 + a) * N + g] = static_cast<float>(q[a] / norm);
    params[10 * N + g] = static_cast<float>(rng.normal());
    for (int c = 0; c < 3; ++c) {
      const double rgb = 0.5 + 0.1 * rng.normal();
      params[(11 + c) * N + g] = static_cast<float>((rgb - 0.5) / c0);
    }
    for (int k = 0; k < 3 * rest; ++k)
      params[(14 + k) * N + g] = static_cast<float>(0.1 * rng.normal());
  }
  return 0;
}

int ref_trainer_step(void* handle) { return static_cast<RefTrainer*>(handle)->trainer->step(); }

// Runs SplatTrainer::train with a callback that cancels once `cancel_at` is
// reached (0 never cancels). Returns train()'s result; `seen` gets the last
// iteration the callback saw.
int ref_trainer_train(void* handle, int cancel_at, int* seen) {
  int last = 0;
  const bool done =
      static_cast<RefTrainer*>(handle)->trainer->train([&](const SplatTrainingProgress& p) {
        last = p.iteration;
        return cancel_at <= 0 || p.iteration < cancel_at;
      });
  if (seen != nullptr) *seen = last;
  return done ? 1 : 0;
}

void ref_trainer_state(void* handle, int* iteration, int* count, float* last_loss,
                       float* smoothed, float* extent, int* sh_degree) {
  const SplatTrainer& tr = *static_cast<RefTrainer*>(handle)->trainer;
  *iteration = tr.iteration();
  *count = static_cast<int>(tr.cloud().size());
  *last_loss = tr.lastLoss();
  *smoothed = tr.smoothedLoss();
  *extent = tr.sceneExtent();
  *sh_degree = tr.shDegreeInUse();
}

int ref_trainer_download(void* handle, float* params, int capacity) {
  auto* h = static_cast<RefTrainer*>(handle);
  return fromCloud(h->trainer->cloud(), h->rest, params, capacity);
}

int ref_trainer_finish(void* handle, float* params, int capacity, int* sh_degree) {
  auto* h = static_cast<RefTrainer*>(handle);
  const GaussianCloud cloud = h->trainer->finish();
  if (sh_degree != nullptr) *sh_degree = cloud.sh_degree;
  return fromCloud(cloud, h->rest, params, capacity);
}

// writeGaussianPly / writeSplat / writeSpz (GaussianCloud.cpp:259-306, 414-443,
// 493-550) of the cloud into `path`; format 0, 1, 2. Returns the writer's result.
int ref_write_cloud(const float* params, int n, int rest, int cloud_sh, int format,
                    int fractional_bits, const char* path) {
  const GaussianCloud cloud = toCloud(params, n, rest, cloud_sh);
  if (format == 0) return writeGaussianPly(path, cloud) ? 1 : 0;
  if (format == 1) return writeSplat(path, cloud) ? 1 : 0;
  return writeSpz(path, cloud, fractional_bits) ? 1 : 0;
}

// downscaleToWidth (ImageIo.cpp:300-337); returns the output width and height
// through w / h and writes the bytes when `out` is given.
// readGaussianPly and GaussianCloud::isValid (GaussianCloud.cpp) on a file:
// the count, whether it is valid, and the least opacity. Returns 1 when read.
int ref_read_ply_stats(const char* path, int* count, int* valid, float* min_opacity,
                       char* reason, int reason_len) {
  GaussianCloud cloud;
  std::string error;
  if (!readGaussianPly(path, &cloud, &error)) {
    if (reason != nullptr && reason_len > 0) {
      std::strncpy(reason, error.c_str(), static_cast<size_t>(reason_len) - 1);
      reason[reason_len - 1] = '\0';
    }
    return 0;
  }
  *count = static_cast<int>(cloud.size());
  std::string why;
  *valid = cloud.isValid(&why) ? 1 : 0;
  float least = 1.f;
  for (const Gaussian& g : cloud.gaussians) least = std::min(least, gaussianOpacity(g));
  *min_opacity = least;
  if (reason != nullptr && reason_len > 0) {
    std::strncpy(reason, why.c_str(), static_cast<size_t>(reason_len) - 1);
    reason[reason_len - 1] = '\0';
  }
  return 1;
}

void ref_downscale(const uint8_t* rgb, int width, int height, int target_width, uint8_t* out,
                   int* w, int* h) {
  ColorBuffer image(width, height);
  std::memcpy(image.pixels.data(), rgb, static_cast<size_t>(width) * height * 3);
  const ColorBuffer scaled = downscaleToWidth(image, target_width);
  *w = scaled.width;
  *h = scaled.height;
  if (out != nullptr) std::memcpy(out, scaled.pixels.data(), scaled.pixels.size());
}

// initializeFromPointCloud (GaussianCloud.cpp:199-257) into `params`
// (component-major); returns the gaussian count.
int ref_initialize_from_points(const float* points, const uint8_t* colors, int n, int sh_degree,
                               float initial_opacity, float* params) {
  std::vector<Vec3f> pts(static_cast<size_t>(n));
  std::vector<std::array<uint8_t, 3>> cols;
  for (int i = 0; i < n; ++i) {
    pts[static_cast<size_t>(i)] = Vec3f(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
    if (colors != nullptr) cols.push_back({colors[3 * i], colors[3 * i + 1], colors[3 * i + 2]});
  }
  const GaussianCloud cloud = initializeFromPointCloud(pts, cols, sh_degree, initial_opacity);
  const int rest = shRestPerChannel(cloud.sh_degree);
  return fromCloud(cloud, rest, params, n);
}

int ref_config_validate(const pxs_train_config* config, char* reason, int len) {
  const std::string why = toConfig(config).validate();
  if (reason != nullptr && len > 0) {
    std::strncpy(reason, why.c_str(), static_cast<size_t>(len) - 1);
    reason[len - 1] = '\0';
  }
  return why.empty() ? 0 : 1;
}

void ref_config_defaults(pxs_train_config* c) {
  const SplatTrainingConfig d;
  c->iterations = d.iterations;
  c->position_lr_initial = d.position_lr_initial;
  c->position_lr_final = d.position_lr_final;
  c->dc_lr = d.dc_lr;
  c->sh_rest_lr_divider = d.sh_rest_lr_divider;
  c->opacity_lr = d.opacity_lr;
  c->scale_lr = d.scale_lr;
  c->rotation_lr = d.rotation_lr;
  c->adam_beta1 = d.adam_beta1;
  c->adam_beta2 = d.adam_beta2;
  c->adam_epsilon = d.adam_epsilon;
  c->ssim_weight = d.ssim_weight;
  c->sh_degree = d.sh_degree;
  c->sh_increase_interval = d.sh_increase_interval;
  c->densify_from_iteration = d.densify_from_iteration;
  c->densify_until_iteration = d.densify_until_iteration;
  c->densify_interval = d.densify_interval;
  c->densify_grad_threshold = d.densify_grad_threshold;
  c->percent_dense = d.percent_dense;
  c->split_scale_divider = d.split_scale_divider;
  c->opacity_reset_interval = d.opacity_reset_interval;
  c->opacity_reset_value = d.opacity_reset_value;
  c->prune_opacity = d.prune_opacity;
  c->prune_scale_fraction = d.prune_scale_fraction;
  c->max_gaussians = d.max_gaussians;
  c->seed = d.seed;
}

// The training and raster settings of the multi-view benchmark step over the
// reference's defaults (SplatTrainingConfig{}, RasterOptions{}): `sh_degree`
// from the start, no densification, no opacity reset, `iterations` for the
// position learning-rate schedule. Sizes let a caller allocate the structs
// without declaring their layout.
int ref_sizeof_train_config() { return static_cast<int>(sizeof(pxs_train_config)); }
int ref_sizeof_raster_options() { return static_cast<int>(sizeof(pxs_raster_options)); }

void ref_bench_settings(pxs_train_config* c, pxs_raster_options* o, int sh_degree,
                        int iterations, int max_gaussians) {
  ref_config_defaults(c);
  c->iterations = iterations;
  c->sh_degree = sh_degree;
  c->sh_increase_interval = 0;
  c->densify_from_iteration = 1000000000;
  c->densify_until_iteration = 1000000000;
  c->opacity_reset_interval = 0;
  c->max_gaussians = max_gaussians;
  const RasterOptions d;
  for (int i = 0; i < 3; ++i) o->background[i] = d.background[i];
  o->sh_degree = sh_degree;
  o->min_alpha = d.min_alpha;
  o->transmittance_cutoff = d.transmittance_cutoff;
  o->screen_dilation = d.screen_dilation;
}

#ifdef PXREF_SHIM
// ------------------------------------------- the drop-in shim, in the engine
// Built into oracle/_ref/libpxshim.so together with
// parallax_b200/shim/CudaSplatTrainer.cpp and linked against libpxs.so: the
// reference's own SplatTrainer and the engine signatures, run on the GPU core.

int ref_shim_availability(int32_t* available, char* name, int name_len, char* reason,
                          int reason_len) {
  const SplatGpuAvailability a = splatGpuAvailability();
  *available = a.available ? 1 : 0;
  if (name != nullptr && name_len > 0) {
    std::strncpy(name, a.device_name.c_str(), static_cast<size_t>(name_len) - 1);
    name[name_len - 1] = '\0';
  }
  if (reason != nullptr && reason_len > 0) {
    std::strncpy(reason, a.reason.c_str(), static_cast<size_t>(reason_len) - 1);
    reason[reason_len - 1] = '\0';
  }
  return 0;
}

// SplatBackend::renderAndAccumulate of makeCudaSplatBackend(), same arguments
// as ref_render_and_accumulate. Returns NaN when the backend fails.
float ref_shim_render_and_accumulate(const float* params, int n, int rest, int cloud_sh,
                                     const double* K, int width, int height, const double* R,
                                     const double* t, const pxs_raster_options* opt,
                                     const float* target, float ssim_weight, float* grads,
                                     float* screen, int32_t* visible) {
  const GaussianCloud cloud = toCloud(params, n, rest, cloud_sh);
  const SplatView view = toView(K, width, height, R, t);
  const size_t values = static_cast<size_t>(width) * height * 3;
  std::vector<float> tgt(target, target + values);
  SplatGradients g;  // left empty: the backend sizes it, as the CPU one does
  std::unique_ptr<SplatBackend> backend = makeCudaSplatBackend(0);
  if (backend == nullptr) return std::numeric_limits<float>::quiet_NaN();
  try {
    const float loss =
        backend->renderAndAccumulate(cloud, view, toOptions(opt), tgt, ssim_weight, &g);
    addGradients(g, rest, grads, screen, visible);
    return loss;
  } catch (const std::exception&) {
    return std::numeric_limits<float>::quiet_NaN();
  }
}

// The reference's SplatTrainer driving makeCudaSplatBackend(); the other
// ref_trainer_* calls work on the handle.
void* ref_shim_trainer_create(const float* params, int n, int rest, int cloud_sh, int n_views,
                              const double* K, const int32_t* sizes, const double* R,
                              const double* t, const float* const* images,
                              const pxs_train_config* config) {
  std::unique_ptr<SplatBackend> backend = makeCudaSplatBackend(0);
  if (backend == nullptr) return nullptr;
  auto* holder = new RefTrainer;
  holder->rest = rest;
  holder->trainer = std::make_unique<SplatTrainer>(
      toCloud(params, n, rest, cloud_sh), toViews(n_views, K, sizes, R, t, images),
      toConfig(config), std::move(backend));
  return holder;
}

// trainSplatsOnGpu through the engine signature. `params` has room for
// max(n, config->max_gaussians) gaussians; on success it receives the trained
// cloud with stride *count. The callback cancels once `cancel_at` is reached
// (0 never). Returns 1 on success, 0 with the message in `error`.
int ref_shim_train_splats_on_gpu(float* params, int n, int rest, int cloud_sh, int n_views,
                                 const double* K, const int32_t* sizes, const double* R,
                                 const double* t, const float* const* images,
                                 const pxs_train_config* config, int cancel_at, int* count,
                                 int* sh_degree, int* last_seen, char* error, int error_len) {
  GaussianCloud cloud = toCloud(params, n, rest, cloud_sh);
  std::string why;
  int seen = 0;
  const SplatTrainingCallback callback = [&](const SplatTrainingProgress& p) {
    seen = p.iteration;
    return cancel_at <= 0 || p.iteration < cancel_at;
  };
  const bool ok = trainSplatsOnGpu(&cloud, toViews(n_views, K, sizes, R, t, images),
                                   toConfig(config), callback, &why);
  if (last_seen != nullptr) *last_seen = seen;
  if (error != nullptr && error_len > 0) {
    std::strncpy(error, why.c_str(), static_cast<size_t>(error_len) - 1);
    error[error_len - 1] = '\0';
  }
  if (!ok) return 0;
  *count = fromCloud(cloud, rest, params, std::max(n, config->max_gaussians));
  *sh_degree = cloud.sh_degree;
  return 1;
}

// The splat stage of the reference pipeline (Pipeline::Impl::runSplatTraining,
// Pipeline.cpp:1844-2009) from the coloured point cloud and the posed frames
// on, as a test driver: the seed budget and point stride (:1858-1874), the
// seed by initializeFromPointCloud, the training views spread over the frames
// and downscaled by downscaleToWidth then divided by 255 (:1888-1917), the
// training config derived from the stage's settings (:1922-1929), the
// progress callback with the cancel token and the time budget (:1931-1957),
// trainSplatsOnGpu -- here the CUDA shim -- with the CPU trainer as the
// fallback (:1959-1991), and the outcome note (:1993-2009). The pipeline's
// checkpoint files and the rest of its stages are not part of it; the caller
// writes the field with the reference's writer and reads it back.
// settings: iterations, max_gaussians, sh_degree, image_width, max_views,
// time_budget_ms (0: none), cancel_at (the iteration at which the cancel token
// is set; 0: never). Frames are 8-bit RGB at sizes[2f], sizes[2f+1] with
// intrinsics K[4f..] for that size. Returns 1 for a successful outcome.
int ref_shim_pipeline_splat_stage(const float* points, const uint8_t* colors, int n_points,
                                  int n_frames, const double* K, const int32_t* sizes,
                                  const double* R, const double* t,
                                  const uint8_t* const* frames, const int32_t* settings,
                                  float* params_out, int capacity, int32_t* out_count,
                                  int32_t* out_rest, int32_t* out_sh, int32_t* cancelled,
                                  char* backend, int backend_len, char* message,
                                  int message_len) {
  const int iterations = settings[0], max_gaussians = settings[1], sh = settings[2];
  const int image_width = settings[3], max_views = settings[4];
  const long long budget_ms = settings[5];
  const int cancel_at = settings[6];
  bool token = false;  // the cancel token
  std::string used;
  auto outcome = [&](bool success, bool was_cancelled, const std::string& note) {
    *cancelled = was_cancelled ? 1 : 0;
    if (message != nullptr && message_len > 0) {
      std::strncpy(message, note.c_str(), static_cast<size_t>(message_len) - 1);
      message[message_len - 1] = '\0';
    }
    if (backend != nullptr && backend_len > 0) {
      std::strncpy(backend, used.c_str(), static_cast<size_t>(backend_len) - 1);
      backend[backend_len - 1] = '\0';
    }
    return success ? 1 : 0;
  };

  // seed from at most a quarter of the budget: every k-th point
  std::vector<Vec3f> pts;
  std::vector<std::array<uint8_t, 3>> cols;
  const size_t n = static_cast<size_t>(std::max(n_points, 0));
  const size_t seed_budget = std::max<size_t>(1, static_cast<size_t>(max_gaussians) / 4);
  const size_t stride = n > seed_budget ? (n + seed_budget - 1) / seed_budget : 1;
  for (size_t i = 0; i < n; i += stride) {
    pts.emplace_back(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
    cols.push_back({colors[3 * i], colors[3 * i + 1], colors[3 * i + 2]});
  }
  if (pts.empty()) return outcome(true, false, "no point cloud to seed the splat field from");
  GaussianCloud cloud = initializeFromPointCloud(pts, cols, sh);
  if (cloud.empty()) return outcome(false, false, "the point cloud produced no gaussians");

  // training views spread evenly over the frames
  const size_t view_budget = std::min<size_t>(static_cast<size_t>(n_frames),
                                              static_cast<size_t>(std::max(4, max_views)));
  std::vector<SplatTrainingView> views;
  for (size_t v = 0; v < view_budget; ++v) {
    const size_t f = view_budget == 1
                         ? 0
                         : static_cast<size_t>(static_cast<double>(v) * (n_frames - 1) /
                                               (view_budget - 1));
    ColorBuffer image;
    image.width = sizes[2 * f];
    image.height = sizes[2 * f + 1];
    image.pixels.assign(frames[f],
                        frames[f] + static_cast<size_t>(image.width) * image.height * 3);
    const ColorBuffer scaled = downscaleToWidth(image, image_width);
    SplatTrainingView tv;
    tv.view = toView(K + 4 * f, image.width, image.height, R + 9 * f, t + 3 * f);
    tv.view.intrinsics = tv.view.intrinsics.scaledTo(scaled.width, scaled.height);
    tv.image.resize(static_cast<size_t>(scaled.width) * scaled.height * 3);
    for (size_t p = 0; p < tv.image.size(); ++p)
      tv.image[p] = static_cast<float>(scaled.pixels[p]) / 255.f;
    views.push_back(std::move(tv));
  }
  if (views.size() < 2)
    return outcome(false, false, "at least two posed views are needed to train splats");

  SplatTrainingConfig tc;
  tc.iterations = std::max(1, iterations);
  tc.sh_degree = sh;
  tc.max_gaussians = max_gaussians;
  tc.densify_until_iteration = tc.iterations / 2;
  tc.opacity_reset_interval = std::max(1, tc.iterations / 3);
  tc.sh_increase_interval = std::max(1, tc.iterations / 8);
  const std::string invalid = tc.validate();
  if (!invalid.empty()) return outcome(false, false, invalid);

  bool was_cancelled = false, out_of_time = false;
  int done = 0;
  const auto started = std::chrono::steady_clock::now();
  const SplatTrainingCallback callback = [&](const SplatTrainingProgress& p) {
    if (cancel_at > 0 && p.iteration >= cancel_at) token = true;
    if (token) {
      was_cancelled = true;
      return false;
    }
    done = p.iteration;
    if (budget_ms > 0) {
      const auto elapsed = std::chrono::duration_cast<std::chrono::milliseconds>(
                               std::chrono::steady_clock::now() - started)
                               .count();
      if (elapsed >= budget_ms) {
        out_of_time = true;
        return false;
      }
    }
    return true;
  };

  std::string gpu_error;
  if (trainSplatsOnGpu(&cloud, views, tc, callback, &gpu_error)) {
    used = "gpu";
  } else if (was_cancelled) {
    return outcome(false, true, "cancelled");
  } else if (out_of_time) {
    used = "gpu";
  } else {
    // no usable device: the reduced CPU run
    SplatTrainingConfig reduced = tc;
    reduced.iterations = std::max(1, tc.iterations / 5);
    reduced.max_gaussians = std::min(tc.max_gaussians, 60000);
    reduced.densify_until_iteration = reduced.iterations / 2;
    reduced.opacity_reset_interval = std::max(1, reduced.iterations / 3);
    reduced.sh_increase_interval = std::max(1, reduced.iterations / 8);
    reduced.sh_degree = std::min(1, sh);
    SplatTrainer trainer(std::move(cloud), std::move(views), reduced);
    if (!trainer.train(callback) && was_cancelled) return outcome(false, true, "cancelled");
    cloud = trainer.finish();
    used = "cpu";
  }
  if (token) return outcome(false, true, "cancelled");
  const int rest = cloud.gaussians.empty() ? 0 : static_cast<int>(cloud.gaussians[0].sh_rest.size()) / 3;
  *out_rest = rest;
  *out_sh = cloud.sh_degree;
  *out_count = fromCloud(cloud, rest, params_out, capacity);
  std::string note = std::to_string(cloud.size()) + " gaussians (" + used + ")";
  if (out_of_time)
    note += ", stopped at iteration " + std::to_string(done) + " when the time budget ran out";
  return outcome(true, false, note);
}
#endif  // PXREF_SHIM

}  // extern "C"
