// CudaSplatTrainer.cpp -- parallax::trainSplatsOnGpu, splatGpuAvailability and
// makeCudaSplatBackend over the C ABI of include/pxs.h.
//
// Link this object (and libpxs.so) ahead of the engine's static library: the
// archive member that holds the Vulkan trainer's host stub
// (src/splat/vulkan/VulkanSplatTrainer.cpp:5-22) is then not pulled in,
// because both of its symbols are already defined here.
//
// Conversions only: the engine's array-of-structs GaussianCloud
// (GaussianCloud.h:41-71) <-> the core's component-major parameter array,
// SplatView <-> pxs_camera (through pxs_camera_from_pose, which applies the
// engine's own float casts), SplatTrainingConfig <-> pxs_train_config (the
// same fields), SplatGradients += the core's gradient array.
#include "CudaSplatTrainer.h"

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "pxs.h"

namespace parallax {
namespace {

int restPerChannel(const GaussianCloud& cloud) {
  return cloud.gaussians.empty() ? 0 : static_cast<int>(cloud.gaussians.front().sh_rest.size()) / 3;
}

// Component-major with N = cloud.size() gaussians per component, in a buffer
// with room for P x max(N, room) floats.
std::vector<float> toParams(const GaussianCloud& cloud, int rest, size_t room) {
  const size_t N = cloud.size();
  const size_t P = static_cast<size_t>(PXS_PARAM_COUNT(rest));
  const size_t stride = N;
  std::vector<float> p(P * std::max(N, room), 0.f);
  for (size_t g = 0; g < N; ++g) {
    const Gaussian& G = cloud.gaussians[g];
    for (int a = 0; a < 3; ++a) {
      p[(PXS_C_POSITION + a) * stride + g] = G.position[a];
      p[(PXS_C_LOG_SCALE + a) * stride + g] = G.log_scale[a];
      p[(PXS_C_DC + a) * stride + g] = G.dc[a];
    }
    p[(PXS_C_ROTATION + 0) * stride + g] = G.rotation.w();
    p[(PXS_C_ROTATION + 1) * stride + g] = G.rotation.x();
    p[(PXS_C_ROTATION + 2) * stride + g] = G.rotation.y();
    p[(PXS_C_ROTATION + 3) * stride + g] = G.rotation.z();
    p[PXS_C_OPACITY * stride + g] = G.opacity_logit;
    for (int k = 0; k < 3 * rest; ++k) p[(PXS_C_SH_REST + k) * stride + g] = G.sh_rest[k];
  }
  return p;
}

// Component-major `p` with `stride` gaussians per component, `count` used.
void fromParams(const std::vector<float>& p, size_t stride, size_t count, int rest,
                GaussianCloud* cloud) {
  cloud->gaussians.resize(count);
  for (size_t g = 0; g < count; ++g) {
    Gaussian& G = cloud->gaussians[g];
    for (int a = 0; a < 3; ++a) {
      G.position[a] = p[(PXS_C_POSITION + a) * stride + g];
      G.log_scale[a] = p[(PXS_C_LOG_SCALE + a) * stride + g];
      G.dc[a] = p[(PXS_C_DC + a) * stride + g];
    }
    G.rotation = Eigen::Quaternionf(
        p[(PXS_C_ROTATION + 0) * stride + g], p[(PXS_C_ROTATION + 1) * stride + g],
        p[(PXS_C_ROTATION + 2) * stride + g], p[(PXS_C_ROTATION + 3) * stride + g]);
    G.opacity_logit = p[PXS_C_OPACITY * stride + g];
    G.sh_rest.resize(static_cast<size_t>(3 * rest));
    for (int k = 0; k < 3 * rest; ++k) G.sh_rest[k] = p[(PXS_C_SH_REST + k) * stride + g];
  }
}

pxs_camera toCamera(const SplatView& view) {
  const CameraIntrinsics& k = view.intrinsics;
  const double intrinsics[4] = {k.fx, k.fy, k.cx, k.cy};
  double R[9], t[3];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) R[r * 3 + c] = view.camera_from_world.R(r, c);
    t[r] = view.camera_from_world.t[r];
  }
  pxs_camera camera;
  pxs_camera_from_pose(intrinsics, k.width, k.height, R, t, &camera);
  return camera;
}

pxs_raster_options toOptions(const RasterOptions& o) {
  pxs_raster_options r;
  for (int c = 0; c < 3; ++c) r.background[c] = o.background[c];
  r.sh_degree = o.sh_degree;
  r.min_alpha = o.min_alpha;
  r.transmittance_cutoff = o.transmittance_cutoff;
  r.screen_dilation = o.screen_dilation;
  return r;
}

pxs_train_config toConfig(const SplatTrainingConfig& c) {
  pxs_train_config r;
  pxs_train_config_defaults(&r);
  r.iterations = c.iterations;
  r.position_lr_initial = c.position_lr_initial;
  r.position_lr_final = c.position_lr_final;
  r.dc_lr = c.dc_lr;
  r.sh_rest_lr_divider = c.sh_rest_lr_divider;
  r.opacity_lr = c.opacity_lr;
  r.scale_lr = c.scale_lr;
  r.rotation_lr = c.rotation_lr;
  r.adam_beta1 = c.adam_beta1;
  r.adam_beta2 = c.adam_beta2;
  r.adam_epsilon = c.adam_epsilon;
  r.ssim_weight = c.ssim_weight;
  r.sh_degree = c.sh_degree;
  r.sh_increase_interval = c.sh_increase_interval;
  r.densify_from_iteration = c.densify_from_iteration;
  r.densify_until_iteration = c.densify_until_iteration;
  r.densify_interval = c.densify_interval;
  r.densify_grad_threshold = c.densify_grad_threshold;
  r.percent_dense = c.percent_dense;
  r.split_scale_divider = c.split_scale_divider;
  r.opacity_reset_interval = c.opacity_reset_interval;
  r.opacity_reset_value = c.opacity_reset_value;
  r.prune_opacity = c.prune_opacity;
  r.prune_scale_fraction = c.prune_scale_fraction;
  r.max_gaussians = c.max_gaussians;
  r.seed = c.seed;
  return r;
}

int progressTrampoline(const pxs_progress* p, void* user) {
  const SplatTrainingCallback& callback = *static_cast<const SplatTrainingCallback*>(user);
  SplatTrainingProgress progress;
  progress.iteration = p->iteration;
  progress.total_iterations = p->total_iterations;
  progress.gaussian_count = p->gaussian_count;
  progress.loss = p->loss;
  progress.smoothed_loss = p->smoothed_loss;
  return callback(progress) ? 1 : 0;
}

class CudaSplatBackend final : public SplatBackend {
 public:
  explicit CudaSplatBackend(pxs_context* context) : context_(context) {}
  ~CudaSplatBackend() override { pxs_context_destroy(context_); }

  std::string name() const override { return "cuda"; }

  float renderAndAccumulate(const GaussianCloud& cloud, const SplatView& view,
                            const RasterOptions& options, const std::vector<float>& target,
                            float ssim_weight, SplatGradients* gradients) override {
    const int rest = restPerChannel(cloud);
    const size_t N = cloud.size();
    if (gradients->position.size() != N) gradients->resize(N, 3 * rest);
    std::vector<float> params = toParams(cloud, rest, N);
    pxs_cloud c{params.data(), static_cast<int32_t>(N), rest, cloud.sh_degree};
    const pxs_camera camera = toCamera(view);
    const pxs_raster_options o = toOptions(options);
    std::vector<float> g(params.size(), 0.f), screen(N, 0.f);
    std::vector<int32_t> visible(N, 0);
    pxs_gradients grads{g.data(), screen.data(), visible.data()};
    float loss = 0.f;
    check(pxs_render_and_accumulate(context_, &c, &camera, &o, target.data(), ssim_weight,
                                    &grads, &loss));
    for (size_t i = 0; i < N; ++i) {
      for (int a = 0; a < 3; ++a) {
        gradients->position[i][a] += g[(PXS_C_POSITION + a) * N + i];
        gradients->log_scale[i][a] += g[(PXS_C_LOG_SCALE + a) * N + i];
        gradients->dc[i][a] += g[(PXS_C_DC + a) * N + i];
      }
      for (int a = 0; a < 4; ++a) gradients->rotation[i][a] += g[(PXS_C_ROTATION + a) * N + i];
      gradients->opacity_logit[i] += g[PXS_C_OPACITY * N + i];
      for (int k = 0; k < 3 * rest; ++k)
        gradients->sh_rest[i * static_cast<size_t>(3 * rest) + k] += g[(PXS_C_SH_REST + k) * N + i];
      gradients->screen_gradient[i] += screen[i];
      gradients->visible_count[i] += visible[i];
    }
    return loss;
  }

  SplatImage render(const GaussianCloud& cloud, const SplatView& view,
                    const RasterOptions& options) override {
    const int rest = restPerChannel(cloud);
    std::vector<float> params = toParams(cloud, rest, cloud.size());
    pxs_cloud c{params.data(), static_cast<int32_t>(cloud.size()), rest, cloud.sh_degree};
    const pxs_camera camera = toCamera(view);
    const pxs_raster_options o = toOptions(options);
    SplatImage image;
    image.width = view.intrinsics.width;
    image.height = view.intrinsics.height;
    const size_t pixels = static_cast<size_t>(image.width) * static_cast<size_t>(image.height);
    image.rgb.assign(pixels * 3, 0.f);
    image.transmittance.assign(pixels, 1.f);
    check(pxs_render(context_, &c, &camera, &o, image.rgb.data(), image.transmittance.data()));
    return image;
  }

 private:
  void check(int status) const {
    if (status != PXS_OK) throw std::runtime_error(pxs_context_last_error(context_));
  }
  pxs_context* context_;
};

}  // namespace

SplatGpuAvailability splatGpuAvailability() {
  SplatGpuAvailability availability;
  int32_t available = 0;
  char name[256] = {0};
  char reason[512] = {0};
  pxs_gpu_availability(&available, name, sizeof(name), reason, sizeof(reason));
  availability.available = available != 0;
  availability.device_name = name;
  availability.reason = reason;
  return availability;
}

bool trainSplatsOnGpu(GaussianCloud* cloud, const std::vector<SplatTrainingView>& views,
                      const SplatTrainingConfig& config, const SplatTrainingCallback& callback,
                      std::string* error) {
  if (cloud == nullptr) {
    if (error != nullptr) *error = "no cloud to train";
    return false;
  }
  const int rest = restPerChannel(*cloud);
  const size_t room = std::max(cloud->size(), static_cast<size_t>(std::max(config.max_gaussians, 0)));
  std::vector<float> params = toParams(*cloud, rest, room);
  pxs_cloud c{params.data(), static_cast<int32_t>(cloud->size()), rest, cloud->sh_degree};
  std::vector<pxs_camera> cameras;
  std::vector<const float*> images;
  cameras.reserve(views.size());
  images.reserve(views.size());
  for (const SplatTrainingView& v : views) {
    cameras.push_back(toCamera(v.view));
    images.push_back(v.image.data());
  }
  const pxs_train_config cfg = toConfig(config);
  char message[512] = {0};
  const int status = pxs_train_splats(
      &c, cameras.data(), images.data(), static_cast<int32_t>(views.size()), &cfg,
      callback ? progressTrampoline : nullptr,
      callback ? const_cast<SplatTrainingCallback*>(&callback) : nullptr, message,
      sizeof(message));
  if (status != PXS_OK) {
    if (error != nullptr) *error = message;
    return false;
  }
  // pxs_train_splats writes the finished cloud (pruned, sorted by opacity)
  // back component-major with c.count gaussians per component.
  fromParams(params, static_cast<size_t>(c.count), static_cast<size_t>(c.count), rest, cloud);
  cloud->sh_degree = config.sh_degree;
  return true;
}

std::unique_ptr<SplatBackend> makeCudaSplatBackend(int device) {
  pxs_context* context = nullptr;
  if (pxs_context_create(device, &context) != PXS_OK) {
    pxs_context_destroy(context);
    return nullptr;
  }
  return std::unique_ptr<SplatBackend>(new CudaSplatBackend(context));
}

}  // namespace parallax
