// api.cpp -- the C ABI (include/pxs.h): contexts, the stateless rasteriser
// entry points on host and device buffers, and the host helpers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "densify.h"
#include "runtime.h"

using pxs::DeviceArray;
using pxs::Error;

struct pxs_context {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string error;
  pxs::Frame frame;
  DeviceArray<float> params, grads, screen_gradient, target, dL, image_a, image_b, m, v;
  DeviceArray<int32_t> visible_count;
  DeviceArray<pxs::StepScalars> scalars;
  DeviceArray<float> acc_gradient, out_params;
  DeviceArray<int32_t> acc_views, source;
  pxs::DensifyWork densify;
  DeviceArray<uint8_t> export_body;
  DeviceArray<int32_t> export_fields;
  DeviceArray<uint8_t> ingest_in, ingest_bytes;
  DeviceArray<double> seed_nearest;
};

namespace {

template <typename F>
int guarded(pxs_context* ctx, F&& body) {
  if (ctx == nullptr) return PXS_ERR_INVALID;
  try {
    PXS_CUDA(cudaSetDevice(ctx->device));
    body();
    ctx->error.clear();
    return PXS_OK;
  } catch (const Error& e) {
    ctx->error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    ctx->error = "host allocation failed";
    return PXS_ERR_NO_MEMORY;
  } catch (const std::exception& e) {
    ctx->error = e.what();
    return PXS_ERR_INVALID;
  }
}

void copy_string(const std::string& s, char* out, size_t len) {
  if (out == nullptr || len == 0) return;
  std::strncpy(out, s.c_str(), len - 1);
  out[len - 1] = '\0';
}

void validate_cloud(const pxs_cloud* cloud) {
  if (cloud == nullptr) throw Error(PXS_ERR_INVALID, "cloud is null");
  if (cloud->count < 0) throw Error(PXS_ERR_INVALID, "negative gaussian count");
  const int S = cloud->rest_per_channel;
  if (S != 0 && S != 3 && S != 8 && S != 15)
    throw Error(PXS_ERR_INVALID, "rest_per_channel must be 0, 3, 8 or 15");
  if (cloud->count > 0 && cloud->params == nullptr) throw Error(PXS_ERR_INVALID, "params is null");
}

pxs_raster_options default_options() {
  pxs_raster_options o;
  o.background[0] = o.background[1] = o.background[2] = 0.f;
  o.sh_degree = 0;
  o.min_alpha = 1.f / 255.f;
  o.transmittance_cutoff = 1e-4f;
  o.screen_dilation = 0.3f;
  return o;
}

// Uploads a host cloud and runs projection and binning for one view.
void render_setup(pxs_context* ctx, const pxs_cloud* cloud, const pxs_camera* camera,
                  const pxs_raster_options* options, bool debug_cov) {
  validate_cloud(cloud);
  if (camera == nullptr) throw Error(PXS_ERR_INVALID, "camera is null");
  const pxs_raster_options opt = options ? *options : default_options();
  const int P = PXS_PARAM_COUNT(cloud->rest_per_channel);
  const size_t values = static_cast<size_t>(P) * static_cast<size_t>(cloud->count);
  float* d_params = ctx->params.reserve(values);
  if (values > 0)
    PXS_CUDA(cudaMemcpyAsync(d_params, cloud->params, values * sizeof(float),
                             cudaMemcpyHostToDevice, ctx->stream));
  const pxs::ViewBatch batch = pxs::make_batch(camera, 1, opt, cloud->sh_degree);
  ctx->frame.prepare(batch, cloud->count, cloud->rest_per_channel, ctx->stream);
  ctx->frame.project(d_params, ctx->stream, debug_cov);
  ctx->frame.bin(true, ctx->stream);
}

template <typename T>
std::vector<T> download(const T* src, size_t n, cudaStream_t stream) {
  std::vector<T> out(n);
  if (n > 0)
    PXS_CUDA(cudaMemcpyAsync(out.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, stream));
  return out;
}

}  // namespace

extern "C" {

const char* pxs_version(void) { return "parallax-b200 0.1 (sm_100a)"; }

void pxs_train_config_defaults(pxs_train_config* c) {
  if (c == nullptr) return;
  c->iterations = 7000;
  c->position_lr_initial = 1.6e-4f;
  c->position_lr_final = 1.6e-6f;
  c->dc_lr = 2.5e-3f;
  c->sh_rest_lr_divider = 20.f;
  c->opacity_lr = 0.05f;
  c->scale_lr = 5e-3f;
  c->rotation_lr = 1e-3f;
  c->adam_beta1 = 0.9f;
  c->adam_beta2 = 0.999f;
  c->adam_epsilon = 1e-15f;
  c->ssim_weight = 0.2f;
  c->sh_degree = 3;
  c->sh_increase_interval = 1000;
  c->densify_from_iteration = 500;
  c->densify_until_iteration = 5000;
  c->densify_interval = 100;
  c->densify_grad_threshold = 2e-4f;
  c->percent_dense = 0.01f;
  c->split_scale_divider = 1.6f;
  c->opacity_reset_interval = 3000;
  c->opacity_reset_value = 0.01f;
  c->prune_opacity = 0.005f;
  c->prune_scale_fraction = 0.1f;
  c->max_gaussians = 600000;
  c->seed = 7u;
}

int pxs_train_config_validate(const pxs_train_config* c, char* reason, size_t reason_len) {
  std::string why;
  if (c == nullptr) why = "config is null";
  else if (c->iterations <= 0) why = "iterations must be positive";
  else if (c->sh_degree < 0 || c->sh_degree > 3) why = "sh_degree must be between 0 and 3";
  else if (c->densify_interval <= 0) why = "densify_interval must be positive";
  else if (c->split_scale_divider <= 1.f) why = "split_scale_divider must be greater than one";
  else if (c->max_gaussians <= 0) why = "max_gaussians must be positive";
  else if (c->ssim_weight < 0.f || c->ssim_weight > 1.f) why = "ssim_weight must be in [0,1]";
  copy_string(why, reason, reason_len);
  return why.empty() ? PXS_OK : PXS_ERR_INVALID;
}

void pxs_camera_from_pose(const double K[4], int32_t width, int32_t height, const double R[9],
                          const double t[3], pxs_camera* out) {
  if (out == nullptr) return;
  for (int i = 0; i < 9; ++i) out->R[i] = static_cast<float>(R[i]);
  for (int i = 0; i < 3; ++i) {
    out->t[i] = static_cast<float>(t[i]);
    // -R^T t, each coefficient as a0*b0 + (a1*b1 + a2*b2) in double (SE3.h:46)
    const double c = -R[0 * 3 + i] * t[0] + (-R[1 * 3 + i] * t[1] + -R[2 * 3 + i] * t[2]);
    out->center[i] = static_cast<float>(c);
  }
  out->fx = static_cast<float>(K[0]);
  out->fy = static_cast<float>(K[1]);
  out->cx = static_cast<float>(K[2]);
  out->cy = static_cast<float>(K[3]);
  out->tan_half_x = static_cast<float>(0.5 * width / K[0]);
  out->tan_half_y = static_cast<float>(0.5 * height / K[1]);
  out->width = width;
  out->height = height;
}

int pxs_gpu_availability(int32_t* available, char* device_name, size_t device_name_len,
                         char* reason, size_t reason_len) {
  int count = 0;
  if (available) *available = 0;
  copy_string("", device_name, device_name_len);
  const cudaError_t err = cudaGetDeviceCount(&count);
  if (err != cudaSuccess || count == 0) {
    cudaGetLastError();
    copy_string(err != cudaSuccess ? std::string("no CUDA device: ") + cudaGetErrorString(err)
                                   : "no CUDA device",
                reason, reason_len);
    return PXS_OK;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) {
    cudaGetLastError();
    copy_string("cannot query device 0", reason, reason_len);
    return PXS_OK;
  }
  copy_string(prop.name, device_name, device_name_len);
  if (prop.major != 10 || prop.minor != 0) {
    copy_string("the library is compiled for sm_100a (B200-class) devices; found sm_" +
                    std::to_string(prop.major) + std::to_string(prop.minor),
                reason, reason_len);
    return PXS_OK;
  }
  if (available) *available = 1;
  copy_string("", reason, reason_len);
  return PXS_OK;
}

int pxs_context_create(int32_t device, pxs_context** out) {
  if (out == nullptr) return PXS_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return PXS_ERR_UNAVAILABLE;
  }
  if (device < 0 || device >= count) return PXS_ERR_INVALID;
  auto* ctx = new (std::nothrow) pxs_context;
  if (ctx == nullptr) return PXS_ERR_NO_MEMORY;
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return PXS_ERR_CUDA;
  }
  ctx->stream = ctx->own_stream;
  *out = ctx;
  return PXS_OK;
}

void pxs_context_destroy(pxs_context* ctx) {
  if (ctx == nullptr) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

int pxs_set_raster_config(int32_t forward_px, int32_t backward_px) {
  auto ok = [](int32_t v) { return v == 0 || v == 1 || v == 2 || v == 4; };
  if (!ok(forward_px) || !ok(backward_px)) return PXS_ERR_INVALID;
  pxs::RasterConfig& rc = pxs::raster_config();
  if (forward_px) rc.forward_px = forward_px;
  if (backward_px) rc.backward_px = backward_px;
  ++rc.generation;
  return PXS_OK;
}

int pxs_get_raster_config(int32_t* forward_px, int32_t* backward_px) {
  const pxs::RasterConfig& rc = pxs::raster_config();
  if (forward_px) *forward_px = rc.forward_px;
  if (backward_px) *backward_px = rc.backward_px;
  return PXS_OK;
}

int pxs_set_raster_schedule(int32_t forward_batch, int32_t backward_batch,
                            int32_t forward_schedule, int32_t backward_schedule) {
  auto batch_ok = [](int32_t v) { return v == 0 || v == 64 || v == 128 || v == 256; };
  auto schedule_ok = [](int32_t v) { return v >= -1 && v <= 2; };
  if (!batch_ok(forward_batch) || !batch_ok(backward_batch) ||
      !schedule_ok(forward_schedule) || !schedule_ok(backward_schedule))
    return PXS_ERR_INVALID;
  pxs::RasterConfig& rc = pxs::raster_config();
  if (forward_batch) rc.forward_batch = forward_batch;
  if (backward_batch) rc.backward_batch = backward_batch;
  if (forward_schedule >= 0) rc.forward_schedule = forward_schedule;
  if (backward_schedule >= 0) rc.backward_schedule = backward_schedule;
  ++rc.generation;
  return PXS_OK;
}

int pxs_get_raster_schedule(int32_t* forward_batch, int32_t* backward_batch,
                            int32_t* forward_schedule, int32_t* backward_schedule) {
  const pxs::RasterConfig& rc = pxs::raster_config();
  if (forward_batch) *forward_batch = rc.forward_batch;
  if (backward_batch) *backward_batch = rc.backward_batch;
  if (forward_schedule) *forward_schedule = rc.forward_schedule;
  if (backward_schedule) *backward_schedule = rc.backward_schedule;
  return PXS_OK;
}

const char* pxs_context_last_error(const pxs_context* ctx) {
  return ctx == nullptr ? "context is null" : ctx->error.c_str();
}

int pxs_context_set_stream(pxs_context* ctx, void* stream) {
  return guarded(ctx, [&] {
    ctx->stream = stream != nullptr ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  });
}

int pxs_context_synchronize(pxs_context* ctx) {
  return guarded(ctx, [&] { PXS_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

int pxs_project(pxs_context* ctx, const pxs_cloud* cloud, const pxs_camera* camera,
                const pxs_raster_options* options, pxs_projected_splat* out, int32_t* count) {
  return guarded(ctx, [&] {
    if (out == nullptr && cloud != nullptr && cloud->count > 0)
      throw Error(PXS_ERR_INVALID, "output is null");
    render_setup(ctx, cloud, camera, options, true);
    pxs::Frame& f = ctx->frame;
    const size_t slots = static_cast<size_t>(f.slot_stride);
    const auto order = download(f.sorted_slots, slots, ctx->stream);
    const auto keys = download(f.depth_key.get(), slots, ctx->stream);
    const auto xy = download(f.xy.get(), slots, ctx->stream);
    const auto co = download(f.conic_op.get(), slots, ctx->stream);
    const auto col = download(f.color.get(), slots, ctx->stream);
    const auto cov = download(f.debug_cov.get(), slots, ctx->stream);
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
    int32_t n = 0;
    for (size_t i = 0; i < slots; ++i) {
      const uint32_t s = order[i];
      if (keys[s] == pxs::kCulledKey) break;
      pxs_projected_splat& p = out[n++];
      p.index = static_cast<int32_t>(s);
      p.mean[0] = xy[s].x;
      p.mean[1] = xy[s].y;
      p.cov2d[0] = cov[s].x;
      p.cov2d[1] = cov[s].y;
      p.cov2d[2] = cov[s].z;
      p.radius = cov[s].w;
      p.conic[0] = co[s].x;
      p.conic[1] = co[s].y;
      p.conic[2] = co[s].z;
      p.opacity = co[s].w;
      float depth;
      std::memcpy(&depth, &keys[s], sizeof(float));
      p.depth = depth;
      p.color[0] = col[s].x;
      p.color[1] = col[s].y;
      p.color[2] = col[s].z;
      uint32_t flags;
      std::memcpy(&flags, &col[s].w, sizeof(uint32_t));
      p.clamped = flags;
    }
    if (count) *count = n;
  });
}

int pxs_tile_lists(pxs_context* ctx, const pxs_cloud* cloud, const pxs_camera* camera,
                   const pxs_raster_options* options, int32_t* offsets, int32_t* entries,
                   int64_t capacity, int64_t* total) {
  int status_capacity = PXS_OK;
  const int status = guarded(ctx, [&] {
    if (offsets == nullptr) throw Error(PXS_ERR_INVALID, "offsets is null");
    render_setup(ctx, cloud, camera, options, false);
    pxs::Frame& f = ctx->frame;
    const int tiles = f.batch.total_tiles;
    const int64_t K = f.last_pair_count;
    if (total) *total = K;
    const auto ranges = download(f.ranges.get(), static_cast<size_t>(tiles), ctx->stream);
    std::vector<uint32_t> vals;
    if (K <= capacity) vals = download(f.sorted_pair_vals, static_cast<size_t>(K), ctx->stream);
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
    // ranges are contiguous in tile order: offsets follow from the ends
    offsets[0] = 0;
    for (int t = 0; t < tiles; ++t) {
      const int len = ranges[t].y - ranges[t].x;
      offsets[t + 1] = offsets[t] + (len > 0 ? len : 0);
    }
    if (K > capacity) {
      status_capacity = PXS_ERR_CAPACITY;
      return;
    }
    if (entries != nullptr)
      for (int64_t i = 0; i < K; ++i) entries[i] = static_cast<int32_t>(vals[i]);
  });
  if (status == PXS_OK && status_capacity != PXS_OK) {
    ctx->error = "entries capacity too small for the pair count";
    return status_capacity;
  }
  return status;
}

int pxs_render(pxs_context* ctx, const pxs_cloud* cloud, const pxs_camera* camera,
               const pxs_raster_options* options, float* rgb, float* transmittance) {
  return guarded(ctx, [&] {
    if (rgb == nullptr) throw Error(PXS_ERR_INVALID, "rgb is null");
    render_setup(ctx, cloud, camera, options, false);
    pxs::Frame& f = ctx->frame;
    f.forward(ctx->stream);
    const size_t pixels = static_cast<size_t>(f.batch.total_pixels);
    if (pixels > 0) {
      PXS_CUDA(cudaMemcpyAsync(rgb, f.rgb.get(), pixels * 3 * sizeof(float),
                               cudaMemcpyDeviceToHost, ctx->stream));
      if (transmittance)
        PXS_CUDA(cudaMemcpyAsync(transmittance, f.transmittance.get(), pixels * sizeof(float),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    }
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

static void loss_common(pxs_context* ctx, const float* rendered, const float* target,
                        int32_t width, int32_t height, float ssim_weight, int mode, float* grad,
                        float* value) {
  if (width < 0 || height < 0) throw Error(PXS_ERR_INVALID, "negative image size");
  const size_t values = static_cast<size_t>(width) * static_cast<size_t>(height) * 3;
  if (values == 0) {
    if (value) *value = 0.f;
    return;
  }
  if (rendered == nullptr || target == nullptr) throw Error(PXS_ERR_INVALID, "image is null");
  pxs_camera cam;
  std::memset(&cam, 0, sizeof(cam));
  cam.width = width;
  cam.height = height;
  const pxs::ViewBatch batch = pxs::make_batch(&cam, 1, default_options(), 0);
  pxs::Frame& f = ctx->frame;
  f.prepare(batch, 0, 0, ctx->stream);
  PXS_CUDA(cudaMemcpyAsync(f.rgb.get(), rendered, values * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
  float* d_target = ctx->target.reserve(values);
  PXS_CUDA(cudaMemcpyAsync(d_target, target, values * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
  float* d_grad = ctx->dL.reserve(values);
  f.loss(d_target, ssim_weight, mode, d_grad, ctx->stream);
  if (grad)
    PXS_CUDA(cudaMemcpyAsync(grad, d_grad, values * sizeof(float), cudaMemcpyDeviceToHost,
                             ctx->stream));
  float result = 0.f;
  PXS_CUDA(cudaMemcpyAsync(&result, f.loss_total.get(), sizeof(float), cudaMemcpyDeviceToHost,
                           ctx->stream));
  PXS_CUDA(cudaStreamSynchronize(ctx->stream));
  if (value) *value = result;
}

int pxs_photometric_loss(pxs_context* ctx, const float* rendered, const float* target,
                         int32_t width, int32_t height, float ssim_weight, float* dL_drgb,
                         float* loss) {
  return guarded(ctx, [&] {
    loss_common(ctx, rendered, target, width, height, ssim_weight, 0, dL_drgb, loss);
  });
}

int pxs_mean_ssim(pxs_context* ctx, const float* rendered, const float* target, int32_t width,
                  int32_t height, float* d_rendered, float* ssim) {
  return guarded(ctx, [&] {
    loss_common(ctx, rendered, target, width, height, 1.f, 1, d_rendered, ssim);
  });
}

// Uploads host gradients, lets the kernels add into them, downloads them.
static void host_gradients_in(pxs_context* ctx, int P, int n, const pxs_gradients* g) {
  const size_t values = static_cast<size_t>(P) * static_cast<size_t>(n);
  float* d_grads = ctx->grads.reserve(values);
  float* d_screen = ctx->screen_gradient.reserve(static_cast<size_t>(n));
  int32_t* d_vis = ctx->visible_count.reserve(static_cast<size_t>(n));
  if (n == 0) return;
  PXS_CUDA(cudaMemcpyAsync(d_grads, g->params, values * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
  PXS_CUDA(cudaMemcpyAsync(d_screen, g->screen_gradient, n * sizeof(float),
                           cudaMemcpyHostToDevice, ctx->stream));
  PXS_CUDA(cudaMemcpyAsync(d_vis, g->visible_count, n * sizeof(int32_t), cudaMemcpyHostToDevice,
                           ctx->stream));
}

static void host_gradients_out(pxs_context* ctx, int P, int n, pxs_gradients* g) {
  const size_t values = static_cast<size_t>(P) * static_cast<size_t>(n);
  if (n == 0) return;
  PXS_CUDA(cudaMemcpyAsync(g->params, ctx->grads.get(), values * sizeof(float),
                           cudaMemcpyDeviceToHost, ctx->stream));
  PXS_CUDA(cudaMemcpyAsync(g->screen_gradient, ctx->screen_gradient.get(), n * sizeof(float),
                           cudaMemcpyDeviceToHost, ctx->stream));
  PXS_CUDA(cudaMemcpyAsync(g->visible_count, ctx->visible_count.get(), n * sizeof(int32_t),
                           cudaMemcpyDeviceToHost, ctx->stream));
}

static void check_gradients(const pxs_gradients* g, int n) {
  if (g == nullptr || (n > 0 && (g->params == nullptr || g->screen_gradient == nullptr ||
                                 g->visible_count == nullptr)))
    throw Error(PXS_ERR_INVALID, "gradients are null");
}

int pxs_backward(pxs_context* ctx, const pxs_cloud* cloud, const pxs_camera* camera,
                 const pxs_raster_options* options, const float* dL_drgb, pxs_gradients* grads) {
  return guarded(ctx, [&] {
    validate_cloud(cloud);
    check_gradients(grads, cloud->count);
    const int P = PXS_PARAM_COUNT(cloud->rest_per_channel);
    render_setup(ctx, cloud, camera, options, false);
    pxs::Frame& f = ctx->frame;
    f.forward(ctx->stream);
    const size_t values = static_cast<size_t>(f.batch.total_pixels) * 3;
    float* d_dL = ctx->dL.reserve(values);
    if (values > 0) {
      if (dL_drgb == nullptr) throw Error(PXS_ERR_INVALID, "dL_drgb is null");
      PXS_CUDA(cudaMemcpyAsync(d_dL, dL_drgb, values * sizeof(float), cudaMemcpyHostToDevice,
                               ctx->stream));
    }
    host_gradients_in(ctx, P, cloud->count, grads);
    f.backward(d_dL, ctx->stream);
    f.param_grads(ctx->params.get(), ctx->grads.get(), ctx->screen_gradient.get(),
                  ctx->visible_count.get(), ctx->stream);
    host_gradients_out(ctx, P, cloud->count, grads);
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int pxs_render_and_accumulate(pxs_context* ctx, const pxs_cloud* cloud, const pxs_camera* camera,
                              const pxs_raster_options* options, const float* target,
                              float ssim_weight, pxs_gradients* grads, float* loss) {
  return guarded(ctx, [&] {
    validate_cloud(cloud);
    check_gradients(grads, cloud->count);
    const int P = PXS_PARAM_COUNT(cloud->rest_per_channel);
    render_setup(ctx, cloud, camera, options, false);
    pxs::Frame& f = ctx->frame;
    const size_t values = static_cast<size_t>(f.batch.total_pixels) * 3;
    float* d_target = ctx->target.reserve(values);
    if (values > 0) {
      if (target == nullptr) throw Error(PXS_ERR_INVALID, "target is null");
      PXS_CUDA(cudaMemcpyAsync(d_target, target, values * sizeof(float), cudaMemcpyHostToDevice,
                               ctx->stream));
    }
    host_gradients_in(ctx, P, cloud->count, grads);
    f.forward(ctx->stream);
    float* d_dL = ctx->dL.reserve(values);
    f.loss(d_target, ssim_weight, 0, d_dL, ctx->stream);
    f.backward(d_dL, ctx->stream);
    f.param_grads(ctx->params.get(), ctx->grads.get(), ctx->screen_gradient.get(),
                  ctx->visible_count.get(), ctx->stream);
    host_gradients_out(ctx, P, cloud->count, grads);
    float value = 0.f;
    PXS_CUDA(cudaMemcpyAsync(&value, f.loss_total.get(), sizeof(float), cudaMemcpyDeviceToHost,
                             ctx->stream));
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (loss) *loss = values > 0 ? value : 0.f;
  });
}

int pxs_render_and_accumulate_device(pxs_context* ctx, const pxs_cloud* cloud,
                                     const pxs_camera* camera,
                                     const pxs_raster_options* options, const float* target,
                                     float ssim_weight, pxs_gradients* grads, float* loss) {
  return guarded(ctx, [&] {
    validate_cloud(cloud);
    check_gradients(grads, cloud->count);
    if (camera == nullptr) throw Error(PXS_ERR_INVALID, "camera is null");
    const pxs_raster_options opt = options ? *options : default_options();
    const pxs::ViewBatch batch = pxs::make_batch(camera, 1, opt, cloud->sh_degree);
    pxs::Frame& f = ctx->frame;
    f.prepare(batch, cloud->count, cloud->rest_per_channel, ctx->stream);
    f.project(cloud->params, ctx->stream);
    f.bin(true, ctx->stream);
    f.forward(ctx->stream);
    const size_t values = static_cast<size_t>(f.batch.total_pixels) * 3;
    float* d_dL = ctx->dL.reserve(values);
    f.loss(target, ssim_weight, 0, d_dL, ctx->stream);
    f.backward(d_dL, ctx->stream);
    f.param_grads(cloud->params, grads->params, grads->screen_gradient, grads->visible_count,
                  ctx->stream);
    if (loss)
      PXS_CUDA(cudaMemcpyAsync(loss, f.loss_total.get(), sizeof(float),
                               cudaMemcpyDeviceToDevice, ctx->stream));
  });
}

int pxs_adam_device(pxs_context* ctx, float* params, float* grads, float* m, float* v,
                    int32_t count, int32_t rest_per_channel, const float lr[6], float beta1,
                    float beta2, float epsilon, float correction1, float correction2,
                    int32_t zero_grads) {
  return guarded(ctx, [&] {
    if (count < 0 || lr == nullptr) throw Error(PXS_ERR_INVALID, "bad Adam arguments");
    pxs::StepScalars s;
    std::memset(&s, 0, sizeof(s));
    for (int i = 0; i < 6; ++i) s.lr[i] = lr[i];
    s.beta1 = beta1;
    s.beta2 = beta2;
    s.epsilon = epsilon;
    s.correction1 = correction1;
    s.correction2 = correction2;
    pxs::StepScalars* d = ctx->scalars.reserve(1);
    PXS_CUDA(cudaMemcpyAsync(d, &s, sizeof(s), cudaMemcpyHostToDevice, ctx->stream));
    pxs::launch_adam(params, grads, m, v, count, rest_per_channel, d, zero_grads, nullptr,
                     nullptr, nullptr, nullptr, ctx->stream);
    PXS_CUDA(cudaGetLastError());
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int pxs_initialize_from_points(pxs_context* ctx, const float* points, const uint8_t* colors,
                               int32_t n, int32_t sh_degree, float initial_opacity,
                               float* params, int32_t* rest_per_channel) {
  return guarded(ctx, [&] {
    if (n < 0) throw Error(PXS_ERR_INVALID, "negative point count");
    const int degree = std::max(0, std::min(3, static_cast<int>(sh_degree)));
    const int S = (degree + 1) * (degree + 1) - 1;
    if (rest_per_channel) *rest_per_channel = S;
    if (n == 0 || params == nullptr) return;
    if (points == nullptr) throw Error(PXS_ERR_INVALID, "points are null");
    // the sampled nearest-neighbour spacing (GaussianCloud.cpp:206-227)
    const int sample = std::min(n, 512);
    const int stride = std::max(1, n / sample);
    const int samples = (n + stride - 1) / stride;  // i = 0, stride, ... < n
    float* d_points = ctx->image_b.reserve(static_cast<size_t>(n) * 3);
    PXS_CUDA(cudaMemcpyAsync(d_points, points, sizeof(float) * 3 * n, cudaMemcpyHostToDevice,
                             ctx->stream));
    double* d_near = ctx->seed_nearest.reserve(static_cast<size_t>(samples));
    pxs::launch_seed_nearest(d_points, n, stride, samples, d_near, ctx->stream);
    PXS_CUDA(cudaGetLastError());
    std::vector<double> nearest(static_cast<size_t>(samples));
    PXS_CUDA(cudaMemcpyAsync(nearest.data(), d_near, sizeof(double) * samples,
                             cudaMemcpyDeviceToHost, ctx->stream));
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
    double spacing = 0.0;
    int counted = 0;
    for (double d : nearest) {
      if (d < 1e29) {
        spacing += d;
        ++counted;
      }
    }
    spacing = counted > 0 ? spacing / counted : 0.01;
    const double sigma = std::max(1e-4, spacing * 0.5);
    const float log_sigma = static_cast<float>(std::log(sigma));
    const float logit = std::log(std::max(1e-6f, initial_opacity) /
                                 std::max(1e-6f, 1.f - initial_opacity));
    const uint8_t* d_colors = nullptr;
    if (colors != nullptr) {
      uint8_t* dc = ctx->ingest_in.reserve(static_cast<size_t>(n) * 3);
      PXS_CUDA(cudaMemcpyAsync(dc, colors, static_cast<size_t>(n) * 3, cudaMemcpyHostToDevice,
                               ctx->stream));
      d_colors = dc;
    }
    const size_t values = static_cast<size_t>(PXS_PARAM_COUNT(S)) * n;
    float* d_params = ctx->params.reserve(values);
    pxs::launch_seed_points(d_points, d_colors, n, S, log_sigma, logit, d_params, ctx->stream);
    PXS_CUDA(cudaGetLastError());
    PXS_CUDA(cudaMemcpyAsync(params, d_params, values * sizeof(float), cudaMemcpyDeviceToHost,
                             ctx->stream));
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int pxs_downscale_to_width(pxs_context* ctx, const uint8_t* rgb, int32_t width, int32_t height,
                           int32_t target_width, uint8_t* out_rgb, float* out_linear,
                           int32_t* out_width, int32_t* out_height) {
  return guarded(ctx, [&] {
    if (width < 0 || height < 0) throw Error(PXS_ERR_INVALID, "negative image size");
    int w = 0, h = 0;
    pxs::downscaled_size(width, height, target_width, &w, &h);
    if (out_width) *out_width = w;
    if (out_height) *out_height = h;
    const size_t in_bytes = static_cast<size_t>(width) * height * 3;
    const size_t out_values = static_cast<size_t>(w) * h * 3;
    if ((out_rgb == nullptr && out_linear == nullptr) || out_values == 0) return;
    if (rgb == nullptr) throw Error(PXS_ERR_INVALID, "image is null");
    uint8_t* d_in = ctx->ingest_in.reserve(in_bytes);
    PXS_CUDA(cudaMemcpyAsync(d_in, rgb, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
    uint8_t* d_bytes = out_rgb ? ctx->ingest_bytes.reserve(out_values) : nullptr;
    float* d_lin = out_linear ? ctx->image_a.reserve(out_values) : nullptr;
    pxs::launch_downscale(d_in, width, height, w, h, d_bytes, d_lin, ctx->stream);
    PXS_CUDA(cudaGetLastError());
    if (out_rgb)
      PXS_CUDA(cudaMemcpyAsync(out_rgb, d_bytes, out_values, cudaMemcpyDeviceToHost, ctx->stream));
    if (out_linear)
      PXS_CUDA(cudaMemcpyAsync(out_linear, d_lin, out_values * sizeof(float),
                               cudaMemcpyDeviceToHost, ctx->stream));
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

// Copies `bytes` out, or reports the size needed.
static int deliver_bytes(const std::vector<uint8_t>& bytes, uint8_t* out, size_t capacity,
                         size_t* size) {
  if (size != nullptr) *size = bytes.size();
  if (out == nullptr || capacity < bytes.size()) return PXS_ERR_CAPACITY;
  std::memcpy(out, bytes.data(), bytes.size());
  return PXS_OK;
}

int pxs_export_cloud(pxs_context* ctx, const pxs_cloud* cloud, int32_t format,
                     int32_t fractional_bits, uint8_t* out, size_t capacity, size_t* size) {
  std::vector<uint8_t> bytes;
  const int status = guarded(ctx, [&] {
    validate_cloud(cloud);
    if (cloud->count <= 0) throw Error(PXS_ERR_INVALID, "the cloud is empty");
    const size_t values =
        static_cast<size_t>(PXS_PARAM_COUNT(cloud->rest_per_channel)) * cloud->count;
    float* d = ctx->params.reserve(values);
    PXS_CUDA(cudaMemcpyAsync(d, cloud->params, values * sizeof(float), cudaMemcpyHostToDevice,
                             ctx->stream));
    bytes = pxs::export_cloud_bytes(d, cloud->count, cloud->rest_per_channel, cloud->sh_degree,
                                    format, fractional_bits, ctx->export_body,
                                    ctx->export_fields, ctx->stream);
  });
  if (status != PXS_OK) return status;
  return deliver_bytes(bytes, out, capacity, size);
}

int pxs_densify_and_prune(pxs_context* ctx, float* params, int32_t* count,
                          int32_t rest_per_channel, const float* screen_gradient,
                          const int32_t* visible_count, const pxs_train_config* config,
                          float extent, int32_t iteration, uint32_t* rng_state,
                          int32_t* source_index, int32_t* cloned, int32_t* split,
                          int32_t* pruned) {
  return guarded(ctx, [&] {
    if (params == nullptr || count == nullptr || config == nullptr || rng_state == nullptr)
      throw Error(PXS_ERR_INVALID, "null argument");
    const int S = rest_per_channel;
    if (S != 0 && S != 3 && S != 8 && S != 15)
      throw Error(PXS_ERR_INVALID, "rest_per_channel must be 0, 3, 8 or 15");
    const int N = *count;
    if (N < 0) throw Error(PXS_ERR_INVALID, "negative count");
    if (cloned) *cloned = 0;
    if (split) *split = 0;
    if (pruned) *pruned = 0;
    if (N == 0) return;  // SplatDensify.cpp:32-33
    const int P = PXS_PARAM_COUNT(S);
    const size_t n = static_cast<size_t>(N);
    const int64_t cap = std::max<int64_t>(config->max_gaussians, N);
    float* d_params = ctx->params.reserve(static_cast<size_t>(P) * n);
    float* d_acc = ctx->acc_gradient.reserve(n);
    int32_t* d_views = ctx->acc_views.reserve(n);
    float* d_out = ctx->out_params.reserve(static_cast<size_t>(P) * static_cast<size_t>(cap));
    int32_t* d_source = ctx->source.reserve(static_cast<size_t>(cap));
    PXS_CUDA(cudaMemcpyAsync(d_params, params, sizeof(float) * P * n, cudaMemcpyHostToDevice,
                             ctx->stream));
    PXS_CUDA(cudaMemcpyAsync(d_acc, screen_gradient, sizeof(float) * n, cudaMemcpyHostToDevice,
                             ctx->stream));
    PXS_CUDA(cudaMemcpyAsync(d_views, visible_count, sizeof(int32_t) * n,
                             cudaMemcpyHostToDevice, ctx->stream));
    pxs::DensifyArgs a;
    a.grad_threshold = config->densify_grad_threshold;
    a.size_threshold = config->percent_dense * extent;
    a.max_scale = config->prune_scale_fraction * extent;
    a.prune_opacity = config->prune_opacity;
    a.log_split_divider = std::log(config->split_scale_divider);
    a.prune_oversized = iteration > config->opacity_reset_interval ? 1 : 0;
    a.has_room = N < config->max_gaussians ? 1 : 0;
    a.max_gaussians = config->max_gaussians;
    a.rng_state = *rng_state;
    const pxs::DensifyResult r =
        pxs::densify_device(ctx->densify, d_params, nullptr, nullptr, N, S, d_acc, d_views, a,
                            d_out, nullptr, nullptr, d_source, cap, ctx->stream);
    const size_t out_values = static_cast<size_t>(P) * static_cast<size_t>(r.count);
    if (out_values > 0)
      PXS_CUDA(cudaMemcpyAsync(params, d_out, sizeof(float) * out_values,
                               cudaMemcpyDeviceToHost, ctx->stream));
    if (source_index != nullptr && r.count > 0)
      PXS_CUDA(cudaMemcpyAsync(source_index, d_source, sizeof(int32_t) * r.count,
                               cudaMemcpyDeviceToHost, ctx->stream));
    PXS_CUDA(cudaStreamSynchronize(ctx->stream));
    *count = static_cast<int32_t>(r.count);
    *rng_state = r.rng_state;
    if (cloned) *cloned = r.cloned;
    if (split) *split = r.split;
    if (pruned) *pruned = r.pruned;
  });
}

}  // extern "C"
