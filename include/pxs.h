/*
 * pxs.h -- C ABI of the B200 Gaussian-splat training core.
 *
 * Every entry point returns an int status (PXS_OK on success) and never throws
 * across the boundary; the message for the last failure on a context or a
 * trainer is read with pxs_context_last_error / pxs_trainer_last_error. This
 * mirrors the reference's "false plus a human-readable string" contract of
 * `trainSplatsOnGpu` (engine/native/cpp/include/parallax/splat/VulkanSplatTrainer.h:27-37).
 *
 * Parameter layout (host and device alike): one float array of P x N values,
 * component-major, so component c of gaussian g lives at params[c * N + g]:
 *
 *   0..2   position (x, y, z)                 Gaussian::position
 *   3..5   log sigma                          Gaussian::log_scale
 *   6..9   rotation quaternion (w, x, y, z)   Gaussian::rotation
 *   10     opacity logit                      Gaussian::opacity_logit
 *   11..13 degree-0 SH coefficient            Gaussian::dc
 *   14..   higher SH, channel-major (R.., G.., B..), rest_per_channel each
 *                                             Gaussian::sh_rest
 *
 * P = 14 + 3 * rest_per_channel. (GaussianCloud.h:41-51 of the reference.)
 * Gradients, Adam moments and the trainer's device state use the same layout.
 */
#ifndef PXS_H
#define PXS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */

#define PXS_OK 0
#define PXS_ERR_INVALID 1     /* bad argument or configuration */
#define PXS_ERR_CUDA 2        /* a CUDA runtime call failed */
#define PXS_ERR_NO_MEMORY 3   /* device or host allocation failed */
#define PXS_ERR_CAPACITY 4    /* a fixed-size buffer would have overflowed */
#define PXS_ERR_UNAVAILABLE 5 /* no usable sm_100 device */
#define PXS_ERR_TIMEOUT 6     /* a bounded device-side wait gave up */

#define PXS_C_POSITION 0
#define PXS_C_LOG_SCALE 3
#define PXS_C_ROTATION 6
#define PXS_C_OPACITY 10
#define PXS_C_DC 11
#define PXS_C_SH_REST 14

/* Floats per gaussian for a given number of higher-order SH coefficients per
 * channel (0, 3, 8 or 15 for degrees 0..3). */
#define PXS_PARAM_COUNT(rest_per_channel) (14 + 3 * (rest_per_channel))

/* Logical binning tile, in pixels. Fixed: tile membership decides which
 * gaussians a pixel sees (SplatRaster.cpp:18, :121-126). */
#define PXS_TILE 16

/* ------------------------------------------------------------------- types */

/*
 * A camera in the single-precision form the rasteriser consumes.
 * Replaces SplatView = {CameraIntrinsics, Pose} (SplatRaster.h:25-29); the
 * double-to-float conversion the reference does at SplatRaster.cpp:206-212 is
 * done once by pxs_camera_from_pose.
 */
typedef struct pxs_camera {
  float R[9];      /* camera-from-world rotation, row-major */
  float t[3];      /* camera-from-world translation */
  float center[3]; /* camera centre in world coordinates, -R^T t */
  float fx, fy, cx, cy;
  float tan_half_x, tan_half_y; /* 0.5 * width / fx, 0.5 * height / fy */
  int32_t width, height;
} pxs_camera;

/* RasterOptions (SplatRaster.h:31-52). */
typedef struct pxs_raster_options {
  float background[3];
  int32_t sh_degree;
  float min_alpha;
  float transmittance_cutoff;
  float screen_dilation;
} pxs_raster_options;

/* ProjectedSplat (SplatRaster.h:56-72). `clamped` has bit c set when colour
 * channel c was clamped at zero. */
typedef struct pxs_projected_splat {
  int32_t index;
  float mean[2];
  float cov2d[3];
  float conic[3];
  float depth;
  float radius;
  float color[3];
  float opacity;
  uint32_t clamped;
} pxs_projected_splat;

/* A cloud in the component-major layout described above. `params` is a host
 * pointer for the host-buffer entry points and a device pointer for the
 * *_device ones. `sh_degree` is GaussianCloud::sh_degree. */
typedef struct pxs_cloud {
  float* params;
  int32_t count;
  int32_t rest_per_channel;
  int32_t sh_degree;
} pxs_cloud;

/* Per-gaussian gradients, SplatGradients (SplatRaster.h:87-115). `params`
 * holds P x count floats in the parameter layout; every entry point ADDS into
 * all three arrays, like rasterizeSplatsBackward (SplatRaster.h:134-137). */
typedef struct pxs_gradients {
  float* params;
  float* screen_gradient;
  int32_t* visible_count;
} pxs_gradients;

/* SplatTrainingConfig (SplatTrainer.h:25-94), same fields and defaults
 * (pxs_train_config_defaults). */
typedef struct pxs_train_config {
  int32_t iterations;
  float position_lr_initial, position_lr_final;
  float dc_lr, sh_rest_lr_divider, opacity_lr, scale_lr, rotation_lr;
  float adam_beta1, adam_beta2, adam_epsilon;
  float ssim_weight;
  int32_t sh_degree, sh_increase_interval;
  int32_t densify_from_iteration, densify_until_iteration, densify_interval;
  float densify_grad_threshold, percent_dense, split_scale_divider;
  int32_t opacity_reset_interval;
  float opacity_reset_value;
  float prune_opacity, prune_scale_fraction;
  int32_t max_gaussians;
  uint32_t seed;
} pxs_train_config;

/* SplatTrainingProgress (SplatTrainer.h:96-104). */
typedef struct pxs_progress {
  int32_t iteration, total_iterations, gaussian_count;
  float loss, smoothed_loss;
} pxs_progress;

/* Returns nonzero to continue, zero to cancel (SplatTrainingCallback,
 * SplatTrainer.h:129-130). */
typedef int (*pxs_progress_fn)(const pxs_progress* progress, void* user);

/* ------------------------------------------------------------ host helpers */

/* Library version string. */
const char* pxs_version(void);

/* SplatTrainingConfig{} defaults. */
void pxs_train_config_defaults(pxs_train_config* config);

/* SplatTrainingConfig::validate (SplatTrainer.cpp:118-126). Returns PXS_OK or
 * PXS_ERR_INVALID and writes the reason into `reason` (may be NULL). */
int pxs_train_config_validate(const pxs_train_config* config, char* reason, size_t reason_len);

/* Builds the float camera from double intrinsics (fx, fy, cx, cy), image size
 * and a camera-from-world pose (R row-major, t), with the reference's casts
 * and its double-precision camera centre (SE3.h:46). */
void pxs_camera_from_pose(const double intrinsics[4], int32_t width, int32_t height,
                          const double R[9], const double t[3], pxs_camera* out);

/* --------------------------------------------------------------- contexts */

typedef struct pxs_context pxs_context;

/* splatGpuAvailability (VulkanSplatTrainer.h:15-25). Writes NUL-terminated
 * strings; returns PXS_OK whether or not a device is available. */
int pxs_gpu_availability(int32_t* available, char* device_name, size_t device_name_len,
                         char* reason, size_t reason_len);

/* A context owns a CUDA stream on `device` and a grow-only device workspace.
 * It is not thread-safe; use one per host thread. */
int pxs_context_create(int32_t device, pxs_context** out);
void pxs_context_destroy(pxs_context* context);
const char* pxs_context_last_error(const pxs_context* context);
/* Runs subsequent device work on `stream` (a cudaStream_t) instead of the
 * context's own; NULL restores the context's stream. */
int pxs_context_set_stream(pxs_context* context, void* stream);
int pxs_context_synchronize(pxs_context* context);

/* ------------------------------------------- rasteriser (host buffers in/out)
 * These copy their inputs to the device, run the sm_100a kernels and copy the
 * results back, so they are drop-in for the reference's host functions. */

/* projectSplats (SplatRaster.h:122-125; SplatRaster.cpp:201-263). Writes the
 * visible splats sorted near to far (ties by gaussian index) into `out`
 * (capacity cloud->count) and their number into `count`. */
int pxs_project(pxs_context* context, const pxs_cloud* cloud, const pxs_camera* camera,
                const pxs_raster_options* options, pxs_projected_splat* out, int32_t* count);

/* The per-tile key lists that rasterizeSplats composites in
 * (SplatRaster.cpp:114-151): for tile t, the gaussian indices
 * entries[offsets[t] .. offsets[t+1]) near to far. `offsets` holds
 * tiles + 1 values; `entries` has room for `capacity` values; `total` gets the
 * pair count even when it exceeds `capacity` (then PXS_ERR_CAPACITY). */
int pxs_tile_lists(pxs_context* context, const pxs_cloud* cloud, const pxs_camera* camera,
                   const pxs_raster_options* options, int32_t* offsets, int32_t* entries,
                   int64_t capacity, int64_t* total);

/* renderSplats (SplatRaster.h:131-132): rgb is width*height*3 floats,
 * transmittance width*height (may be NULL). */
int pxs_render(pxs_context* context, const pxs_cloud* cloud, const pxs_camera* camera,
               const pxs_raster_options* options, float* rgb, float* transmittance);

/* photometricLoss (SplatRaster.h:153-154). dL_drgb may be NULL. */
int pxs_photometric_loss(pxs_context* context, const float* rendered, const float* target,
                         int32_t width, int32_t height, float ssim_weight, float* dL_drgb,
                         float* loss);

/* meanSsim (SplatRaster.h:158-159). d_rendered may be NULL. */
int pxs_mean_ssim(pxs_context* context, const float* rendered, const float* target,
                  int32_t width, int32_t height, float* d_rendered, float* ssim);

/* rasterizeSplatsBackward (SplatRaster.h:139-143): renders `cloud` from
 * `camera`, back-propagates `dL_drgb` and ADDS into `grads`. */
int pxs_backward(pxs_context* context, const pxs_cloud* cloud, const pxs_camera* camera,
                 const pxs_raster_options* options, const float* dL_drgb,
                 pxs_gradients* grads);

/* SplatBackend::renderAndAccumulate (SplatTrainer.h:118-122;
 * SplatTrainer.cpp:104-113): render, score against `target`, ADD the
 * gradients, return the loss. */
int pxs_render_and_accumulate(pxs_context* context, const pxs_cloud* cloud,
                              const pxs_camera* camera, const pxs_raster_options* options,
                              const float* target, float ssim_weight, pxs_gradients* grads,
                              float* loss);

/* ------------------------------------------------ device-resident variants
 * Same operations on device pointers, queued on the context's stream; nothing
 * is copied and nothing waits for the device unless stated. */

/* renderAndAccumulate on device buffers. `loss` is a device pointer to one
 * float that receives the loss. Pair buffers grow on demand, which reads the
 * pair count back to the host once per call. */
int pxs_render_and_accumulate_device(pxs_context* context, const pxs_cloud* cloud,
                                     const pxs_camera* camera,
                                     const pxs_raster_options* options,
                                     const float* target, float ssim_weight,
                                     pxs_gradients* grads, float* loss);

/* One Adam step over every parameter, the trainer's applyGradients
 * (SplatTrainer.cpp:56-65, :218-256), including the quaternion renormalisation.
 * `lr` holds the six group learning rates (position, log_scale, rotation,
 * opacity, dc, sh_rest); correction1/2 are 1 - beta^t. Device pointers.
 * When `zero_grads` is nonzero the gradient array is cleared afterwards. */
int pxs_adam_device(pxs_context* context, float* params, float* grads, float* m, float* v,
                    int32_t count, int32_t rest_per_channel, const float lr[6],
                    float beta1, float beta2, float epsilon, float correction1,
                    float correction2, int32_t zero_grads);

/* ------------------------------------------------- allocation-free variant
 * No counterpart in the reference. For callers that cannot allocate device
 * memory: a host framework whose caching allocator owns the GPU's memory and
 * its budget (memory taken behind its back can push it out of memory), or a
 * loop sharing the GPU with other streams, where the device-wide
 * synchronisation of cudaFree would stall them. It also needs no context,
 * whose buffers grow by allocation.
 *
 * The photometric loss of n_views images of width x height, on device
 * buffers: rendered, target and dL_drgb hold n_views * height * width * 3
 * floats (image after image, row-major RGB). It is pxs_photometric_loss per
 * image, batched: per_view_loss[v] (device, n_views floats) gets image v's
 * loss and `loss` (device, one float) their mean; dL_drgb, per_view_loss and
 * loss may each be NULL. Work is queued on `stream` (a cudaStream_t; NULL is
 * the default stream) and nothing waits for it.
 *
 * The kernel's scratch (per-image descriptors and sums) lives in a static
 * array of PXS_STATIC_LOSS_SCRATCH_BYTES in device memory, which every GPU
 * that loads this library holds until the process exits; so n_views is
 * limited to PXS_STATIC_LOSS_MAX_VIEWS, and a larger count is rejected with
 * PXS_ERR_INVALID. The call allocates no device memory and calls no
 * allocating routine. The first call on each device (the current one) looks
 * up the array's address and sets the kernel's shared-memory limit, once; make
 * that first call before any stream capture. On a thread with no current
 * context that first call also creates the device's primary context and loads
 * this library's kernels, which takes device memory of its own (as any first
 * CUDA call does); a caller whose allocator owns the device's memory should
 * make it, or create the context, before setting its memory budget. Every call on a device shares
 * the one array: calls whose work overlaps on the GPU (two streams, two host
 * threads) race and give wrong results, so order them (one stream, or
 * events). Each call clears the sums it uses before the kernel runs.
 * On failure the reason is written to `error` (may be NULL). */
#define PXS_STATIC_LOSS_MAX_VIEWS 64
#define PXS_STATIC_LOSS_SCRATCH_BYTES 16384
int pxs_photometric_loss_static(const float* rendered, const float* target, int32_t width,
                                int32_t height, int32_t n_views, float ssim_weight,
                                float* dL_drgb, float* per_view_loss, float* loss,
                                void* stream, char* error, size_t error_len);

/* --------------------------------------------------------------- trainer
 * A device-resident SplatTrainer (SplatTrainer.h:132-161): the cloud, the
 * gradients, the Adam moments and the training images stay in device memory
 * from create to destroy. The schedule (view order, SH warm-up, learning-rate
 * decay, densify cadence, opacity reset) is the reference trainer's
 * (SplatTrainer.cpp:163-383). */

typedef struct pxs_trainer pxs_trainer;

/* `images[v]` is views[v]'s width*height*3 linear RGB target, row-major. */
int pxs_trainer_create(const pxs_train_config* config, const pxs_cloud* initial,
                       const pxs_camera* cameras, const float* const* images, int32_t n_views,
                       int32_t device, pxs_trainer** out);
void pxs_trainer_destroy(pxs_trainer* trainer);
const char* pxs_trainer_last_error(const pxs_trainer* trainer);

/* SplatTrainer::step (SplatTrainer.cpp:326-362): one iteration on the next
 * view. `stepped` is 0 once the schedule is finished. It runs the batched
 * step over that one view: no host round trip inside the step, and one
 * replay of a captured graph when all the trainer's views share a size
 * (pxs_trainer_step_views runs the plain per-view sequence instead). */
int pxs_trainer_step(pxs_trainer* trainer, int32_t* stepped);

/* SplatTrainer::train (SplatTrainer.cpp:364-376). `completed` is 0 when the
 * callback cancelled. */
int pxs_trainer_train(pxs_trainer* trainer, pxs_progress_fn callback, void* user,
                      int32_t* completed);

/* The batched form: renders and differentiates `n_views` views in one pass of
 * each kernel, accumulates their gradients and takes one Adam step.
 * `view_ids` may be NULL to take the next n_views of the shuffled order.
 * When `graph` is nonzero the step runs as a captured CUDA graph (captured on
 * first use, re-captured when the gaussian count changes). */
int pxs_trainer_step_batch(pxs_trainer* trainer, int32_t n_views, const int32_t* view_ids,
                           int32_t graph, float* loss);

/* A trainer over several independent scenes in one cloud, for batches that
 * render and differentiate views of many scenes of uneven sizes in one pass
 * of each kernel. Scene s has its own cloud (clouds[s]; all with the same
 * rest_per_channel and sh_degree) and views_per_scene[s] consecutive entries
 * of cameras / images. The scenes are joined into one cloud (scene after
 * scene, component-major), every view renders only its own scene's
 * gaussians, and the position learning rate of each gaussian uses its own
 * scene's camera extent (positionLearningRate, SplatTrainer.cpp:200-208), so a
 * step over a batch of views updates every scene as its own trainer would.
 * Train with pxs_trainer_step_batch / step_views / accumulate; read the
 * result with pxs_trainer_download (the joined cloud, scene after scene).
 * Densification resizes one cloud, so with more than one scene the config
 * must not densify (densify_from_iteration past the last iteration), and
 * pxs_trainer_finish is refused. */
int pxs_trainer_create_scenes(const pxs_train_config* config, const pxs_cloud* clouds,
                              int32_t n_scenes, const int32_t* views_per_scene,
                              const pxs_camera* cameras, const float* const* images,
                              int32_t device, pxs_trainer** trainer);

/* The data-parallel split of pxs_trainer_step_batch, for one trainer per GPU
 * over a shared cloud. pxs_trainer_accumulate renders and differentiates this
 * rank's `n_views` views (a graph replay when `graph` is nonzero) and leaves
 * the step's sums in the trainer's reduction block with no optimiser step;
 * `loss` (may be NULL) gets the mean loss of these views. The caller sums the
 * block of pxs_trainer_reduction_block over the ranks (one all-reduce in
 * place, on or after the trainer's stream) and calls pxs_trainer_apply, which
 * takes the Adam step and the schedule's densify / opacity reset. With `loss`
 * NaN, apply takes the mean loss over all ranks' views from the summed block,
 * so no separate reduction of the loss is needed. Ranks that apply identical
 * sums stay identical.
 * The block is (values + 2) x count + 2 floats: the parameter gradients
 * (values x count, the parameter layout), the screen gradient (count), the
 * visible counts as floats (count; exact integers) and the loss tail (the
 * rank's mean loss times its views, its views). pxs_trainer_gradients returns
 * pointers to its first three parts. Both are device pointers, valid until the
 * cloud is resized (densify). No reference counterpart: the reference trains
 * on one device (SplatTrainer.cpp:326-362); its gradients are sums over views
 * (SplatRaster.h:133-137), which is what makes the split exact. */
int pxs_trainer_accumulate(pxs_trainer* trainer, int32_t n_views, const int32_t* view_ids,
                           int32_t graph, float* loss);
int pxs_trainer_apply(pxs_trainer* trainer, float loss);
int pxs_trainer_reduction_block(pxs_trainer* trainer, float** block, int64_t* values);
int pxs_trainer_gradients(pxs_trainer* trainer, float** params, float** screen_gradient,
                          float** visible_count, int32_t* count, int32_t* values);

/* Plain form of the same multi-view step: per-view kernel sequences with
 * host-synchronised sizes and no graph. Same arithmetic, same result. */
int pxs_trainer_step_views(pxs_trainer* trainer, int32_t n_views, const int32_t* view_ids,
                           float* loss);

/* Renders the trainer's current cloud from `camera` into host memory (rgb
 * width*height*3, transmittance width*height or NULL): SplatBackend::render
 * (SplatTrainer.h:123-124). NULL options use the trainer's current ones. */
int pxs_trainer_render(pxs_trainer* trainer, const pxs_camera* camera,
                       const pxs_raster_options* options, float* rgb, float* transmittance);

/* Pixels per thread of the compositing kernel and of its adjoint: 1, 2 or 4
 * each (0 keeps the current value; anything else is PXS_ERR_INVALID). The
 * setting is process-wide and read at launch; a trainer re-captures its step
 * graph after a change. The results do not depend on it beyond the order in
 * which the adjoint sums gradients. */
int pxs_set_raster_config(int32_t forward_px, int32_t backward_px);
int pxs_get_raster_config(int32_t* forward_px, int32_t* backward_px);

/* The launch shape of the two-pixel compositing kernel and of its adjoint:
 * the tile-list entries each CTA stages per batch (64, 128 or 256; 0 keeps
 * the current value) and how CTAs map to tiles: 0 one CTA per tile in tile
 * order, 1 one CTA per tile with the tiles of longest lists first, 2 one
 * persistent launch of as many CTAs as the device holds at once, taking tiles
 * longest-list first from a device counter (-1 keeps the current value).
 * The logical 16-pixel tiles, and so every result, stay the same: only the
 * order in which the adjoint's atomics sum gradients changes. Process-wide,
 * read at launch; a trainer re-captures its step graph after a change.
 * Defaults: batches 128 / 256, schedule 0 / 0. The reference's Vulkan
 * trainer fixes both: one workgroup per tile in tile order
 * (VulkanSplatTrainer.cpp:570, 607; forward.comp:14, backward.comp:16). */
int pxs_set_raster_schedule(int32_t forward_batch, int32_t backward_batch,
                            int32_t forward_schedule, int32_t backward_schedule);
int pxs_get_raster_schedule(int32_t* forward_batch, int32_t* backward_batch,
                            int32_t* forward_schedule, int32_t* backward_schedule);

/* The autotuner, on the batch of `view_ids` (NULL: the first n_views views):
 * first the pixels per thread of the compositing kernel and its adjoint (1,
 * 2 or 4 each, the pair timed together: the two-pixel forward records which
 * 8x8 blocks took each entry, which the two-pixel adjoint uses); then, for the
 * two-pixel forms chosen, the per-block entry batch (64 / 128 / 256) and the
 * tile schedule (0 / 1 / 2) of each kernel, one at a time. Keeps the fastest
 * settings (pxs_get_raster_config / pxs_get_raster_schedule read them) and
 * writes the pixels per thread to forward_px / backward_px (either may be
 * NULL). The schedule of training, the cloud and its gradients are not
 * changed. */
int pxs_trainer_autotune(pxs_trainer* trainer, int32_t n_views, const int32_t* view_ids,
                         int32_t* forward_px, int32_t* backward_px);
/* The last autotune's measurements, one line per candidate (mean time per
 * launch), into `text` (truncated to `capacity`). */
int pxs_trainer_autotune_report(pxs_trainer* trainer, char* text, size_t capacity);

/* Measures this device's FP32 FMA throughput (TFLOP/s) with a microkernel:
 * the roofline denominator of the FP32-bound compositing kernels. */
int pxs_measure_fp32_peak(int32_t device, float* tflops);

/* The CUDA stream (a cudaStream_t) the trainer's kernels run on. */
int pxs_trainer_stream(pxs_trainer* trainer, void** stream);

/* Stage timing of the batched step: when enabled, CUDA events are recorded on
 * the trainer's stream between its stages (project, bin, forward, loss,
 * backward, param_grads, adam; inside the captured graph as event nodes) and
 * their elapsed times accumulated. pxs_trainer_stage_times returns the
 * accumulated milliseconds per stage and the number of steps timed. */
int pxs_trainer_set_timing(pxs_trainer* trainer, int32_t enable);
int pxs_trainer_stage_times(pxs_trainer* trainer, float* ms, int32_t capacity,
                            int32_t* n_stages, int32_t* n_steps);

/* Tile pairs and kernel launches of the last step. */
int pxs_trainer_step_info(pxs_trainer* trainer, int64_t* pairs, int64_t* kernel_launches);

/* Re-runs the last batch's forward pass counting the (pixel, entry) pairs the
 * compositing loop evaluates and those passing both alpha tests. */
int pxs_trainer_pair_stats(pxs_trainer* trainer, int64_t* evaluated, int64_t* contributing);

/* Replaces the resident target images of `view_ids` from host memory (queued
 * on the trainer's stream; pinned memory makes the copies asynchronous). */
int pxs_trainer_set_images(pxs_trainer* trainer, int32_t n, const int32_t* view_ids,
                           const float* const* images);

/* iteration, gaussian count, last loss, smoothed loss, scene extent and the
 * SH degree in use (SplatTrainer.h:144-153). Any pointer may be NULL. */
int pxs_trainer_state(pxs_trainer* trainer, int32_t* iteration, int32_t* count,
                      float* last_loss, float* smoothed_loss, float* extent,
                      int32_t* sh_degree_in_use);

/* Copies the current cloud to host memory (capacity in gaussians). */
int pxs_trainer_download(pxs_trainer* trainer, float* params, int32_t capacity,
                         int32_t* count);

/* SplatTrainer::finish (SplatTrainer.cpp:378-383): prune below
 * prune_opacity, stable sort by descending opacity logit, copy out. */
int pxs_trainer_finish(pxs_trainer* trainer, float* params, int32_t capacity, int32_t* count);

/* trainSplatsOnGpu (VulkanSplatTrainer.h:35-37, VulkanSplatTrainer.cpp:885-907)
 * on SoA buffers: trains `cloud` in place and writes the finished cloud back
 * into cloud->params, updating cloud->count (the buffer must hold
 * config->max_gaussians gaussians). A cancelled run still writes back. */
int pxs_train_splats(pxs_cloud* cloud, const pxs_camera* cameras, const float* const* images,
                     int32_t n_views, const pxs_train_config* config,
                     pxs_progress_fn callback, void* user, char* error, size_t error_len);

/* densifyAndPrune (SplatDensify.h:55-57; SplatDensify.cpp:28-109) on host
 * buffers, run as flag, scan and compaction kernels. `params` must hold room
 * for config->max_gaussians gaussians; `count` is updated in place.
 * `source_index` (room for max_gaussians) receives each new gaussian's old
 * index or -1; `rng_state` is advanced like the reference's. `stats` are the
 * accumulated screen gradient and visible count per gaussian. */
int pxs_densify_and_prune(pxs_context* context, float* params, int32_t* count,
                          int32_t rest_per_channel, const float* screen_gradient,
                          const int32_t* visible_count, const pxs_train_config* config,
                          float extent, int32_t iteration, uint32_t* rng_state,
                          int32_t* source_index, int32_t* cloned, int32_t* split,
                          int32_t* pruned);

/* initializeFromPointCloud (GaussianCloud.cpp:199-257), the pipeline's seed
 * for training: one isotropic gaussian per point (n points, x y z floats),
 * sigma half the mean nearest-neighbour distance over a sample of at most 512
 * points (searched on the device), identity rotation, opacity logit from
 * `initial_opacity`, DC from the point's 8-bit colour (`colors` may be NULL),
 * zero higher SH. sh_degree is clamped to 0..3; `rest_per_channel` receives
 * its SH-rest count and `params` (may be NULL to ask only for that) receives
 * the component-major cloud, 14 + 3 * rest_per_channel rows of n. */
int pxs_initialize_from_points(pxs_context* context, const float* points,
                               const uint8_t* colors, int32_t n, int32_t sh_degree,
                               float initial_opacity, float* params,
                               int32_t* rest_per_channel);

/* ---------------------------------------------------------- image ingest
 * The training images of Pipeline::Impl::runSplatTraining
 * (Pipeline.cpp:1892-1917): an 8-bit RGB frame box-filtered to a target width
 * by downscaleToWidth (ImageIo.cpp:300-337, the frame unchanged when it is no
 * wider), each byte then divided by 255. pxs_downscale_to_width runs it on the
 * device for host buffers: out_rgb gets the downscaled bytes and out_linear
 * the floats (either may be NULL; with both NULL only the size is written).
 * pxs_trainer_ingest_images replaces the resident images of `view_ids` from
 * 8-bit frames, downscaled to each view's width on the device (the result
 * must have the view's size); only the 8-bit frames cross to the device. */
int pxs_downscale_to_width(pxs_context* context, const uint8_t* rgb, int32_t width,
                           int32_t height, int32_t target_width, uint8_t* out_rgb,
                           float* out_linear, int32_t* out_width, int32_t* out_height);
int pxs_trainer_ingest_images(pxs_trainer* trainer, int32_t n, const int32_t* view_ids,
                              const uint8_t* const* frames, const int32_t* widths,
                              const int32_t* heights);

/* The same ingest, asynchronous, for a training loop that feeds each step's
 * frames from host memory: the frames are copied to the device on the
 * trainer's own copy stream, into one of two staging buffers, while the
 * steps before the one that needs them run, and are downscaled and converted
 * into the views' training images (as pxs_trainer_ingest_images does) by the
 * first step call (pxs_trainer_step, _step_batch, _step_views, _accumulate)
 * whose views include one of theirs; _ingest_images, _set_images and
 * _autotune apply every staged set first, and a stage call with both buffers
 * busy applies the older set. Sets take effect in the order they were
 * staged. So a loop that stages step s+1's frames and then runs step s
 * copies them while step s runs. The frames must stay valid and unchanged
 * until the call that applies them returns; page-locked frames let the copy
 * overlap the step.
 * No reference counterpart: the reference converts on the host before
 * training (Pipeline.cpp:1892-1917). */
int pxs_trainer_stage_images(pxs_trainer* trainer, int32_t n, const int32_t* view_ids,
                             const uint8_t* const* frames, const int32_t* widths,
                             const int32_t* heights);

/* ------------------------------------------------------- trained-cloud files
 * The reference's writers (GaussianCloud.h:95-131) into memory: the bytes of
 * the file writeGaussianPly (GaussianCloud.cpp:259-306), writeSplat
 * (:414-443) or writeSpz (:493-550; `fractional_bits` clamped to 0..20 as
 * there) would write for the cloud. The body is packed on the device
 * (transposed and quantised) and copied back once; .spz is then gzipped on the
 * host with the reference's deflate settings. `out` receives at most
 * `capacity` bytes and `size` the file's size; with `out` NULL or too small
 * the call returns PXS_ERR_CAPACITY and only sets `size`. An empty cloud is
 * PXS_ERR_INVALID (the reference returns false), as is .spz above SH
 * degree 3. */
#define PXS_FORMAT_PLY 0
#define PXS_FORMAT_SPLAT 1
#define PXS_FORMAT_SPZ 2
int pxs_export_cloud(pxs_context* context, const pxs_cloud* cloud, int32_t format,
                     int32_t fractional_bits, uint8_t* out, size_t capacity, size_t* size);
/* The same for a trainer's current cloud, already on the device (a trainer
 * over several scenes is refused: download and split it instead). */
int pxs_trainer_export(pxs_trainer* trainer, int32_t format, int32_t fractional_bits,
                       uint8_t* out, size_t capacity, size_t* size);

/* -------------------------------------------------------- synthetic scenes
 * Seeded generators for the benchmark workloads. The generator is the
 * reference's xorshift64 Rng with a Box-Muller normal
 * (engine/native/cpp/include/parallax/testing/SyntheticScene.h:80-107). */

/* means U[-1,1]^3, log sigma N(log_scale_mean, 0.5), random unit quaternions,
 * opacity logits N(0,1), dc with 0.5 + C0*dc ~ N(0.5, 0.1), sh_rest N(0, 0.1). */
int pxs_synthetic_cloud(uint64_t seed, int32_t count, int32_t rest_per_channel,
                        float log_scale_mean, float* params);

/* `count` cameras on a sphere of `radius` looking at the origin with the given
 * horizontal field of view. layout 0: Fibonacci sphere; layout 1: half on the
 * upper hemisphere, half on a ring at jittered height +-0.2 and radius +-0.1. */
int pxs_synthetic_cameras(uint64_t seed, int32_t count, int32_t layout, double radius,
                          int32_t width, int32_t height, double fov_degrees, pxs_camera* out);

#ifdef __cplusplus
}
#endif

#endif /* PXS_H */
