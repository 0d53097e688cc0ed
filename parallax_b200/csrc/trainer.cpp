// trainer.cpp -- the device-resident trainer behind pxs_trainer_* and
// pxs_train_splats.
//
// The schedule is SplatTrainer's (SplatTrainer.cpp:163-383): one view per
// step from a std::mt19937-driven std::shuffle of the views (the same
// libstdc++ algorithm, so the same order for the same seed), SH bands
// unlocked every sh_increase_interval, a geometric position learning rate
// scaled by the camera extent, Adam with bias correction at t = iteration+1,
// densify/prune every densify_interval inside [from, until], opacity reset
// every opacity_reset_interval before densify_until. Per-step scalars are
// computed on the host with the same libm as the reference (std::pow,
// std::log) and handed to the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "densify.h"
#include "runtime.h"

namespace pxs {

struct GraphState {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int N = -1, V = -1;
  int64_t pixels = -1, pair_capacity = -1, record_capacity = -1;
  int tiles = -1;
  int generation = -1;
  int raster_generation = -1;
  int64_t allocations = -1;
  bool timing = false;
  int64_t launches = 0;
  void reset() {
    if (exec != nullptr) cudaGraphExecDestroy(exec);
    if (graph != nullptr) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    N = V = tiles = generation = raster_generation = -1;
    pixels = pair_capacity = record_capacity = allocations = -1;
  }
};

}  // namespace pxs

using pxs::DeviceArray;
using pxs::Error;

struct pxs_trainer {
  pxs_train_config cfg;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string error;

  int N = 0, S = 0, P = 14, cloud_sh = 0;
  DeviceArray<float> params, m, v, acc_gradient;
  DeviceArray<int32_t> visible_count, acc_views;
  // The step's sums in one allocation, so a data-parallel caller sums them
  // over the ranks with one collective: the parameter gradients (P x N), the
  // screen gradient (N), the visible counts as floats (N, exact integers; the
  // kernels count in visible_count and accumulate() copies them here) and a
  // loss tail (the mean loss of this rank's views times their number, and the
  // number), from which apply() takes the mean over all ranks' views.
  DeviceArray<float> grad_block;
  size_t n_alloc() const { return static_cast<size_t>(std::max(N, 1)); }
  float* d_grads() const { return grad_block.get(); }
  float* d_screen() const { return grad_block.get() + static_cast<size_t>(P) * n_alloc(); }
  float* d_visible_f() const { return d_screen() + n_alloc(); }
  float* d_loss_tail() const { return d_visible_f() + n_alloc(); }
  size_t block_values() const { return static_cast<size_t>(P + 2) * n_alloc() + 2; }
  DeviceArray<float> next_params, next_m, next_v;

  std::vector<pxs_camera> cameras;
  std::vector<int64_t> image_offset;  // first pixel of each view in `images`
  bool uniform_views = true;          // every view has the same size
  DeviceArray<float> images;
  DeviceArray<uint8_t> ingest_in;  // staging for 8-bit frames

  // Frames staged for coming steps (pxs_trainer_stage_images): each set is
  // copied to the device on copy_stream into one of two staging buffers while
  // the steps before it run, and converted into the image store on `stream`
  // by the first step that uses one of its views (older sets first, so images
  // are replaced in the order they were staged). A staging buffer is refilled
  // only after the conversion that read it (consumed_event) has run.
  struct StagedFrame {
    int view, width, height, out_width, out_height;
    size_t offset;
  };
  struct StagedSet {
    int slot;
    std::vector<StagedFrame> frames;
  };
  cudaStream_t copy_stream = nullptr;
  DeviceArray<uint8_t> stage_buf[2];
  cudaEvent_t staged_event[2] = {}, consumed_event[2] = {};
  bool consumed_recorded[2] = {false, false};
  std::vector<StagedSet> pending;  // oldest first, at most two

  int iteration = 0;
  float extent = 1.f, last_loss = 0.f, smoothed_loss = 0.f;
  // several independent scenes in one cloud (pxs_trainer_create_scenes): the
  // gaussian range and camera extent of each scene, the scene of each view,
  // and per gaussian its scene's extent for the position learning rate
  int n_scenes = 1;
  std::vector<int32_t> scene_offset, scene_count;
  std::vector<int> view_scene;
  std::vector<float> scene_extent;
  DeviceArray<float> position_scale;
  std::mt19937 engine;
  std::vector<int> order;
  size_t cursor = 0;
  uint32_t densify_rng = 1u;

  pxs::Frame frame;
  pxs::DensifyWork dwork;
  DeviceArray<pxs::StepScalars> scalars;
  DeviceArray<float> dL, loss_acc;
  std::string tune_log;       // the autotuner's timings, one line per candidate
  pxs::GraphState graph;      // the batched step
  pxs::GraphState graph_acc;  // its data-parallel accumulate half
  pxs::GraphState graph_one;  // the one-view step (step())
  bool pending_apply = false;
  int generation = 0;  // bumped whenever a state buffer is reallocated
  float* host_loss = nullptr;     // pinned
  int32_t* host_overflow = nullptr;
  int64_t* host_pairs = nullptr;  // pinned: the last batched step's pair count

  // stage timing: events recorded between the stages of the batched step
  // (captured as event nodes when the step is a graph)
  static constexpr int kStages = 7;
  bool timing = false;
  cudaEvent_t events[kStages + 1] = {};
  double stage_ms[kStages] = {};
  int timed_steps = 0;
  int64_t last_pairs = 0;
  int64_t last_launches = 0;
  DeviceArray<unsigned long long> pair_counts;

  ~pxs_trainer() {
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    graph.reset();
    graph_acc.reset();
    graph_one.reset();
    for (int k = 0; k < 2; ++k) {
      if (staged_event[k]) cudaEventDestroy(staged_event[k]);
      if (consumed_event[k]) cudaEventDestroy(consumed_event[k]);
    }
    if (copy_stream) cudaStreamDestroy(copy_stream);
    for (cudaEvent_t& e : events)
      if (e) cudaEventDestroy(e);
    if (host_loss) cudaFreeHost(host_loss);
    if (host_overflow) cudaFreeHost(host_overflow);
    if (host_pairs) cudaFreeHost(host_pairs);
    if (stream) cudaStreamDestroy(stream);
  }

  // ---------------------------------------------------------- schedule

  // SplatTrainer::Impl::shDegreeInUse (SplatTrainer.cpp:193-198)
  int sh_degree_in_use() const {
    const int unlocked = cfg.sh_increase_interval > 0 ? iteration / cfg.sh_increase_interval
                                                      : cfg.sh_degree;
    return std::min(cfg.sh_degree, std::max(0, unlocked));
  }

  // positionLearningRate (SplatTrainer.cpp:200-208)
  float position_lr() const {
    const float t = cfg.iterations <= 1
                        ? 1.f
                        : static_cast<float>(iteration) / static_cast<float>(cfg.iterations - 1);
    const float ratio = cfg.position_lr_final / std::max(cfg.position_lr_initial, 1e-30f);
    const float base = cfg.position_lr_initial * std::pow(ratio, std::clamp(t, 0.f, 1.f));
    // several scenes: the Adam kernel multiplies by each gaussian's scene extent
    return n_scenes > 1 ? base : base * extent;
  }

  const float* position_scales() const { return n_scenes > 1 ? position_scale.get() : nullptr; }

  // nextView (SplatTrainer.cpp:210-216)
  int next_view() {
    if (cursor >= order.size()) {
      std::shuffle(order.begin(), order.end(), engine);
      cursor = 0;
    }
    return order[cursor++];
  }

  pxs::StepScalars step_scalars() const {
    pxs::StepScalars s;
    std::memset(&s, 0, sizeof(s));
    s.lr[0] = position_lr();
    s.lr[1] = cfg.scale_lr;
    s.lr[2] = cfg.rotation_lr;
    s.lr[3] = cfg.opacity_lr;
    s.lr[4] = cfg.dc_lr;
    s.lr[5] = cfg.dc_lr / std::max(1.f, cfg.sh_rest_lr_divider);
    s.beta1 = cfg.adam_beta1;
    s.beta2 = cfg.adam_beta2;
    s.epsilon = cfg.adam_epsilon;
    const int t = iteration + 1;
    s.correction1 = 1.f - std::pow(cfg.adam_beta1, static_cast<float>(t));
    s.correction2 = 1.f - std::pow(cfg.adam_beta2, static_cast<float>(t));
    return s;
  }

  pxs_raster_options options() const {
    pxs_raster_options o;
    o.background[0] = o.background[1] = o.background[2] = 0.f;
    o.sh_degree = sh_degree_in_use();
    o.min_alpha = 1.f / 255.f;
    o.transmittance_cutoff = 1e-4f;
    o.screen_dilation = 0.3f;
    return o;
  }

  pxs::ViewBatch batch_for(const std::vector<int>& ids) const {
    std::vector<pxs_camera> cams;
    for (int id : ids) cams.push_back(cameras[static_cast<size_t>(id)]);
    pxs::ViewBatch b = pxs::make_batch(cams.data(), static_cast<int>(cams.size()), options(),
                                       cloud_sh);
    for (size_t i = 0; i < ids.size(); ++i)
      b.views[i].target_offset = image_offset[static_cast<size_t>(ids[i])];
    if (n_scenes > 1) {
      b.own_ranges = true;
      for (size_t i = 0; i < ids.size(); ++i) {
        const int sc = view_scene[static_cast<size_t>(ids[i])];
        b.views[i].gauss_offset = scene_offset[static_cast<size_t>(sc)];
        b.views[i].gauss_count = scene_count[static_cast<size_t>(sc)];
      }
    }
    return b;
  }

  void upload_scalars() {
    const pxs::StepScalars s = step_scalars();
    PXS_CUDA(cudaMemcpyAsync(scalars.get(), &s, sizeof(s), cudaMemcpyHostToDevice, stream));
  }

  void adam() {
    pxs::launch_adam(params.get(), d_grads(), m.get(), v.get(), N, S, scalars.get(), 1,
                     d_screen(), visible_count.get(), acc_gradient.get(),
                     acc_views.get(), stream, position_scales());
    PXS_CUDA(cudaGetLastError());
  }

  // The tail of SplatTrainer::step after the optimiser (SplatTrainer.cpp:349-360).
  void after_step() {
    ++iteration;
    if (n_scenes == 1 && iteration >= cfg.densify_from_iteration &&
        iteration <= cfg.densify_until_iteration && iteration % cfg.densify_interval == 0) {
      densify();
    }
    if (cfg.opacity_reset_interval > 0 && iteration % cfg.opacity_reset_interval == 0 &&
        iteration < cfg.densify_until_iteration) {
      // resetOpacity (SplatTrainer.cpp:301-309), sigmoidInverse (:67-70)
      const float clamped = std::clamp(cfg.opacity_reset_value, 1e-6f, 1.f - 1e-6f);
      const float ceiling = std::log(clamped / (1.f - clamped));
      pxs::launch_reset_opacity(params.get(), m.get(), v.get(), N, ceiling, stream);
      PXS_CUDA(cudaGetLastError());
    }
  }

  void record_loss(float loss) {
    last_loss = loss;
    smoothed_loss = iteration == 0 ? loss : 0.99f * smoothed_loss + 0.01f * loss;
  }

  // densifyAndPrune + remapState (SplatTrainer.cpp:267-299)
  void densify() {
    pxs::DensifyArgs a;
    a.grad_threshold = cfg.densify_grad_threshold;
    a.size_threshold = cfg.percent_dense * extent;
    a.max_scale = cfg.prune_scale_fraction * extent;
    a.prune_opacity = cfg.prune_opacity;
    a.log_split_divider = std::log(cfg.split_scale_divider);
    a.prune_oversized = iteration > cfg.opacity_reset_interval ? 1 : 0;
    a.has_room = N < cfg.max_gaussians ? 1 : 0;
    a.max_gaussians = cfg.max_gaussians;
    a.rng_state = densify_rng;
    const int64_t cap = std::max<int64_t>(static_cast<int64_t>(cfg.max_gaussians),
                                          static_cast<int64_t>(N) * 3);
    const size_t values = static_cast<size_t>(P) * static_cast<size_t>(cap);
    next_params.reserve(values);
    next_m.reserve(values);
    next_v.reserve(values);
    const pxs::DensifyResult r = pxs::densify_device(
        dwork, params.get(), m.get(), v.get(), N, S, acc_gradient.get(), acc_views.get(), a,
        next_params.get(), next_m.get(), next_v.get(), nullptr, cap, stream);
    densify_rng = r.rng_state;
    params.swap(next_params);
    m.swap(next_m);
    v.swap(next_v);
    N = static_cast<int>(r.count);
    resize_state();
  }

  // Gradients and statistics for the current count, zeroed.
  void resize_state() {
    ++generation;
    const size_t n = static_cast<size_t>(std::max(N, 1));
    grad_block.reserve(block_values());
    visible_count.reserve(n);
    acc_gradient.reserve(n);
    acc_views.reserve(n);
    PXS_CUDA(cudaMemsetAsync(grad_block.get(), 0, sizeof(float) * block_values(), stream));
    PXS_CUDA(cudaMemsetAsync(visible_count.get(), 0, sizeof(int32_t) * n, stream));
    PXS_CUDA(cudaMemsetAsync(acc_gradient.get(), 0, sizeof(float) * n, stream));
    PXS_CUDA(cudaMemsetAsync(acc_views.get(), 0, sizeof(int32_t) * n, stream));
  }

  // ---------------------------------------------------------- staged ingest

  // Enqueues, on `stream`, the conversion of the oldest `count` staged sets
  // into the image store, each after its copy; their buffers are then free.
  void convert_staged(size_t count) {
    for (size_t i = 0; i < count && i < pending.size(); ++i) {
      const StagedSet& set = pending[i];
      const int k = set.slot;
      PXS_CUDA(cudaStreamWaitEvent(stream, staged_event[k], 0));
      // frames at their view's size go through one launch for the set; the
      // others are downscaled one by one
      std::vector<const uint8_t*> src;
      std::vector<float*> dst;
      std::vector<int64_t> bytes;
      for (const StagedFrame& f : set.frames) {
        const uint8_t* in = stage_buf[k].get() + f.offset;
        float* out = images.get() + image_offset[static_cast<size_t>(f.view)] * 3;
        const int64_t n = static_cast<int64_t>(f.width) * f.height * 3;
        if (f.width == f.out_width && f.height == f.out_height &&
            pxs::linear_frame_ok(in, out, n)) {
          src.push_back(in);
          dst.push_back(out);
          bytes.push_back(n);
          continue;
        }
        pxs::launch_downscale(in, f.width, f.height, f.out_width, f.out_height, nullptr, out,
                              stream);
        PXS_CUDA(cudaGetLastError());
      }
      if (!src.empty()) {
        pxs::launch_bytes_to_linear_frames(src.data(), dst.data(), bytes.data(),
                                           static_cast<int>(src.size()), stream);
        PXS_CUDA(cudaGetLastError());
      }
      PXS_CUDA(cudaEventRecord(consumed_event[k], stream));
      consumed_recorded[k] = true;
    }
    pending.erase(pending.begin(), pending.begin() + std::min(count, pending.size()));
  }

  // Every staged set, before images are replaced another way.
  void consume_staged() { convert_staged(pending.size()); }

  // The staged sets a step over `views` needs: up to the newest set holding
  // one of them (older sets first). Sets for later steps stay in flight.
  void consume_staged_for(const std::vector<int>& views) {
    size_t need = 0;
    for (size_t i = 0; i < pending.size(); ++i)
      for (const StagedFrame& f : pending[i].frames)
        if (std::find(views.begin(), views.end(), f.view) != views.end()) need = i + 1;
    convert_staged(need);
  }

  void stage_frames(int n, const int32_t* ids, const uint8_t* const* frames,
                    const int32_t* widths, const int32_t* heights) {
    std::vector<StagedFrame> staged;
    size_t total = 0;
    for (int i = 0; i < n; ++i) {
      const int id = ids[i];
      if (id < 0 || id >= static_cast<int>(cameras.size()))
        throw Error(PXS_ERR_INVALID, "view id out of range");
      const pxs_camera& cam = cameras[static_cast<size_t>(id)];
      int w = 0, h = 0;
      pxs::downscaled_size(widths[i], heights[i], cam.width, &w, &h);
      if (w != cam.width || h != cam.height)
        throw Error(PXS_ERR_INVALID, "the downscaled frame does not match the view's size");
      const size_t bytes = static_cast<size_t>(widths[i]) * heights[i] * 3;
      if (bytes == 0) continue;
      if (frames[i] == nullptr) throw Error(PXS_ERR_INVALID, "frame is null");
      staged.push_back({id, widths[i], heights[i], w, h, total});
      total += (bytes + 255) / 256 * 256;
    }
    if (staged.empty()) return;
    if (copy_stream == nullptr) {
      PXS_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
      for (int k = 0; k < 2; ++k) {
        PXS_CUDA(cudaEventCreateWithFlags(&staged_event[k], cudaEventDisableTiming));
        PXS_CUDA(cudaEventCreateWithFlags(&consumed_event[k], cudaEventDisableTiming));
      }
    }
    // both buffers hold sets no step has used yet: the older one takes effect
    // now, which frees its buffer
    if (pending.size() == 2) convert_staged(1);
    const int k = pending.empty() ? 0 : 1 - pending.front().slot;
    if (total > stage_buf[k].capacity()) {
      // grown only when both streams are idle
      PXS_CUDA(cudaStreamSynchronize(stream));
      PXS_CUDA(cudaStreamSynchronize(copy_stream));
      stage_buf[k].reserve(total);
    }
    if (consumed_recorded[k]) PXS_CUDA(cudaStreamWaitEvent(copy_stream, consumed_event[k], 0));
    for (size_t i = 0, j = 0; i < static_cast<size_t>(n); ++i) {
      const size_t bytes = static_cast<size_t>(widths[i]) * heights[i] * 3;
      if (bytes == 0) continue;
      const StagedFrame& f = staged[j++];
      PXS_CUDA(cudaMemcpyAsync(stage_buf[k].get() + f.offset, frames[i], bytes,
                               cudaMemcpyHostToDevice, copy_stream));
    }
    PXS_CUDA(cudaEventRecord(staged_event[k], copy_stream));
    pending.push_back({k, std::move(staged)});
  }

  // ---------------------------------------------------------- steps

  bool schedule_done() {
    if (iteration >= cfg.iterations) return true;
    if (cameras.empty() || N == 0) {
      iteration = cfg.iterations;
      return true;
    }
    return false;
  }

  // SplatTrainer::step (SplatTrainer.cpp:326-362): one view, synchronised.
  // The batched step over that one view: its pair and record buffers are
  // sized once with headroom (no host round trip inside the step) and, when
  // every view has the same size, the step is one replay of its own graph.
  bool step() {
    if (schedule_done()) return false;
    const int id = next_view();
    consume_staged_for({id});
    run_batch({id}, uniform_views, true, graph_one);
    record_loss(*host_loss);
    after_step();
    return true;
  }

  std::vector<int> take_views(int n_views, const int32_t* ids) {
    std::vector<int> out;
    for (int i = 0; i < n_views; ++i) {
      const int id = ids != nullptr ? ids[i] : next_view();
      if (id < 0 || id >= static_cast<int>(cameras.size()))
        throw Error(PXS_ERR_INVALID, "view id out of range");
      out.push_back(id);
    }
    consume_staged_for(out);
    return out;
  }

  // Plain multi-view step: per-view kernel sequences, host-synchronised pair
  // counts, no graph; gradients accumulate over the views, then one Adam.
  float step_views(int n_views, const int32_t* ids) {
    if (schedule_done()) return 0.f;
    const int64_t before = pxs::g_kernel_launches;
    last_pairs = 0;
    const std::vector<int> views = take_views(n_views, ids);
    float* acc = loss_acc.reserve(static_cast<size_t>(views.size()) + 1);
    for (size_t i = 0; i < views.size(); ++i) {
      const pxs::ViewBatch b = batch_for({views[i]});
      frame.prepare(b, N, S, stream);
      frame.project(params.get(), stream);
      last_pairs += frame.bin(true, stream);
      frame.forward(stream);
      float* d_dL = dL.reserve(static_cast<size_t>(b.total_pixels) * 3 + 1);
      frame.loss(images.get(), cfg.ssim_weight, 0, d_dL, stream);
      frame.backward(d_dL, stream);
      frame.param_grads(params.get(), d_grads(), d_screen(), visible_count.get(),
                        stream);
      PXS_CUDA(cudaMemcpyAsync(acc + i, frame.loss_total.get(), sizeof(float),
                               cudaMemcpyDeviceToDevice, stream));
    }
    std::vector<float> losses(views.size());
    PXS_CUDA(cudaMemcpyAsync(losses.data(), acc, sizeof(float) * views.size(),
                             cudaMemcpyDeviceToHost, stream));
    upload_scalars();
    adam();
    last_launches = pxs::g_kernel_launches - before;
    PXS_CUDA(cudaStreamSynchronize(stream));
    float sum = 0.f;
    for (float l : losses) sum += l;
    const float loss = views.empty() ? 0.f : sum / static_cast<float>(views.size());
    record_loss(loss);
    after_step();
    return loss;
  }

  void mark(int i) {
    if (timing) PXS_CUDA(cudaEventRecordWithFlags(events[i], stream, cudaEventRecordExternal));
  }

  void set_timing(bool on) {
    if (on && events[0] == nullptr)
      for (cudaEvent_t& e : events) PXS_CUDA(cudaEventCreate(&e));
    timing = on;
    for (double& ms : stage_ms) ms = 0.0;
    timed_steps = 0;
  }

  void collect_timing() {
    if (!timing) return;
    for (int i = 0; i < kStages; ++i) {
      float ms = 0.f;
      PXS_CUDA(cudaEventElapsedTime(&ms, events[i], events[i + 1]));
      stage_ms[i] += ms;
    }
    ++timed_steps;
  }

  // Enqueues the batched step body (everything after the view upload); the
  // optimiser step is left out for the data-parallel split (accumulate).
  void enqueue_batch_body(bool with_adam) {
    mark(0);
    frame.project(params.get(), stream);
    mark(1);
    frame.bin(false, stream);
    mark(2);
    frame.forward(stream);
    mark(3);
    frame.loss(images.get(), cfg.ssim_weight, 0, dL.get(), stream);
    mark(4);
    frame.backward(dL.get(), stream);
    mark(5);
    frame.param_grads(params.get(), d_grads(), d_screen(), visible_count.get(),
                      stream);
    mark(6);
    if (!with_adam)
      pxs::launch_pack_reduction(visible_count.get(), d_visible_f(), N, frame.loss_total.get(),
                                 frame.V, d_loss_tail(), stream);
    if (with_adam)
      pxs::launch_adam_checked(params.get(), d_grads(), m.get(), v.get(), N, S, scalars.get(),
                               d_screen(), visible_count.get(), acc_gradient.get(),
                               acc_views.get(), frame.overflow.get(), stream,
                               position_scales());
    mark(7);
    PXS_CUDA(cudaMemcpyAsync(host_loss, frame.loss_total.get(), sizeof(float),
                             cudaMemcpyDeviceToHost, stream));
    PXS_CUDA(cudaMemcpyAsync(host_overflow, frame.overflow.get(), sizeof(int32_t),
                             cudaMemcpyDeviceToHost, stream));
    PXS_CUDA(cudaMemcpyAsync(host_pairs, frame.d_total_pairs.get(), sizeof(int64_t),
                             cudaMemcpyDeviceToHost, stream));
  }

  // Runs the batched body for `views`, replayed from `g` when use_graph, and
  // redoes it with larger pair buffers while the pairs overflow. The
  // optimiser, when included, skips a step whose pairs overflowed.
  void run_batch(const std::vector<int>& views, bool use_graph, bool with_adam,
                 pxs::GraphState& g) {
    const pxs::ViewBatch b = batch_for(views);
    frame.prepare(b, N, S, stream);  // also uploads the view descriptors
    dL.reserve(static_cast<size_t>(b.total_pixels) * 3 + 1);
    if (frame.pair_capacity == 0 || frame.record_capacity == 0) {
      // learn the pair count once, then run unsynchronised with headroom
      frame.project(params.get(), stream);
      const int64_t K = frame.bin(true, stream);
      frame.reserve_pairs(K + K / 2 + 65536);
      frame.reserve_records(frame.last_record_count + frame.last_record_count / 2 + 65536);
    }
    for (int attempt = 0; attempt < 3; ++attempt) {
      upload_scalars();
      if (use_graph) {
        const bool stale = g.exec == nullptr || g.N != N || g.V != frame.V ||
                           g.timing != timing || g.pixels != b.total_pixels ||
                           g.tiles != b.total_tiles || g.pair_capacity != frame.pair_capacity ||
                           g.record_capacity != frame.record_capacity ||
                           g.generation != generation ||
                           g.raster_generation != pxs::raster_config().generation ||
                           g.allocations != pxs::g_device_allocations;
        if (stale) {
          g.reset();
          const int64_t before = pxs::g_kernel_launches;
          PXS_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
          try {
            enqueue_batch_body(with_adam);
          } catch (...) {
            cudaGraph_t dropped = nullptr;
            cudaStreamEndCapture(stream, &dropped);
            if (dropped) cudaGraphDestroy(dropped);
            throw;
          }
          PXS_CUDA(cudaStreamEndCapture(stream, &g.graph));
          PXS_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
          g.N = N;
          g.V = frame.V;
          g.pixels = b.total_pixels;
          g.tiles = b.total_tiles;
          g.pair_capacity = frame.pair_capacity;
          g.record_capacity = frame.record_capacity;
          g.generation = generation;
          g.raster_generation = pxs::raster_config().generation;
          g.allocations = pxs::g_device_allocations;
          g.timing = timing;
          g.launches = pxs::g_kernel_launches - before;
        }
        PXS_CUDA(cudaGraphLaunch(g.exec, stream));
        last_launches = g.launches;
      } else {
        const int64_t before = pxs::g_kernel_launches;
        enqueue_batch_body(with_adam);
        last_launches = pxs::g_kernel_launches - before;
      }
      PXS_CUDA(cudaStreamSynchronize(stream));
      if (*host_overflow == 0) {
        collect_timing();
        last_pairs = *host_pairs;
        return;
      }
      // the pairs did not fit: nothing of this step counts; grow and redo
      PXS_CUDA(cudaMemsetAsync(d_grads(), 0, sizeof(float) * (P + 1) * n_alloc(), stream));
      PXS_CUDA(cudaMemsetAsync(visible_count.get(), 0, sizeof(int32_t) * std::max(N, 1), stream));
      frame.project(params.get(), stream);
      const int64_t K = frame.bin(true, stream);
      frame.reserve_pairs(K + K / 2 + 65536);
      frame.reserve_records(frame.last_record_count + frame.last_record_count / 2 + 65536);
      g.reset();
    }
    throw Error(PXS_ERR_CAPACITY, "tile pairs overflowed three times");
  }

  // Times the compositing kernels with 1, 2 and 4 pixels per thread on one
  // batch of views and keeps the fastest forward + backward pair.
  // The schedule, the parameters and the gradients are left as they were.
  void autotune(int n_views, const int32_t* ids, int* forward_px, int* backward_px) {
    consume_staged();  // the loss reads the training images
    tune_log.clear();
    std::vector<int> views;
    for (int i = 0; i < n_views; ++i) {
      const int id = ids != nullptr ? ids[i] : i % static_cast<int>(cameras.size());
      if (id < 0 || id >= static_cast<int>(cameras.size()))
        throw Error(PXS_ERR_INVALID, "view id out of range");
      views.push_back(id);
    }
    const pxs::ViewBatch b = batch_for(views);
    frame.prepare(b, N, S, stream);
    frame.project(params.get(), stream);
    frame.bin(true, stream);
    float* d_dL = dL.reserve(static_cast<size_t>(b.total_pixels) * 3 + 1);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PXS_CUDA(cudaEventCreate(&e0));
    PXS_CUDA(cudaEventCreate(&e1));
    auto time_ms = [&](auto&& body) {
      body();  // warm
      PXS_CUDA(cudaEventRecord(e0, stream));
      for (int r = 0; r < 3; ++r) body();
      PXS_CUDA(cudaEventRecord(e1, stream));
      PXS_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      PXS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      return ms;
    };
    pxs::RasterConfig& rc = pxs::raster_config();
    const int candidates[3] = {1, 2, 4};
    // the pair is timed together: the two-pixel forward also records which
    // blocks took each entry, which the two-pixel adjoint then skips by
    float best = 0.f;
    bool have_best = false;
    int best_fwd = rc.forward_px, best_bwd = rc.backward_px;
    try {
      for (int fpx : candidates) {
        rc.forward_px = fpx;
        const float f_ms = time_ms([&] { frame.forward(stream); });
        frame.loss(images.get(), cfg.ssim_weight, 0, d_dL, stream);
        for (int bpx : candidates) {
          rc.backward_px = bpx;
          const float b_ms = time_ms([&] { frame.backward(d_dL, stream); });
          const float ms = f_ms + b_ms;
          tune_log += "pixels per thread " + std::to_string(fpx) + "/" + std::to_string(bpx) +
                      ": forward " + std::to_string(f_ms / 3.f) + " ms, adjoint " +
                      std::to_string(b_ms / 3.f) + " ms\n";
          if (!have_best || ms < best) {
            best = ms;
            best_fwd = fpx;
            best_bwd = bpx;
            have_best = true;
          }
        }
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    rc.forward_px = best_fwd;
    rc.backward_px = best_bwd;
    // then, for the two-pixel forms, the per-block batch and the tile
    // schedule of each kernel, one knob at a time, the others held
    try {
      auto tune = [&](const char* what, int& knob, std::initializer_list<int> values,
                      auto&& measure) {
        int best_value = knob;
        float best_ms = 0.f;
        bool have = false;
        for (int value : values) {
          knob = value;
          const float ms = measure();
          tune_log += std::string(what) + " " + std::to_string(value) + ": " +
                      std::to_string(ms / 3.f) + " ms\n";
          if (!have || ms < best_ms) {
            best_ms = ms;
            best_value = value;
            have = true;
          }
        }
        knob = best_value;
      };
      auto fwd_ms = [&] { return time_ms([&] { frame.forward(stream); }); };
      auto bwd_ms = [&] {
        frame.forward(stream);  // block bits and the last contributors of this forward
        return time_ms([&] { frame.backward(d_dL, stream); });
      };
      if (rc.forward_px == 2) {
        tune("forward batch", rc.forward_batch, {64, 128, 256}, fwd_ms);
        tune("forward schedule", rc.forward_schedule, {0, 1, 2}, fwd_ms);
      }
      if (rc.backward_px == 2) {
        frame.forward(stream);
        frame.loss(images.get(), cfg.ssim_weight, 0, d_dL, stream);
        tune("adjoint batch", rc.backward_batch, {64, 128, 256}, bwd_ms);
        tune("adjoint schedule", rc.backward_schedule, {0, 1, 2}, bwd_ms);
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ++rc.generation;
    if (forward_px) *forward_px = best_fwd;
    if (backward_px) *backward_px = best_bwd;
  }

  // Batched step: every view of the batch in one pass of each kernel, one
  // Adam, optionally replayed from a captured CUDA graph.
  float step_batch(int n_views, const int32_t* ids, bool use_graph) {
    if (schedule_done()) return 0.f;
    const std::vector<int> views = take_views(n_views, ids);
    run_batch(views, use_graph, true, graph);
    record_loss(*host_loss);
    after_step();
    return *host_loss;
  }

  // The data-parallel split of step_batch. accumulate() renders and
  // differentiates this rank's views and leaves the summed gradients, screen
  // gradients and visible counts in the trainer's buffers, with no optimiser
  // step; the caller sums those buffers over the ranks; apply() then takes
  // the Adam step (and the schedule's densify and opacity reset) with the
  // summed gradients and records `loss`, the mean over all ranks' views.
  // Ranks that apply the same sums stay identical.
  float accumulate(int n_views, const int32_t* ids, bool use_graph) {
    if (schedule_done()) throw Error(PXS_ERR_INVALID, "the schedule is finished");
    if (pending_apply) throw Error(PXS_ERR_INVALID, "accumulate twice without apply");
    const std::vector<int> views = take_views(n_views, ids);
    run_batch(views, use_graph, false, graph_acc);
    pending_apply = true;
    return *host_loss;
  }

  void apply(float loss) {
    if (!pending_apply) throw Error(PXS_ERR_INVALID, "apply without accumulate");
    if (std::isnan(loss)) {
      // the mean over every rank's views, from the summed loss tail
      float tail[2];
      PXS_CUDA(cudaMemcpyAsync(tail, d_loss_tail(), sizeof(tail), cudaMemcpyDeviceToHost,
                               stream));
      PXS_CUDA(cudaStreamSynchronize(stream));
      loss = tail[1] > 0.f ? tail[0] / tail[1] : 0.f;
    }
    // the (summed) visible counts back to the integers the statistics keep
    pxs::launch_unpack_visible(d_visible_f(), visible_count.get(), N, stream);
    upload_scalars();
    adam();
    PXS_CUDA(cudaStreamSynchronize(stream));
    pending_apply = false;
    record_loss(loss);
    after_step();
  }
};

namespace {

template <typename F>
int guarded(pxs_trainer* t, F&& body) {
  if (t == nullptr) return PXS_ERR_INVALID;
  try {
    PXS_CUDA(cudaSetDevice(t->device));
    body();
    t->error.clear();
    return PXS_OK;
  } catch (const Error& e) {
    t->error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    t->error = "host allocation failed";
    return PXS_ERR_NO_MEMORY;
  } catch (const std::exception& e) {
    t->error = e.what();
    return PXS_ERR_INVALID;
  }
}

// cameraExtent (SplatTrainer.cpp:74-85) on the float camera centres.
float camera_extent(const std::vector<pxs_camera>& cams) {
  if (cams.empty()) return 1.f;
  float c[3] = {0.f, 0.f, 0.f};
  for (const pxs_camera& k : cams)
    for (int i = 0; i < 3; ++i) c[i] += k.center[i];
  for (int i = 0; i < 3; ++i) c[i] /= static_cast<float>(cams.size());
  float furthest = 0.f;
  for (const pxs_camera& k : cams) {
    const float d0 = k.center[0] - c[0], d1 = k.center[1] - c[1], d2 = k.center[2] - c[2];
    furthest = std::max(furthest, std::sqrt(d0 * d0 + (d1 * d1 + d2 * d2)));
  }
  return std::max(furthest * 1.1f, 1e-3f);
}

}  // namespace

extern "C" {

int pxs_trainer_create(const pxs_train_config* config, const pxs_cloud* initial,
                       const pxs_camera* cameras, const float* const* images, int32_t n_views,
                       int32_t device, pxs_trainer** out) {
  if (out == nullptr || config == nullptr || initial == nullptr) return PXS_ERR_INVALID;
  *out = nullptr;
  if (pxs_train_config_validate(config, nullptr, 0) != PXS_OK) return PXS_ERR_INVALID;
  if (n_views < 0 || (n_views > 0 && (cameras == nullptr || images == nullptr)))
    return PXS_ERR_INVALID;
  const int S = initial->rest_per_channel;
  if (initial->count < 0 || (S != 0 && S != 3 && S != 8 && S != 15)) return PXS_ERR_INVALID;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return PXS_ERR_UNAVAILABLE;
  }
  if (device < 0 || device >= count) return PXS_ERR_INVALID;
  auto* t = new (std::nothrow) pxs_trainer;
  if (t == nullptr) return PXS_ERR_NO_MEMORY;
  t->device = device;
  const int status = guarded(t, [&] {
    PXS_CUDA(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking));
    PXS_CUDA(cudaMallocHost(reinterpret_cast<void**>(&t->host_loss), sizeof(float)));
    PXS_CUDA(cudaMallocHost(reinterpret_cast<void**>(&t->host_overflow), sizeof(int32_t)));
    *t->host_overflow = 0;
    PXS_CUDA(cudaMallocHost(reinterpret_cast<void**>(&t->host_pairs), sizeof(int64_t)));
    *t->host_pairs = 0;
    t->cfg = *config;
    t->N = initial->count;
    t->S = S;
    t->P = PXS_PARAM_COUNT(S);
    t->cloud_sh = initial->sh_degree;
    const size_t values = static_cast<size_t>(t->P) * static_cast<size_t>(t->N);
    t->params.reserve(std::max<size_t>(values, 1));
    t->m.reserve(std::max<size_t>(values, 1));
    t->v.reserve(std::max<size_t>(values, 1));
    if (values > 0)
      PXS_CUDA(cudaMemcpyAsync(t->params.get(), initial->params, values * sizeof(float),
                               cudaMemcpyHostToDevice, t->stream));
    PXS_CUDA(cudaMemsetAsync(t->m.get(), 0, std::max<size_t>(values, 1) * sizeof(float), t->stream));
    PXS_CUDA(cudaMemsetAsync(t->v.get(), 0, std::max<size_t>(values, 1) * sizeof(float), t->stream));
    t->resize_state();
    t->cameras.assign(cameras, cameras + n_views);
    for (int v = 1; v < n_views; ++v)
      if (cameras[v].width != cameras[0].width || cameras[v].height != cameras[0].height)
        t->uniform_views = false;
    int64_t total = 0;
    for (int v = 0; v < n_views; ++v) {
      t->image_offset.push_back(total);
      total += static_cast<int64_t>(cameras[v].width) * cameras[v].height;
    }
    t->images.reserve(static_cast<size_t>(total) * 3 + 1);
    for (int v = 0; v < n_views; ++v) {
      const size_t vals = static_cast<size_t>(cameras[v].width) * cameras[v].height * 3;
      if (vals > 0)
        PXS_CUDA(cudaMemcpyAsync(t->images.get() + t->image_offset[v] * 3, images[v],
                                 vals * sizeof(float), cudaMemcpyHostToDevice, t->stream));
    }
    t->scalars.reserve(1);
    // TrainingRng(seed) and the initial shuffle (SplatTrainer.cpp:17, :163-177)
    t->engine.seed(config->seed == 0u ? 1u : config->seed);
    t->densify_rng = config->seed == 0u ? 1u : config->seed;
    t->extent = camera_extent(t->cameras);
    t->order.resize(static_cast<size_t>(n_views));
    std::iota(t->order.begin(), t->order.end(), 0);
    std::shuffle(t->order.begin(), t->order.end(), t->engine);
    PXS_CUDA(cudaStreamSynchronize(t->stream));
  });
  if (status != PXS_OK) {
    delete t;
    return status;
  }
  *out = t;
  return PXS_OK;
}

void pxs_trainer_destroy(pxs_trainer* t) {
  if (t == nullptr) return;
  cudaSetDevice(t->device);
  if (t->stream) cudaStreamSynchronize(t->stream);
  delete t;
}

const char* pxs_trainer_last_error(const pxs_trainer* t) {
  return t == nullptr ? "trainer is null" : t->error.c_str();
}

int pxs_trainer_step(pxs_trainer* t, int32_t* stepped) {
  return guarded(t, [&] {
    const bool s = t->step();
    if (stepped) *stepped = s ? 1 : 0;
  });
}

int pxs_trainer_train(pxs_trainer* t, pxs_progress_fn callback, void* user, int32_t* completed) {
  return guarded(t, [&] {
    if (completed) *completed = 1;
    while (t->step()) {
      if (callback == nullptr) continue;
      pxs_progress p;
      p.iteration = t->iteration;
      p.total_iterations = t->cfg.iterations;
      p.gaussian_count = t->N;
      p.loss = t->last_loss;
      p.smoothed_loss = t->smoothed_loss;
      if (!callback(&p, user)) {
        if (completed) *completed = 0;
        return;
      }
    }
  });
}

int pxs_trainer_step_batch(pxs_trainer* t, int32_t n_views, const int32_t* view_ids,
                           int32_t use_graph, float* loss) {
  return guarded(t, [&] {
    if (n_views <= 0) throw Error(PXS_ERR_INVALID, "n_views must be positive");
    const float l = t->step_batch(n_views, view_ids, use_graph != 0);
    if (loss) *loss = l;
  });
}

int pxs_trainer_accumulate(pxs_trainer* t, int32_t n_views, const int32_t* view_ids,
                           int32_t use_graph, float* loss) {
  return guarded(t, [&] {
    if (n_views <= 0) throw Error(PXS_ERR_INVALID, "n_views must be positive");
    const float l = t->accumulate(n_views, view_ids, use_graph != 0);
    if (loss) *loss = l;
  });
}

int pxs_trainer_apply(pxs_trainer* t, float loss) {
  return guarded(t, [&] { t->apply(loss); });
}

int pxs_trainer_gradients(pxs_trainer* t, float** params, float** screen_gradient,
                          float** visible_count, int32_t* count, int32_t* values) {
  return guarded(t, [&] {
    if (params) *params = t->d_grads();
    if (screen_gradient) *screen_gradient = t->d_screen();
    if (visible_count) *visible_count = t->d_visible_f();
    if (count) *count = t->N;
    if (values) *values = t->P;
  });
}

int pxs_trainer_reduction_block(pxs_trainer* t, float** block, int64_t* values) {
  return guarded(t, [&] {
    if (block) *block = t->grad_block.get();
    if (values) *values = static_cast<int64_t>(t->block_values());
  });
}

int pxs_trainer_autotune(pxs_trainer* t, int32_t n_views, const int32_t* view_ids,
                         int32_t* forward_px, int32_t* backward_px) {
  return guarded(t, [&] {
    if (n_views <= 0) throw Error(PXS_ERR_INVALID, "n_views must be positive");
    int f = 0, b = 0;
    t->autotune(n_views, view_ids, &f, &b);
    if (forward_px) *forward_px = f;
    if (backward_px) *backward_px = b;
  });
}

int pxs_trainer_autotune_report(pxs_trainer* t, char* text, size_t capacity) {
  return guarded(t, [&] {
    if (text == nullptr || capacity == 0) throw Error(PXS_ERR_INVALID, "no buffer");
    std::strncpy(text, t->tune_log.c_str(), capacity - 1);
    text[capacity - 1] = '\0';
  });
}

int pxs_trainer_step_views(pxs_trainer* t, int32_t n_views, const int32_t* view_ids,
                           float* loss) {
  return guarded(t, [&] {
    if (n_views <= 0) throw Error(PXS_ERR_INVALID, "n_views must be positive");
    const float l = t->step_views(n_views, view_ids);
    if (loss) *loss = l;
  });
}

int pxs_trainer_render(pxs_trainer* t, const pxs_camera* camera,
                       const pxs_raster_options* options, float* rgb, float* transmittance) {
  return guarded(t, [&] {
    if (camera == nullptr || rgb == nullptr) throw Error(PXS_ERR_INVALID, "null argument");
    const pxs_raster_options opt = options != nullptr ? *options : t->options();
    const pxs::ViewBatch b = pxs::make_batch(camera, 1, opt, t->cloud_sh);
    t->graph.reset();  // the frame's buffers may be resized
    t->graph_acc.reset();
    t->graph_one.reset();
    t->frame.prepare(b, t->N, t->S, t->stream);
    t->frame.project(t->params.get(), t->stream);
    t->frame.bin(true, t->stream);
    t->frame.forward(t->stream);
    const size_t pixels = static_cast<size_t>(b.total_pixels);
    if (pixels > 0) {
      PXS_CUDA(cudaMemcpyAsync(rgb, t->frame.rgb.get(), pixels * 3 * sizeof(float),
                               cudaMemcpyDeviceToHost, t->stream));
      if (transmittance != nullptr)
        PXS_CUDA(cudaMemcpyAsync(transmittance, t->frame.transmittance.get(),
                                 pixels * sizeof(float), cudaMemcpyDeviceToHost, t->stream));
    }
    PXS_CUDA(cudaStreamSynchronize(t->stream));
  });
}

int pxs_measure_fp32_peak(int32_t device, float* tflops) {
  if (tflops == nullptr) return PXS_ERR_INVALID;
  try {
    PXS_CUDA(cudaSetDevice(device));
    *tflops = pxs::measure_fp32_peak_tflops(nullptr);
    return PXS_OK;
  } catch (const Error& e) {
    return e.code;
  }
}

int pxs_trainer_stream(pxs_trainer* t, void** stream) {
  return guarded(t, [&] {
    if (stream == nullptr) throw Error(PXS_ERR_INVALID, "stream is null");
    *stream = static_cast<void*>(t->stream);
  });
}

int pxs_trainer_set_timing(pxs_trainer* t, int32_t enable) {
  return guarded(t, [&] { t->set_timing(enable != 0); });
}

int pxs_trainer_stage_times(pxs_trainer* t, float* ms, int32_t capacity, int32_t* n_stages,
                            int32_t* n_steps) {
  return guarded(t, [&] {
    if (n_stages) *n_stages = pxs_trainer::kStages;
    if (n_steps) *n_steps = t->timed_steps;
    if (ms != nullptr)
      for (int i = 0; i < std::min<int>(capacity, pxs_trainer::kStages); ++i)
        ms[i] = static_cast<float>(t->stage_ms[i]);
  });
}

int pxs_trainer_step_info(pxs_trainer* t, int64_t* pairs, int64_t* kernel_launches) {
  return guarded(t, [&] {
    if (pairs) *pairs = t->last_pairs;
    if (kernel_launches) *kernel_launches = t->last_launches;
  });
}

int pxs_trainer_pair_stats(pxs_trainer* t, int64_t* evaluated, int64_t* contributing) {
  return guarded(t, [&] {
    if (t->frame.sorted_pair_vals == nullptr) throw Error(PXS_ERR_INVALID, "no batch yet");
    unsigned long long* c = t->pair_counts.reserve(2);
    PXS_CUDA(cudaMemsetAsync(c, 0, 2 * sizeof(unsigned long long), t->stream));
    t->frame.forward(t->stream, c);
    unsigned long long host[2] = {0, 0};
    PXS_CUDA(cudaMemcpyAsync(host, c, sizeof(host), cudaMemcpyDeviceToHost, t->stream));
    PXS_CUDA(cudaStreamSynchronize(t->stream));
    if (evaluated) *evaluated = static_cast<int64_t>(host[0]);
    if (contributing) *contributing = static_cast<int64_t>(host[1]);
  });
}

int pxs_trainer_set_images(pxs_trainer* t, int32_t n, const int32_t* view_ids,
                           const float* const* images) {
  return guarded(t, [&] {
    t->consume_staged();
    for (int i = 0; i < n; ++i) {
      const int id = view_ids[i];
      if (id < 0 || id >= static_cast<int>(t->cameras.size()))
        throw Error(PXS_ERR_INVALID, "view id out of range");
      const size_t vals = static_cast<size_t>(t->cameras[id].width) * t->cameras[id].height * 3;
      if (vals > 0)
        PXS_CUDA(cudaMemcpyAsync(t->images.get() + t->image_offset[id] * 3, images[i],
                                 vals * sizeof(float), cudaMemcpyHostToDevice, t->stream));
    }
  });
}

int pxs_trainer_state(pxs_trainer* t, int32_t* iteration, int32_t* count, float* last_loss,
                      float* smoothed_loss, float* extent, int32_t* sh_degree_in_use) {
  return guarded(t, [&] {
    if (iteration) *iteration = t->iteration;
    if (count) *count = t->N;
    if (last_loss) *last_loss = t->last_loss;
    if (smoothed_loss) *smoothed_loss = t->smoothed_loss;
    if (extent) *extent = t->extent;
    if (sh_degree_in_use) *sh_degree_in_use = t->sh_degree_in_use();
  });
}

int pxs_trainer_download(pxs_trainer* t, float* params, int32_t capacity, int32_t* count) {
  return guarded(t, [&] {
    if (count) *count = t->N;
    if (t->N > capacity) throw Error(PXS_ERR_CAPACITY, "capacity below the gaussian count");
    const size_t values = static_cast<size_t>(t->P) * static_cast<size_t>(t->N);
    if (values > 0) {
      if (params == nullptr) throw Error(PXS_ERR_INVALID, "params is null");
      PXS_CUDA(cudaMemcpyAsync(params, t->params.get(), values * sizeof(float),
                               cudaMemcpyDeviceToHost, t->stream));
    }
    PXS_CUDA(cudaStreamSynchronize(t->stream));
  });
}

int pxs_trainer_finish(pxs_trainer* t, float* params, int32_t capacity, int32_t* count) {
  return guarded(t, [&] {
    if (t->n_scenes > 1)
      throw Error(PXS_ERR_INVALID,
                  "finish() prunes and sorts one cloud; download the scenes instead");
    ++t->generation;
    DeviceArray<float> out;
    out.reserve(static_cast<size_t>(t->P) * static_cast<size_t>(std::max(t->N, 1)));
    const int64_t n = pxs::finish_device(t->dwork, t->params.get(), t->N, t->S,
                                         t->cfg.prune_opacity, out.get(), t->stream);
    if (count) *count = static_cast<int32_t>(n);
    if (n > capacity) throw Error(PXS_ERR_CAPACITY, "capacity below the finished count");
    const size_t values = static_cast<size_t>(t->P) * static_cast<size_t>(n);
    if (values > 0) {
      if (params == nullptr) throw Error(PXS_ERR_INVALID, "params is null");
      PXS_CUDA(cudaMemcpyAsync(params, out.get(), values * sizeof(float), cudaMemcpyDeviceToHost,
                               t->stream));
    }
    PXS_CUDA(cudaStreamSynchronize(t->stream));
    // the trainer is spent (SplatTrainer.h:155-156): keep the finished cloud
    t->params.swap(out);
    t->N = static_cast<int>(n);
    t->cloud_sh = t->cfg.sh_degree;
    t->iteration = t->cfg.iterations;
  });
}

int pxs_trainer_stage_images(pxs_trainer* t, int32_t n, const int32_t* view_ids,
                             const uint8_t* const* frames, const int32_t* widths,
                             const int32_t* heights) {
  return guarded(t, [&] {
    if (n < 0 || (n > 0 && (view_ids == nullptr || frames == nullptr || widths == nullptr ||
                            heights == nullptr)))
      throw Error(PXS_ERR_INVALID, "null argument");
    t->stage_frames(n, view_ids, frames, widths, heights);
  });
}

int pxs_trainer_ingest_images(pxs_trainer* t, int32_t n, const int32_t* view_ids,
                              const uint8_t* const* frames, const int32_t* widths,
                              const int32_t* heights) {
  return guarded(t, [&] {
    if (n < 0 || (n > 0 && (view_ids == nullptr || frames == nullptr || widths == nullptr ||
                            heights == nullptr)))
      throw Error(PXS_ERR_INVALID, "null argument");
    t->consume_staged();
    for (int i = 0; i < n; ++i) {
      const int id = view_ids[i];
      if (id < 0 || id >= static_cast<int>(t->cameras.size()))
        throw Error(PXS_ERR_INVALID, "view id out of range");
      const pxs_camera& cam = t->cameras[static_cast<size_t>(id)];
      int w = 0, h = 0;
      pxs::downscaled_size(widths[i], heights[i], cam.width, &w, &h);
      if (w != cam.width || h != cam.height)
        throw Error(PXS_ERR_INVALID, "the downscaled frame does not match the view's size");
      const size_t in_bytes = static_cast<size_t>(widths[i]) * heights[i] * 3;
      if (in_bytes == 0) continue;
      if (frames[i] == nullptr) throw Error(PXS_ERR_INVALID, "frame is null");
      // the staging buffer is reused by the next frame: the stream orders the
      // next copy after this frame's downscale; it is grown only when idle
      if (in_bytes > t->ingest_in.capacity()) PXS_CUDA(cudaStreamSynchronize(t->stream));
      uint8_t* d_in = t->ingest_in.reserve(in_bytes);
      PXS_CUDA(cudaMemcpyAsync(d_in, frames[i], in_bytes, cudaMemcpyHostToDevice, t->stream));
      pxs::launch_downscale(d_in, widths[i], heights[i], w, h, nullptr,
                            t->images.get() + t->image_offset[static_cast<size_t>(id)] * 3,
                            t->stream);
      PXS_CUDA(cudaGetLastError());
    }
    // the frames may be released once the call returns
    PXS_CUDA(cudaStreamSynchronize(t->stream));
  });
}

int pxs_trainer_export(pxs_trainer* t, int32_t format, int32_t fractional_bits, uint8_t* out,
                       size_t capacity, size_t* size) {
  std::vector<uint8_t> bytes;
  const int status = guarded(t, [&] {
    if (t->n_scenes > 1)
      throw Error(PXS_ERR_INVALID, "a trainer over several scenes exports no single file");
    DeviceArray<uint8_t> body;
    DeviceArray<int32_t> fields;
    bytes = pxs::export_cloud_bytes(t->params.get(), t->N, t->S, t->cloud_sh, format,
                                    fractional_bits, body, fields, t->stream);
  });
  if (status != PXS_OK) return status;
  if (size != nullptr) *size = bytes.size();
  if (out == nullptr || capacity < bytes.size()) return PXS_ERR_CAPACITY;
  std::memcpy(out, bytes.data(), bytes.size());
  return PXS_OK;
}

int pxs_trainer_create_scenes(const pxs_train_config* config, const pxs_cloud* clouds,
                              int32_t n_scenes, const int32_t* views_per_scene,
                              const pxs_camera* cameras, const float* const* images,
                              int32_t device, pxs_trainer** out) {
  if (out == nullptr || config == nullptr || clouds == nullptr || views_per_scene == nullptr ||
      n_scenes <= 0)
    return PXS_ERR_INVALID;
  *out = nullptr;
  // densification resizes one cloud; several scenes train at a fixed size
  const int last = std::min(config->densify_until_iteration, config->iterations);
  if (n_scenes > 1 && config->densify_from_iteration <= last) return PXS_ERR_INVALID;
  const int S = clouds[0].rest_per_channel;
  int64_t total = 0;
  int n_views = 0;
  for (int s = 0; s < n_scenes; ++s) {
    if (clouds[s].rest_per_channel != S || clouds[s].sh_degree != clouds[0].sh_degree ||
        clouds[s].count < 0 || views_per_scene[s] < 0 ||
        (clouds[s].count > 0 && clouds[s].params == nullptr))
      return PXS_ERR_INVALID;
    total += clouds[s].count;
    n_views += views_per_scene[s];
  }
  if (total > INT32_MAX / 2) return PXS_ERR_INVALID;
  // one component-major cloud holding the scenes one after another
  const size_t P = static_cast<size_t>(PXS_PARAM_COUNT(S));
  std::vector<float> joined;
  try {
    joined.resize(P * static_cast<size_t>(total));
  } catch (const std::bad_alloc&) {
    return PXS_ERR_NO_MEMORY;
  }
  std::vector<int32_t> offsets;
  int64_t at = 0;
  for (int s = 0; s < n_scenes; ++s) {
    offsets.push_back(static_cast<int32_t>(at));
    const size_t n = static_cast<size_t>(clouds[s].count);
    for (size_t c = 0; c < P; ++c)
      std::copy(clouds[s].params + c * n, clouds[s].params + (c + 1) * n,
                joined.begin() + static_cast<ptrdiff_t>(c * static_cast<size_t>(total) + at));
    at += clouds[s].count;
  }
  pxs_cloud all{joined.data(), static_cast<int32_t>(total), S, clouds[0].sh_degree};
  pxs_trainer* t = nullptr;
  const int status = pxs_trainer_create(config, &all, cameras, images, n_views, device, &t);
  if (status != PXS_OK) return status;
  const int configured = guarded(t, [&] {
    t->n_scenes = n_scenes;
    t->scene_offset = offsets;
    t->scene_count.clear();
    t->view_scene.clear();
    t->scene_extent.clear();
    std::vector<float> scale(static_cast<size_t>(std::max<int64_t>(total, 1)), 1.f);
    int view = 0;
    for (int s = 0; s < n_scenes; ++s) {
      t->scene_count.push_back(clouds[s].count);
      std::vector<pxs_camera> cams(cameras + view, cameras + view + views_per_scene[s]);
      const float e = camera_extent(cams);  // each scene's own extent
      t->scene_extent.push_back(e);
      for (int i = 0; i < clouds[s].count; ++i) scale[static_cast<size_t>(offsets[s] + i)] = e;
      for (int k = 0; k < views_per_scene[s]; ++k) t->view_scene.push_back(s);
      view += views_per_scene[s];
    }
    float* d = t->position_scale.reserve(scale.size());
    PXS_CUDA(cudaMemcpyAsync(d, scale.data(), scale.size() * sizeof(float),
                             cudaMemcpyHostToDevice, t->stream));
    PXS_CUDA(cudaStreamSynchronize(t->stream));
  });
  if (configured != PXS_OK) {
    pxs_trainer_destroy(t);
    return configured;
  }
  *out = t;
  return PXS_OK;
}

int pxs_train_splats(pxs_cloud* cloud, const pxs_camera* cameras, const float* const* images,
                     int32_t n_views, const pxs_train_config* config, pxs_progress_fn callback,
                     void* user, char* error, size_t error_len) {
  auto fail = [&](int code, const std::string& why) {
    if (error != nullptr && error_len > 0) {
      std::strncpy(error, why.c_str(), error_len - 1);
      error[error_len - 1] = '\0';
    }
    return code;
  };
  if (cloud == nullptr || config == nullptr) return fail(PXS_ERR_INVALID, "null argument");
  char reason[256];
  if (pxs_train_config_validate(config, reason, sizeof(reason)) != PXS_OK)
    return fail(PXS_ERR_INVALID, reason);
  int32_t available = 0;
  char why[256];
  pxs_gpu_availability(&available, nullptr, 0, why, sizeof(why));
  if (!available) return fail(PXS_ERR_UNAVAILABLE, why);
  pxs_trainer* t = nullptr;
  int status = pxs_trainer_create(config, cloud, cameras, images, n_views, 0, &t);
  if (status != PXS_OK) return fail(status, "could not set up the GPU trainer");
  int32_t completed = 1;
  status = pxs_trainer_train(t, callback, user, &completed);
  if (status == PXS_OK) {
    // a cancelled run still writes back (VulkanSplatTrainer.cpp:856-867, :904-905)
    int32_t n = 0;
    status = pxs_trainer_finish(t, cloud->params, config->max_gaussians, &n);
    if (status == PXS_OK) {
      cloud->count = n;
      cloud->sh_degree = config->sh_degree;
    }
  }
  const std::string message = status == PXS_OK ? "" : t->error;
  pxs_trainer_destroy(t);
  if (status != PXS_OK) return fail(status, message);
  if (error != nullptr && error_len > 0) error[0] = '\0';
  return PXS_OK;
}

}  // extern "C"
