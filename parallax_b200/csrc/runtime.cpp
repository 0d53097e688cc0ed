// runtime.cpp -- the per-batch rasterisation frame: buffers and stage launches.
#include "runtime.h"

#include <algorithm>
#include <cmath>

namespace pxs {

int g_fail_allocation_after = 0;
int64_t g_device_allocations = 0;
int64_t g_kernel_launches = 0;

void check_cuda(cudaError_t err, const char* what) {
  if (err != cudaSuccess) {
    cudaGetLastError();
    throw Error(PXS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
  }
}

int bits_for(int64_t count) {
  int bits = 1;
  while (bits < 40 && (int64_t(1) << bits) < count) ++bits;
  return bits;
}

// ssimKernel (SplatRaster.cpp:587-600), with the same libm expf as the reference.
void ssim_kernel_weights(float out[11]) {
  float total = 0.f;
  for (int i = -5; i <= 5; ++i) {
    const float v = std::exp(-0.5f * static_cast<float>(i * i) / (1.5f * 1.5f));
    out[i + 5] = v;
    total += v;
  }
  for (int i = 0; i < 11; ++i) out[i] /= total;
}

void downscaled_size(int width, int height, int target_width, int* out_width, int* out_height) {
  if (width <= 0 || height <= 0 || target_width <= 0 || width <= target_width) {
    *out_width = width;
    *out_height = height;
    return;
  }
  *out_width = target_width;
  *out_height = std::max(1, static_cast<int>(std::lround(static_cast<double>(height) *
                                                          target_width / width)));
}

ViewBatch make_batch(const pxs_camera* cameras, int n_views, const pxs_raster_options& options,
                     int cloud_sh_degree) {
  ViewBatch b;
  b.views.resize(static_cast<size_t>(n_views));
  int tile_offset = 0, row_offset = 0;
  int64_t loss_tile_offset = 0;
  int64_t pixel_offset = 0;
  for (int v = 0; v < n_views; ++v) {
    ViewDesc& d = b.views[static_cast<size_t>(v)];
    std::memset(&d, 0, sizeof(d));
    d.cam = cameras[v];
    if (d.cam.width < 0 || d.cam.height < 0) throw Error(PXS_ERR_INVALID, "negative image size");
    for (int c = 0; c < 3; ++c) d.background[c] = options.background[c];
    d.sh_degree = std::min(options.sh_degree, cloud_sh_degree);
    d.tiles_x = (d.cam.width + kTile - 1) / kTile;
    d.tiles_y = (d.cam.height + kTile - 1) / kTile;
    if (d.tiles_x > kMaxTilesX || d.tiles_y > kMaxTilesY)
      throw Error(PXS_ERR_INVALID, "image too large (at most 2048 tiles across and down)");
    d.tile_offset = tile_offset;
    d.row_offset = row_offset;
    d.loss_tile_offset = static_cast<int32_t>(loss_tile_offset);
    loss_tile_offset += loss_tiles(d.cam.width, d.cam.height);
    d.pixel_offset = pixel_offset;
    d.target_offset = pixel_offset;
    d.min_alpha = options.min_alpha;
    d.transmittance_cutoff = options.transmittance_cutoff;
    d.screen_dilation = options.screen_dilation;
    tile_offset += d.tiles_x * d.tiles_y;
    row_offset += d.tiles_y;
    b.max_tiles_x = std::max(b.max_tiles_x, d.tiles_x);
    b.max_tiles_y = std::max(b.max_tiles_y, d.tiles_y);
    pixel_offset += static_cast<int64_t>(d.cam.width) * d.cam.height;
    b.max_width = std::max(b.max_width, d.cam.width);
    b.max_height = std::max(b.max_height, d.cam.height);
  }
  b.total_pixels = pixel_offset;
  b.total_tiles = tile_offset;
  b.total_rows = row_offset;
  return b;
}

void Frame::ensure_scan_scratch(int64_t n) {
  if (n <= scan_capacity_) return;
  const size_t bytes = scan_scratch_bytes(n) + 64;
  char* base = scan_scratch.reserve(bytes);
  scan_ = ScanScratch();
  scan_scratch_assign(scan_, base, n);
  scan_capacity_ = n;
}

void Frame::prepare(const ViewBatch& b, int n, int s, cudaStream_t stream) {
  if (!configured_) {
    configure_loss_kernel();
    configure_bin_kernels();
    configure_param_grads_kernel();
    PXS_CUDA(cudaGetLastError());
    configured_ = true;
  }
  batch = b;
  N = n;
  S = s;
  V = static_cast<int>(b.views.size());
  int widest = 1;  // the largest gaussian range of a view
  for (ViewDesc& d : batch.views) {
    if (!batch.own_ranges) {
      d.gauss_offset = 0;
      d.gauss_count = N;
    } else if (d.gauss_offset < 0 || d.gauss_count < 0 ||
               static_cast<int64_t>(d.gauss_offset) + d.gauss_count > N) {
      throw Error(PXS_ERR_INVALID, "a view's gaussian range lies outside the cloud");
    }
    widest = std::max(widest, d.gauss_count);
  }
  slot_stride = round_up(widest, kSortTile);
  const size_t slots = static_cast<size_t>(V) * static_cast<size_t>(slot_stride);
  d_views.reserve(static_cast<size_t>(std::max(V, 1)));
  if (V > 0)
    PXS_CUDA(cudaMemcpyAsync(d_views.get(), batch.views.data(), sizeof(ViewDesc) * V,
                             cudaMemcpyHostToDevice, stream));
  xy.reserve(slots);
  conic_op.reserve(slots);
  color.reserve(slots);
  depth_key.reserve(slots);
  rect.reserve(slots);
  tile_count.reserve(slots);
  sort_keys.reserve(slots);
  sort_vals.reserve(slots);
  sort_keys_alt.reserve(slots);
  sort_vals_alt.reserve(slots);
  const size_t row_chunks = static_cast<size_t>(std::max(batch.total_rows, 1)) *
                            static_cast<size_t>(std::max(slot_chunks_per_view(slot_stride), 1));
  row_chunk_counts.reserve(row_chunks);
  row_chunk_offsets.reserve(row_chunks);
  d_total_pairs.reserve(1);
  screen.reserve(slots);
  overflow.reserve(1);
  const size_t pixels = static_cast<size_t>(std::max<int64_t>(batch.total_pixels, 1));
  rgb.reserve(pixels * 3);
  dL.reserve(pixels * 3);
  transmittance.reserve(pixels);
  last.reserve(pixels);
  ranges.reserve(static_cast<size_t>(std::max(batch.total_tiles, 1)));
  tile_order.reserve(static_cast<size_t>(std::max(batch.total_tiles, 1)));
  order_work.reserve(64);
  tickets.reserve(2);
  order_ready = false;
  tile_counts.reserve(static_cast<size_t>(std::max(batch.total_tiles, 1)));
  tile_offsets.reserve(static_cast<size_t>(std::max(batch.total_tiles, 1)));
  row_ranges.reserve(static_cast<size_t>(std::max(batch.total_rows, 1)));
  n_chunks.reserve(1);
  d_total_records.reserve(1);
  loss_sums.reserve(static_cast<size_t>(2 * std::max(V, 1)));
  loss_per_view.reserve(static_cast<size_t>(std::max(V, 1)));
  loss_total.reserve(1);
  // the depth sort's histograms; the tile sort's are sized in reserve_pairs
  const size_t depth_hist = radix_hist_entries(static_cast<int64_t>(slots), slot_stride, 8);
  if (hist.capacity() < depth_hist) {
    hist.reserve(depth_hist);
    hist_scanned.reserve(depth_hist);
  }
  ensure_scan_scratch(std::max<int64_t>(std::max<int64_t>(static_cast<int64_t>(slots),
                                                          static_cast<int64_t>(hist.capacity())),
                                        batch.total_tiles));
  // the chunk table depends on the rows as well as on the record capacity; size
  // it here, before any stream capture of the binning stage
  if (record_capacity > 0) ensure_chunks();
}

void Frame::reserve_pairs(int64_t capacity) {
  if (capacity > INT32_MAX) throw Error(PXS_ERR_CAPACITY, "more than 2^31 tile pairs");
  if (capacity <= pair_capacity && tile_slots.get() != nullptr) return;
  const size_t cap = static_cast<size_t>(std::max<int64_t>(capacity, 1));
  tile_slots.reserve(cap);
  block_bits.reserve(cap);
  pair_capacity = static_cast<int64_t>(cap);
}

void Frame::reserve_records(int64_t capacity) {
  if (capacity > INT32_MAX) throw Error(PXS_ERR_CAPACITY, "more than 2^31 tile-row records");
  if (capacity <= record_capacity && rec_vals.get() != nullptr) return;
  const size_t cap = static_cast<size_t>(std::max<int64_t>(capacity, 1));
  rec_vals.reserve(cap);
  rec_xr.reserve(cap);
  record_capacity = static_cast<int64_t>(cap);
  ensure_chunks();
}

void Frame::ensure_chunks() {
  const int64_t need = max_row_chunks(std::max<int64_t>(record_capacity, 1), batch.total_rows);
  const size_t per = static_cast<size_t>(std::max(batch.max_tiles_x, 1));
  if (need > max_chunks || chunk_counts.capacity() < static_cast<size_t>(need) * per) {
    chunks.reserve(static_cast<size_t>(need));
    chunk_counts.reserve(static_cast<size_t>(need) * per);
    chunk_base.reserve(static_cast<size_t>(need) * per);
    max_chunks = need;
  }
}

void Frame::project(const float* params, cudaStream_t stream, bool want_debug) {
  ProjectedSoA out;
  out.xy = xy.get();
  out.conic_op = conic_op.get();
  out.color = color.get();
  out.depth_key = depth_key.get();
  out.rect = rect.get();
  out.tile_count = tile_count.get();
  out.debug_cov = nullptr;
  if (want_debug) out.debug_cov = debug_cov.reserve(static_cast<size_t>(V) * slot_stride);
  launch_project(params, N, S, slot_stride, d_views.get(), V, out, stream);
  PXS_CUDA(cudaGetLastError());
}

int64_t Frame::bin(bool host_sync, cudaStream_t stream) {
  order_ready = false;  // new tile lists
  const int64_t slots = static_cast<int64_t>(V) * slot_stride;
  if (slots == 0) {
    last_pair_count = 0;
    return 0;
  }
  // 1. every slot near to far within its view (stable: equal depths by index)
  PXS_CUDA(cudaMemcpyAsync(sort_keys.get(), depth_key.get(), sizeof(uint32_t) * slots,
                           cudaMemcpyDeviceToDevice, stream));
  launch_iota(sort_vals.get(), slots, stream);
  uint32_t *k = sort_keys.get(), *v = sort_vals.get();
  uint32_t *ka = sort_keys_alt.get(), *va = sort_vals_alt.get();
  radix_sort_pairs(k, v, ka, va, slots, slot_stride, 32, hist.get(), hist_scanned.get(), scan_,
                   stream);
  sorted_slots = v;  // k holds their keys: kCulledKey for a culled slot
  // 2. one record per covered tile row, grouped by row and near to far within
  //    a row: per (view, slot chunk) row counts, their scan in (row, chunk)
  //    order, then each chunk writes its records at its bases
  const int cpv = slot_chunks_per_view(slot_stride);
  const int64_t n_row_chunks = static_cast<int64_t>(batch.total_rows) * cpv;
  launch_slot_row_counts(v, k, rect.get(), d_views.get(), V, slot_stride,
                         batch.max_tiles_y, row_chunk_counts.get(), stream);
  exclusive_scan_i32_to_i64(row_chunk_counts.get(), row_chunk_offsets.get(), n_row_chunks,
                            d_total_records.get(), scan_, stream);
  PXS_CUDA(cudaGetLastError());
  if (host_sync) {
    PXS_CUDA(cudaMemcpyAsync(&last_record_count, d_total_records.get(), sizeof(int64_t),
                             cudaMemcpyDeviceToHost, stream));
    PXS_CUDA(cudaStreamSynchronize(stream));
    if (last_record_count > record_capacity)
      reserve_records(last_record_count + last_record_count / 8 + 1024);
  } else if (rec_vals.get() == nullptr || tile_slots.get() == nullptr) {
    throw Error(PXS_ERR_INVALID, "pair buffers must be reserved before an unsynchronised bin");
  }
  PXS_CUDA(cudaMemsetAsync(overflow.get(), 0, sizeof(int32_t), stream));
  launch_slot_row_expand(v, k, rect.get(), d_views.get(), V, slot_stride,
                         batch.max_tiles_y, row_chunk_offsets.get(), record_capacity,
                         rec_vals.get(), rec_xr.get(), stream);
  launch_row_ranges_from_chunks(row_chunk_offsets.get(), batch.total_rows, cpv,
                                d_total_records.get(), record_capacity, row_ranges.get(),
                                overflow.get(), stream);
  const uint32_t* rv = rec_vals.get();
  // 4. tile lengths from chunked rows, their offsets, then the lists themselves
  ensure_chunks();
  launch_tile_lists(row_ranges.get(), rv, rec_xr.get(), d_views.get(), V, batch.total_rows,
                    batch.max_tiles_x, max_chunks, chunks.get(), n_chunks.get(),
                    chunk_counts.get(), chunk_base.get(), tile_counts.get(), stream);
  exclusive_scan_i32_to_i64(tile_counts.get(), tile_offsets.get(), batch.total_tiles,
                            d_total_pairs.get(), scan_, stream);
  PXS_CUDA(cudaGetLastError());
  int64_t K = -1;
  if (host_sync) {
    PXS_CUDA(cudaMemcpyAsync(&last_pair_count, d_total_pairs.get(), sizeof(int64_t),
                             cudaMemcpyDeviceToHost, stream));
    PXS_CUDA(cudaStreamSynchronize(stream));
    K = last_pair_count;
    if (K > pair_capacity) reserve_pairs(K + K / 8 + 1024);
  }
  launch_ranges_from_offsets(tile_counts.get(), tile_offsets.get(), batch.total_tiles,
                             pair_capacity, ranges.get(), overflow.get(), stream);
  launch_chunk_expand(chunks.get(), n_chunks.get(), rv, rec_xr.get(), d_views.get(), V,
                      batch.max_tiles_x, max_chunks, chunk_base.get(), tile_offsets.get(),
                      pair_capacity, tile_slots.get(), stream);
  sorted_pair_vals = tile_slots.get();
  PXS_CUDA(cudaGetLastError());
  return K;
}

// The heaviest-first tile order of the current lists, when a schedule wants it.
const int* Frame::ordered_tiles(int schedule, cudaStream_t stream) {
  if (schedule == 0) return nullptr;
  if (!order_ready) {
    launch_tile_order(ranges.get(), batch.total_tiles, tile_order.get(), order_work.get(),
                      stream);
    PXS_CUDA(cudaGetLastError());
    order_ready = true;
  }
  return tile_order.get();
}

void Frame::forward(cudaStream_t stream, unsigned long long* counts) {
  const int* order = counts ? nullptr : ordered_tiles(raster_config().forward_schedule, stream);
  have_block_bits =
      launch_forward(ranges.get(), sorted_pair_vals, xy.get(), conic_op.get(), color.get(),
                     d_views.get(), V, batch.total_tiles, rgb.get(), transmittance.get(),
                     last.get(), stream, counts, block_bits.get(), order, tickets.get());
  PXS_CUDA(cudaGetLastError());
}

void Frame::loss(const float* target, float ssim_weight, int mode, float* grad_out,
                 cudaStream_t stream) {
  LossParams lp;
  ssim_kernel_weights(lp.kernel);
  lp.ssim_weight = ssim_weight;
  lp.mode = mode;
  int64_t tiles = 0;
  for (const ViewDesc& d : batch.views) tiles += loss_tiles(d.cam.width, d.cam.height);
  launch_loss(rgb.get(), target, d_views.get(), V, batch.max_width, batch.max_height, lp,
              grad_out, loss_sums.get(), loss_per_view.get(), loss_total.get(), stream, tiles);
  PXS_CUDA(cudaGetLastError());
}

void Frame::backward(const float* dL_drgb, cudaStream_t stream) {
  const size_t slots = static_cast<size_t>(V) * static_cast<size_t>(slot_stride);
  PXS_CUDA(cudaMemsetAsync(screen.get(), 0, sizeof(ScreenGrad) * slots, stream));
  const int* order = ordered_tiles(raster_config().backward_schedule, stream);
  launch_backward(ranges.get(), sorted_pair_vals, xy.get(), conic_op.get(), color.get(),
                  d_views.get(), V, batch.total_tiles, transmittance.get(), last.get(), dL_drgb,
                  screen.get(), stream, have_block_bits ? block_bits.get() : nullptr, order,
                  tickets.get() + 1);
  PXS_CUDA(cudaGetLastError());
}

void Frame::param_grads(const float* params, float* grads, float* screen_gradient,
                        int32_t* visible_count, cudaStream_t stream) {
  launch_param_grads(params, N, S, slot_stride, d_views.get(), V, depth_key.get(), conic_op.get(),
                     color.get(), screen.get(), grads, screen_gradient, visible_count, stream);
  PXS_CUDA(cudaGetLastError());
}

}  // namespace pxs
