// kernels.h -- host-side launchers of the sm_100a kernels.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace pxs {

// Per-step optimiser scalars, read by the Adam kernel from device memory so a
// captured graph picks up each step's values.
struct StepScalars {
  float lr[6];  // position, log_scale, rotation, opacity, dc, sh_rest
  float beta1, beta2, epsilon;
  float correction1, correction2;
  float pad;
};

struct LossParams {
  float kernel[11];   // ssimKernel() (SplatRaster.cpp:587-600), computed on the host
  float ssim_weight;
  int mode;           // 0 photometric loss gradient, 1 SSIM gradient
};

struct ScanScratch {
  static constexpr int kLevels = 6;
  char* level[kLevels] = {};
};

// project.cu
void launch_project(const float* params, int N, int S, int64_t slot_stride,
                    const ViewDesc* views, int n_views, const ProjectedSoA& out,
                    cudaStream_t stream);
void configure_param_grads_kernel();  // once per device, outside graph capture
void launch_param_grads(const float* params, int N, int S, int64_t slot_stride,
                        const ViewDesc* views, int n_views, const uint32_t* depth_key,
                        const float4* conic_op, const float4* color, const ScreenGrad* screen,
                        float* grads, float* screen_gradient, int32_t* visible_count,
                        cudaStream_t stream);

// sort.cu
size_t scan_scratch_bytes(int64_t n, int level = 0);
void scan_scratch_assign(ScanScratch& s, char* base, int64_t n);
void exclusive_scan_i32_to_i64(const int32_t* in, int64_t* out, int64_t n, int64_t* total,
                               ScanScratch& scratch, cudaStream_t stream);
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, ScanScratch& scratch,
                        cudaStream_t stream);
size_t radix_hist_entries(int64_t n, int64_t segment_len, int max_bits);
// Sorts (keys, vals) by the low `total_bits` bits of the keys, stably, each
// `segment_len` run independently (segment_len a multiple of kSortTile, or 0
// for one segment). keys/vals and the *_alt buffers are swapped so that on
// return keys/vals hold the result. Returns the number of passes.
int radix_sort_pairs(uint32_t*& keys, uint32_t*& vals, uint32_t*& keys_alt,
                     uint32_t*& vals_alt, int64_t n, int64_t segment_len, int total_bits,
                     uint32_t* hist, uint32_t* hist_scanned, ScanScratch& scratch,
                     cudaStream_t stream, const int64_t* n_device = nullptr);
void launch_iota(uint32_t* out, int64_t n, cudaStream_t stream);

// bin.cu
void configure_bin_kernels();  // once per device, outside graph capture
// Tile-row records grouped by row, depth order within a row (bin.cu): per
// (view, chunk of depth-sorted slots) the splats covering each tile row of the
// view, counts[(row_offset + y) * cpv + c]; after their exclusive scan into
// offsets, each chunk writes its records (slot ids) at its bases.
int slot_chunks_per_view(int64_t slot_stride);
void launch_slot_row_counts(const uint32_t* sorted_slots, const uint32_t* sorted_keys,
                            const uint2* rect, const ViewDesc* views, int n_views,
                            int64_t slot_stride, int max_tiles_y, int32_t* counts,
                            cudaStream_t stream);
void launch_slot_row_expand(const uint32_t* sorted_slots, const uint32_t* sorted_keys,
                            const uint2* rect, const ViewDesc* views, int n_views,
                            int64_t slot_stride, int max_tiles_y, const int64_t* offsets,
                            int64_t capacity, uint32_t* rec_slots, uint32_t* rec_xr,
                            cudaStream_t stream);
// Per-row record ranges from the chunk offsets, clamped to the capacity
// (records past it raise the overflow flag).
void launch_row_ranges_from_chunks(const int64_t* offsets, int total_rows, int cpv,
                                   const int64_t* total, int64_t capacity, int2* row_ranges,
                                   int32_t* overflow, cudaStream_t stream);
// Upper bound on the number of row chunks for `records` records.
int64_t max_row_chunks(int64_t records, int total_rows);
// Chunk table, per-chunk column counts, per-chunk bases and tile lengths.
void launch_tile_lists(const int2* row_ranges, const uint32_t* rec_slots, const uint32_t* rec_xr,
                       const ViewDesc* views, int n_views, int total_rows, int max_tiles_x,
                       int64_t max_chunks, int4* chunks, int32_t* n_chunks,
                       int32_t* chunk_counts, int32_t* chunk_base, int32_t* tile_counts,
                       cudaStream_t stream);
void launch_ranges_from_offsets(const int32_t* counts, const int64_t* offsets, int64_t n_tiles,
                                int64_t capacity, int2* ranges, int32_t* overflow,
                                cudaStream_t stream);
void launch_chunk_expand(const int4* chunks, const int32_t* n_chunks, const uint32_t* rec_slots,
                         const uint32_t* rec_xr, const ViewDesc* views, int n_views, int max_tiles_x,
                         int64_t max_chunks, const int32_t* chunk_base,
                         const int64_t* tile_offsets, int64_t capacity, uint32_t* tile_slots,
                         cudaStream_t stream);

// raster.cu
// Launch parameters of the compositing kernels, read at launch; set before a
// graph is captured:
//   pixels per thread (1, 2 or 4; TileGeom in raster_common.cuh);
//   for the two-pixel forms, the tile-list entries staged per batch (64, 128
//   or 256) and the CTA-to-tile schedule (TileSchedule in raster_common.cuh:
//   0 tile order, 1 heaviest tiles first, 2 persistent, heaviest first).
struct RasterConfig {
  int forward_px = 2;
  int backward_px = 2;
  int forward_batch = 128;
  int backward_batch = 256;
  int forward_schedule = 0;
  int backward_schedule = 0;
  int generation = 0;  // bumped on every change; captured graphs compare it
};
RasterConfig& raster_config();

// The heaviest-first tile order of the schedules above: the tiles sorted by
// decreasing floor(log2(list length)) (a counting sort over 32 classes; the
// order inside a class is arbitrary and does not change any result). `work`
// holds 64 ints.
void launch_tile_order(const int2* ranges, int total_tiles, int* order, int* work,
                       cudaStream_t stream);

// The forward pass; with two pixels per thread and `block_bits` given it also
// writes, per tile-list entry, a byte whose bit b is set when some pixel of
// the tile's 8x8 block b (b = 2 * row block + column block) took the entry.
// Returns whether it wrote them.
bool launch_forward(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                    const float4* conic_op, const float4* color, const ViewDesc* views,
                    int n_views, int total_tiles, float* rgb, float* T, int32_t* last,
                    cudaStream_t stream, unsigned long long* counts = nullptr,
                    uint8_t* block_bits = nullptr, const int* tile_order = nullptr,
                    int* ticket = nullptr);
// The adjoint. `block_bits`, when the forward wrote them, replace the
// geometric warp masks in the two-pixel form: a warp walks only the entries
// one of its pixels took.
void launch_backward(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                     const float4* conic_op, const float4* color, const ViewDesc* views,
                     int n_views, int total_tiles, const float* T_final, const int32_t* last,
                     const float* dL_drgb, ScreenGrad* screen, cudaStream_t stream,
                     const uint8_t* block_bits = nullptr, const int* tile_order = nullptr,
                     int* ticket = nullptr);

// loss.cu
size_t loss_smem_bytes();
void configure_loss_kernel();  // once per device, outside graph capture
// Output tiles of one view in the loss kernel.
int64_t loss_tiles(int width, int height);
// `flat_tiles` >= 0: a one-dimensional grid of that many CTAs over every
// view's own tiles (the sum of loss_tiles over the views); otherwise a grid
// sized for the largest view.
void launch_loss(const float* rendered, const float* target, const ViewDesc* views, int n_views,
                 int max_width, int max_height, const LossParams& lp, float* grad_out,
                 double* sums, float* per_view, float* total, cudaStream_t stream,
                 int64_t flat_tiles = -1);

// export.cu: the reference's file formats packed on the device
void launch_pack_ply(const float* params, int n, const int* field_src, int fields, float* out,
                     cudaStream_t stream);
void launch_pack_splat(const float* params, int n, uint8_t* out, cudaStream_t stream);
void launch_pack_spz(const float* params, int n, int fractional_bits, int rest_stored,
                     int rest_degree, uint8_t* out, cudaStream_t stream);

// export.cu: initializeFromPointCloud's device parts
void launch_seed_nearest(const float* points, int n, int stride, int samples, double* nearest,
                         cudaStream_t stream);
void launch_seed_points(const float* points, const uint8_t* colors, int n, int S,
                        float log_sigma, float logit, float* params, cudaStream_t stream);

// ingest.cu: downscaleToWidth's box filter (and the /255 to float) on the device
void launch_downscale(const uint8_t* src, int width, int height, int out_width, int out_height,
                      uint8_t* out_bytes, float* out_linear, cudaStream_t stream);
// Frames already at their view's size, bytes to linear floats (byte / 255,
// as launch_downscale writes for them), up to kMaxLinearFrames per launch.
// Each frame must pass linear_frame_ok: a whole number of 16-byte groups,
// both addresses 16-byte aligned.
constexpr int kMaxLinearFrames = 16;
bool linear_frame_ok(const uint8_t* src, const float* out, int64_t bytes);
void launch_bytes_to_linear_frames(const uint8_t* const* src, float* const* out,
                                   const int64_t* bytes, int n, cudaStream_t stream);

// peak.cu
float measure_fp32_peak_tflops(cudaStream_t stream);

// adam.cu
// `position_scale` (N floats, optional) multiplies the position learning rate
// per gaussian: each scene's extent, when one cloud holds several scenes.
void launch_pack_reduction(const int32_t* visible, float* visible_f, int N,
                           const float* loss_mean, int n_views, float* tail,
                           cudaStream_t stream);
void launch_unpack_visible(const float* visible_f, int32_t* visible, int N, cudaStream_t stream);
void launch_adam(float* params, float* grads, float* m, float* v, int N, int S,
                 const StepScalars* scalars, int zero_grads, float* screen_gradient,
                 int32_t* visible_count, float* acc_gradient, int32_t* acc_views,
                 cudaStream_t stream, const float* position_scale = nullptr);
// Same step, skipped entirely when *skip is nonzero (a batch whose pairs overflowed).
void launch_adam_checked(float* params, float* grads, float* m, float* v, int N, int S,
                         const StepScalars* scalars, float* screen_gradient,
                         int32_t* visible_count, float* acc_gradient, int32_t* acc_views,
                         const int32_t* skip, cudaStream_t stream,
                         const float* position_scale = nullptr);
void launch_reset_opacity(float* params, float* m, float* v, int N, float ceiling,
                          cudaStream_t stream);

}  // namespace pxs
