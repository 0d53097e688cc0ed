// runtime.h -- host runtime of the splat training core: device buffers, the
// per-batch rasterisation frame and the stage pipeline.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.h"

namespace pxs {

// A failure carrying a pxs status code; caught at the C boundary.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

void check_cuda(cudaError_t err, const char* what);
#define PXS_CUDA(call) ::pxs::check_cuda((call), #call)

// Test hook: when positive, the n-th following device allocation fails as if
// the device were out of memory (counted down per allocation).
extern int g_fail_allocation_after;
// Device allocations made by DeviceArray so far. A captured graph holds raw
// buffer addresses, so it is stale once this has moved since the capture.
extern int64_t g_device_allocations;

// Grow-only device array; contents are not preserved across growth.
template <typename T>
class DeviceArray {
 public:
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  DeviceArray(DeviceArray&& o) noexcept : ptr_(o.ptr_), cap_(o.cap_) { o.ptr_ = nullptr; o.cap_ = 0; }
  DeviceArray& operator=(DeviceArray&& o) noexcept {
    if (this != &o) {
      release();
      ptr_ = o.ptr_;
      cap_ = o.cap_;
      o.ptr_ = nullptr;
      o.cap_ = 0;
    }
    return *this;
  }
  ~DeviceArray() { release(); }

  T* reserve(size_t n) {
    if (n <= cap_ && ptr_ != nullptr) return ptr_;
    release();
    const size_t count = n > 0 ? n : 1;
    if (g_fail_allocation_after > 0 && --g_fail_allocation_after == 0)
      throw Error(PXS_ERR_NO_MEMORY, "device allocation failed (injected)");
    const cudaError_t err = cudaMalloc(reinterpret_cast<void**>(&ptr_), count * sizeof(T));
    if (err != cudaSuccess) {
      cudaGetLastError();
      ptr_ = nullptr;
      cap_ = 0;
      throw Error(PXS_ERR_NO_MEMORY, std::string("cudaMalloc of ") +
                                         std::to_string(count * sizeof(T)) +
                                         " bytes failed: " + cudaGetErrorString(err));
    }
    cap_ = count;
    ++g_device_allocations;
    return ptr_;
  }
  void release() {
    if (ptr_ != nullptr) cudaFree(ptr_);
    ptr_ = nullptr;
    cap_ = 0;
  }
  T* get() const { return ptr_; }
  size_t capacity() const { return cap_; }
  void swap(DeviceArray& o) noexcept {
    std::swap(ptr_, o.ptr_);
    std::swap(cap_, o.cap_);
  }

 private:
  T* ptr_ = nullptr;
  size_t cap_ = 0;
};

// The host description of one batch of views.
struct ViewBatch {
  std::vector<ViewDesc> views;
  int64_t total_pixels = 0;
  int total_tiles = 0;
  int total_rows = 0;       // tile rows over all views
  int max_tiles_x = 0, max_tiles_y = 0;
  int max_width = 0, max_height = 0;
  // the views carry their own gaussian ranges (several scenes); otherwise
  // Frame::prepare gives every view the whole cloud
  bool own_ranges = false;
};

// The bytes of a cloud's file in `format` (PXS_FORMAT_*), packed on the device
// from component-major device params and copied back once.
std::vector<uint8_t> export_cloud_bytes(const float* d_params, int n, int S, int sh_degree,
                                        int format, int fractional_bits,
                                        DeviceArray<uint8_t>& body, DeviceArray<int32_t>& fields,
                                        cudaStream_t stream);

// downscaleToWidth's output size (ImageIo.cpp:300-304): the image itself when
// it is no wider than the target.
void downscaled_size(int width, int height, int target_width, int* out_width, int* out_height);

ViewBatch make_batch(const pxs_camera* cameras, int n_views, const pxs_raster_options& options,
                     int cloud_sh_degree);
int bits_for(int64_t count);  // bits to represent values in [0, count)
void ssim_kernel_weights(float out[11]);  // ssimKernel() with the host libm

// Buffers and stages of one rasterisation batch: V views of an N-gaussian cloud.
class Frame {
 public:
  // Sizes the per-slot and per-pixel buffers and uploads the views.
  void prepare(const ViewBatch& batch, int N, int S, cudaStream_t stream);
  // Project every (view, gaussian) slot.
  void project(const float* params, cudaStream_t stream, bool debug_cov = false);
  // Depth sort, pair emission, tile sort and ranges. With host_sync the pair
  // count is read back and the pair buffers grown to fit; otherwise the
  // preallocated capacity is used and an overflow raises the overflow flag.
  // Returns the pair count when synchronised, -1 otherwise.
  int64_t bin(bool host_sync, cudaStream_t stream);
  // counts (device, 2 values) receives evaluated and contributing pairs when given.
  void forward(cudaStream_t stream, unsigned long long* counts = nullptr);
  // Loss and dL/drgb against `target` (the batch's pixels, 3 floats each).
  void loss(const float* target, float ssim_weight, int mode, float* grad_out,
            cudaStream_t stream);
  void backward(const float* dL_drgb, cudaStream_t stream);
  void param_grads(const float* params, float* grads, float* screen_gradient,
                   int32_t* visible_count, cudaStream_t stream);
  void reserve_pairs(int64_t capacity);
  void reserve_records(int64_t capacity);

  // sizes
  int N = 0, S = 0, V = 0;
  int64_t slot_stride = 0;
  ViewBatch batch;
  int64_t pair_capacity = 0;
  int64_t record_capacity = 0;
  int64_t last_pair_count = 0;
  int64_t last_record_count = 0;

  // device buffers
  DeviceArray<ViewDesc> d_views;
  DeviceArray<float2> xy;
  DeviceArray<float4> conic_op, color, debug_cov;
  DeviceArray<uint32_t> depth_key;
  DeviceArray<uint2> rect;
  DeviceArray<int32_t> tile_count;
  DeviceArray<uint32_t> sort_keys, sort_vals, sort_keys_alt, sort_vals_alt;
  // per (tile row, chunk of depth-sorted slots): records and their offsets
  DeviceArray<int32_t> row_chunk_counts;
  DeviceArray<int64_t> row_chunk_offsets, d_total_pairs, d_total_records;
  DeviceArray<uint32_t> rec_vals;  // tile-row records (slot ids) by row, near to far
  DeviceArray<uint32_t> rec_xr;    // each record's tile-column range (x0 | x1 << 16)
  DeviceArray<int2> row_ranges;
  DeviceArray<int32_t> tile_counts, chunk_counts, chunk_base, n_chunks;
  DeviceArray<int4> chunks;
  int64_t max_chunks = 0;
  DeviceArray<int64_t> tile_offsets;
  DeviceArray<uint32_t> tile_slots;  // per-tile key lists (pair_capacity)
  // per list entry, which 8x8 blocks of its tile took it (pair_capacity bytes),
  // written by the two-pixel forward pass for its adjoint
  DeviceArray<uint8_t> block_bits;
  bool have_block_bits = false;
  DeviceArray<uint32_t> hist, hist_scanned;
  DeviceArray<char> scan_scratch;
  DeviceArray<int2> ranges;
  // heaviest-first tile order (launch_tile_order) and the persistent
  // schedule's counters (forward, adjoint)
  DeviceArray<int32_t> tile_order, order_work, tickets;
  bool order_ready = false;
  const int* ordered_tiles(int schedule, cudaStream_t stream);
  DeviceArray<float> rgb, transmittance, dL;
  DeviceArray<int32_t> last;
  DeviceArray<double> loss_sums;
  DeviceArray<float> loss_per_view, loss_total;
  DeviceArray<ScreenGrad> screen;
  DeviceArray<int32_t> overflow;

  // after bin(): the per-tile lists and the depth-sorted slots
  uint32_t* sorted_pair_vals = nullptr;
  uint32_t* sorted_slots = nullptr;

 private:
  void ensure_scan_scratch(int64_t n);
  void ensure_chunks();
  ScanScratch scan_;
  int64_t scan_capacity_ = 0;
  bool configured_ = false;
};

}  // namespace pxs
