// common.cuh -- shared device definitions of the splat training core (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pxs.h"

namespace pxs {

constexpr int kTile = PXS_TILE;           // logical binning tile, pixels
constexpr int kTilePixels = kTile * kTile;
constexpr float kMaxAlpha = 0.99f;        // SplatRaster.cpp:22
constexpr float kFrustumSlack = 1.3f;     // SplatRaster.cpp:26
constexpr float kShC0 = 0.28209479177387814f;  // GaussianCloud.h:54

// Items per radix-sort block tile; the per-view slot stride is padded to it so
// a sort block never straddles two views.
constexpr int kSortThreads = 256;
constexpr int kSortItemsPerThread = 16;
constexpr int kSortTile = kSortThreads * kSortItemsPerThread;

constexpr uint32_t kCulledKey = 0xFFFFFFFFu;

// Widest image, in tiles, the row-binning kernels stage in shared memory.
constexpr int kMaxTilesX = 2048;
constexpr int kMaxTilesY = 2048;

// Everything a kernel needs to know about one view of a batch.
struct ViewDesc {
  pxs_camera cam;
  float background[3];
  int32_t sh_degree;         // min(options.sh_degree, cloud sh_degree)
  int32_t tiles_x, tiles_y;
  int32_t tile_offset;       // first global tile id of this view
  int32_t row_offset;        // first global tile-row id of this view
  int64_t pixel_offset;      // first pixel of this view in the image arrays
  float min_alpha;
  float transmittance_cutoff;
  float screen_dilation;
  int32_t loss_tile_offset;  // first output tile of this view in the loss kernel's flat grid
  int64_t target_offset;     // first pixel of this view's target image
  // the gaussians this view renders: [gauss_offset, gauss_offset + gauss_count)
  // of the parameter arrays; slot v * slot_stride + i holds gaussian
  // gauss_offset + i (one cloud: 0 and N for every view; a batch of several
  // independent scenes: each view's own scene)
  int32_t gauss_offset;
  int32_t gauss_count;
};

// Per-step screen-space gradient accumulators of one (view, gaussian) slot
// (the per-splat vectors of SplatRaster.cpp:337-342), 12 floats, 16-byte aligned.
struct alignas(16) ScreenGrad {
  float dmean[2];
  float dconic[3];
  float dopacity;
  float dcolor[3];
  float dmean_abs;
  float touched;  // 1 when any pixel reached the uncapped-alpha branch
  float pad;
};
static_assert(sizeof(ScreenGrad) == 48, "ScreenGrad layout");

// Device views of the per-slot projection outputs.
struct ProjectedSoA {
  float2* xy;          // mean
  float4* conic_op;    // conic (a, b, c), opacity
  float4* color;       // r, g, b, clamp flags (bits in .w)
  uint32_t* depth_key; // float bits of depth; kCulledKey when culled
  uint2* rect;         // x0 | x1 << 16, y0 | y1 << 16 (tile coordinates)
  int32_t* tile_count; // tiles touched
  float4* debug_cov;   // optional: cov2d (xx, xy, yy), radius
};

__host__ __device__ inline int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Kernel launches issued by this library (host counter, bumped at every
// launch site; a captured graph's count is taken while capturing).
extern int64_t g_kernel_launches;
inline void count_launch() { ++g_kernel_launches; }

#if defined(__CUDACC__)
__device__ inline int warp_id() { return threadIdx.x >> 5; }
__device__ inline int lane_id() { return threadIdx.x & 31; }

__device__ inline unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Inclusive warp scan of a 32-bit integer.
__device__ inline int warp_inclusive_scan(int v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane_id() >= o) v += n;
  }
  return v;
}

__device__ inline int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ inline float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Vector reduction to global memory (sm_90+): one L2 atomic for four floats.
__device__ inline void red_add_v4(float* address, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(address), "f"(a), "f"(b),
               "f"(c), "f"(d)
               : "memory");
}

// Looks up which view of a batch a global tile belongs to (views are few).
__device__ inline int view_of_tile(const ViewDesc* views, int n_views, int tile) {
  int v = 0;
  while (v + 1 < n_views && views[v + 1].tile_offset <= tile) ++v;
  return v;
}
#endif  // __CUDACC__

}  // namespace pxs
