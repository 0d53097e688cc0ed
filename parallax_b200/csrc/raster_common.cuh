// raster_common.cuh -- per-tile helpers shared by the compositing kernel and
// its adjoint. The adjoint must take exactly the forward's branch decisions
// (power > 0, the alpha floor, the 0.99 cap), so the per-pair quantities are
// evaluated here with non-contracting intrinsics: the same rounding whatever
// -fmad setting the including file is compiled with.
#pragma once

#include "common.cuh"

namespace pxs {

constexpr int kBatch = 256;

struct TileInfo {
  int view;
  int px, py;  // this thread's pixel
  bool inside;
  int2 range;
};

// Threads map to pixels by warps of 8x4 (warp w covers columns
// 8*(w%2) .. +8 and rows 4*(w/2) .. +4 of the 16x16 tile), so a warp's pixels
// are compact and can skip the entries whose footprint misses them.
__device__ __forceinline__ TileInfo tile_info(const ViewDesc* __restrict__ views, int n_views,
                                              const int2* __restrict__ ranges) {
  TileInfo info;
  const int tile = blockIdx.x;
  info.view = view_of_tile(views, n_views, tile);
  const ViewDesc& vd = views[info.view];
  const int local = tile - vd.tile_offset;
  const int tx = local % vd.tiles_x, ty = local / vd.tiles_x;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  info.px = tx * kTile + (w & 1) * 8 + (lane & 7);
  info.py = ty * kTile + (w >> 1) * 4 + (lane >> 3);
  info.inside = info.px < vd.cam.width && info.py < vd.cam.height;
  info.range = ranges[tile];
  return info;
}

// Bit w is set when some pixel of warp w's 8x4 block may see this splat with
// power >= `floor` (and so possibly alpha >= min_alpha). The region
// {d : d^T A d <= -2 floor} of the conic A lies in the box
// |dx| <= sqrt(-2 floor (A^-1)_xx), |dy| <= sqrt(-2 floor (A^-1)_yy); the box is
// widened by 10% and half a pixel, which covers the rounding of the computed
// power for any splat narrower than ~1000 px of standard deviation (wider ones
// get every bit). No floor (min_alpha = 0) sets every bit.
__device__ __forceinline__ uint32_t warp_mask(float2 mean, const float4& co, float floor,
                                              int tile_px, int tile_py) {
  if (!(floor > -1e30f)) return 0xFFu;
  const float det = co.x * co.z - co.y * co.y;
  if (!(det > 0.f)) return 0xFFu;
  const float k = -2.f * floor;
  const float ex = sqrtf(k * co.z / det) * 1.1f + 0.5f;
  const float ey = sqrtf(k * co.x / det) * 1.1f + 0.5f;
  if (!(ex < 1e4f && ey < 1e4f)) return 0xFFu;
  uint32_t m = 0u;
#pragma unroll
  for (int w = 0; w < 8; ++w) {
    const float x_lo = (float)(tile_px + (w & 1) * 8) + 0.5f, x_hi = x_lo + 7.f;
    const float y_lo = (float)(tile_py + (w >> 1) * 4) + 0.5f, y_hi = y_lo + 3.f;
    if (x_lo <= mean.x + ex && x_hi >= mean.x - ex && y_lo <= mean.y + ey &&
        y_hi >= mean.y - ey)
      m |= 1u << w;
  }
  return m;
}

// -0.5 (a dx^2 + c dy^2) - b dx dy, each product and sum rounded in the
// reference's order (SplatRaster.cpp:295-297).
__device__ __forceinline__ float splat_power(const float4& co, float dx, float dy) {
  const float t1 = __fmul_rn(__fmul_rn(co.x, dx), dx);
  const float t2 = __fmul_rn(__fmul_rn(co.z, dy), dy);
  const float t3 = __fmul_rn(__fmul_rn(co.y, dx), dy);
  return __fsub_rn(__fmul_rn(-0.5f, __fadd_rn(t1, t2)), t3);
}

// A power below which opacity * exp(power) is certainly under min_alpha, so
// exp need not be evaluated: ln(min_alpha / opacity) less a 1e-5 margin that
// covers the rounding of logf, expf and the product (all far below 1e-6 in
// log space for the |ln| <= 5.6 that opacity >= min_alpha allows). -inf when
// min_alpha is 0.
__device__ __forceinline__ float power_floor(float opacity, float min_alpha) {
  return logf(min_alpha / opacity) - 1e-5f;
}

}  // namespace pxs
