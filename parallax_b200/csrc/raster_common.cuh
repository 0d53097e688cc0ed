// raster_common.cuh -- per-tile helpers shared by the compositing kernel and
// its adjoint. The adjoint must take exactly the forward's branch decisions
// (power > 0, the alpha floor, the 0.99 cap), so the per-pair quantities are
// evaluated here with non-contracting intrinsics: the same rounding whatever
// -fmad setting the including file is compiled with.
#pragma once

#include "common.cuh"

namespace pxs {

constexpr int kBatch = 256;

// Pixels per thread. A warp covers an 8-wide block of 4*PX rows: lane l owns
// column l%8 and the PX adjacent rows PX*(l/8) + p (p < PX); warp w covers
// columns 8*(w%2) .. +8 and rows 4*PX*(w/2) .. +4*PX of the 16x16 tile. PX = 1 gives 8 warps of 8x4,
// PX = 2 4 warps of 8x8, PX = 4 2 warps of 8x16. More pixels per thread share
// each staged entry and each warp-level reduction among more pixels.
template <int PX>
struct TileGeom {
  static constexpr int kThreads = kTilePixels / PX;
  static constexpr int kWarps = kThreads / 32;
  static constexpr int kBlockH = 4 * PX;
};

template <int PX>
struct TileInfo {
  int view;
  int px;      // this thread's column
  int py0;     // its first row; pixel p is at row py0 + p
  int tile_px, tile_py;
  int2 range;
};

template <int PX>
__device__ __forceinline__ TileInfo<PX> tile_info(const ViewDesc* __restrict__ views,
                                                  int n_views, const int2* __restrict__ ranges,
                                                  int tile) {
  TileInfo<PX> info;
  info.view = view_of_tile(views, n_views, tile);
  const ViewDesc& vd = views[info.view];
  const int local = tile - vd.tile_offset;
  const int tx = local % vd.tiles_x, ty = local / vd.tiles_x;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  info.tile_px = tx * kTile;
  info.tile_py = ty * kTile;
  info.px = info.tile_px + (w & 1) * 8 + (lane & 7);
  info.py0 = info.tile_py + (w >> 1) * TileGeom<PX>::kBlockH + PX * (lane >> 3);
  info.range = ranges[tile];
  return info;
}

template <int PX>
__device__ __forceinline__ TileInfo<PX> tile_info(const ViewDesc* __restrict__ views,
                                                  int n_views, const int2* __restrict__ ranges) {
  return tile_info<PX>(views, n_views, ranges, (int)blockIdx.x);
}

// CTAs of `kernel` with `threads` threads that are resident on the current
// device at once: the grid of a persistent launch.
template <typename Kernel>
inline int resident_ctas(Kernel kernel, int threads) {
  int device = 0, sms = 1, per_sm = 1;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  return (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
}

// How the two-pixel compositing kernel and its adjoint map CTAs to tiles
// (RasterConfig::forward_schedule / backward_schedule):
//   kTileOrder   one CTA per tile, in tile order;
//   kHeavyFirst  one CTA per tile, tiles with the longest lists first
//                (tile = order[blockIdx.x]; the block scheduler starts
//                CTAs roughly in index order);
//   kPersistent  as many CTAs as fit on the device, each taking the next
//                tile of that order from a device counter until none is left.
enum TileSchedule { kTileOrder = 0, kHeavyFirst = 1, kPersistent = 2 };

// Runs body(tile) for the tiles of this CTA under a schedule. `order` is the
// heaviest-first tile order (schedules 1 and 2), `ticket` the counter of the
// persistent schedule, zero at launch.
template <typename Body>
__device__ __forceinline__ void for_each_tile(int schedule, const int* __restrict__ order,
                                              int* __restrict__ ticket, int total_tiles,
                                              Body&& body) {
  if (schedule == kTileOrder) {
    body((int)blockIdx.x);
    return;
  }
  if (schedule == kHeavyFirst) {
    body(order[blockIdx.x]);
    return;
  }
  __shared__ int s_next;
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(ticket, 1);
    __syncthreads();
    const int item = s_next;
    __syncthreads();  // every thread has read it before thread 0 takes the next
    if (item >= total_tiles) break;
    body(order[item]);
  }
}

// Paired FP32 multiply, add and fused multiply-add (f32x2) as inline PTX
// with round-to-nearest. Each component rounds as the scalar __fmul_rn /
// __fadd_rn / __fmaf_rn does (checked against them on random pairs). A paired
// add whose operand is a paired product was nevertheless found contracted
// into one rounding in the generated code, so the exact paths never feed a
// paired product straight into a paired add (splat_power2); the compositing
// tests hold the two-pixel kernels' transmittance bit-identical to the
// one-pixel kernel's scalar arithmetic.
__device__ __forceinline__ unsigned long long f2_to_b64(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 b64_to_f2(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ float2 mul2_rn(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_to_b64(a)), "l"(f2_to_b64(b)));
  return b64_to_f2(d);
}
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_to_b64(a)), "l"(f2_to_b64(b)));
  return b64_to_f2(d);
}

__device__ __forceinline__ float2 fma2_rn(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;"
      : "=l"(d) : "l"(f2_to_b64(a)), "l"(f2_to_b64(b)), "l"(f2_to_b64(c)));
  return b64_to_f2(d);
}

// The hardware square-root approximation (relative error about 2^-22).
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// The least q(dx, dy) = a dx^2 + 2 b dx dy + c dy^2 of a conic (a, b, c) =
// (co.x, co.y, co.z), positive definite, over the rectangle [dx0, dx1] x
// [dy0, dy1]: 0 when it holds the origin, else on its boundary, where each
// edge's least value is at the edge's stationary point clamped to the edge.
__device__ __forceinline__ float rect_min_q(const float4& co, float dx0, float dx1, float dy0,
                                            float dy1) {
  if (dx0 <= 0.f && dx1 >= 0.f && dy0 <= 0.f && dy1 >= 0.f) return 0.f;
  const float a = co.x, b = co.y, c = co.z;
  const float ia = __fdividef(1.f, a), ic = __fdividef(1.f, c);
  auto q = [&](float x, float y) { return a * x * x + 2.f * b * x * y + c * y * y; };
  auto clampf = [](float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); };
  float best = q(dx0, clampf(-b * dx0 * ic, dy0, dy1));
  best = fminf(best, q(dx1, clampf(-b * dx1 * ic, dy0, dy1)));
  best = fminf(best, q(clampf(-b * dy0 * ia, dx0, dx1), dy0));
  best = fminf(best, q(clampf(-b * dy1 * ia, dx0, dx1), dy1));
  return best;
}

// Bit w is set when some pixel of warp w's block may see this splat with
// power >= `floor` (and so possibly alpha >= min_alpha), i.e. q = -2 power <=
// k = -2 floor somewhere in the block. The region
// {d : d^T A d <= -2 floor} of the conic A lies in the box
// |dx| <= sqrt(-2 floor (A^-1)_xx), |dy| <= sqrt(-2 floor (A^-1)_yy); the box is
// widened by 10% and half a pixel, which covers the rounding of the computed
// power for any splat narrower than ~1000 px of standard deviation (wider ones
// get every bit). No floor (min_alpha = 0) sets every bit. With kRefine the
// box's blocks are tested against the ellipse itself (below); it costs
// registers, so only the compositing pass, which walks by these masks, uses it.
template <int PX, bool kRefine = false>
__device__ __forceinline__ uint32_t warp_mask(float2 mean, const float4& co, float floor,
                                              int tile_px, int tile_py) {
  constexpr uint32_t kAll = (1u << TileGeom<PX>::kWarps) - 1u;
  if (!(floor > -1e30f)) return kAll;
  const float det = co.x * co.z - co.y * co.y;
  if (!(det > 0.f)) return kAll;
  // hardware approximations (relative error ~1e-7): the 10% widening covers them
  const float k = -2.f * floor;
  const float inv_det = __fdividef(1.f, det);
  const float ex = sqrt_approx(k * co.z * inv_det) * 1.1f + 0.5f;
  const float ey = sqrt_approx(k * co.x * inv_det) * 1.1f + 0.5f;
  if (!(ex < 1e4f && ey < 1e4f)) return kAll;
  // a block whose box test passes is then dropped when the least q over its
  // rectangle of pixel centres exceeds k: the footprint ellipse misses it
  // although the box does not. Only for conics with a c < 10 det (|rho| <=
  // 0.95): the absolute terms of q then sum to at most 38 q, so the float
  // rounding of q, here and in the kernels' per-pixel power, stays ten times
  // under the margin below. More elongated splats keep the box test alone.
  const bool refine = kRefine && co.x * co.z < 10.f * det;
  const float q_cut = k * 1.0001f + 1e-4f;
  uint32_t m = 0u;
#pragma unroll
  for (int w = 0; w < TileGeom<PX>::kWarps; ++w) {
    const float x_lo = (float)(tile_px + (w & 1) * 8) + 0.5f, x_hi = x_lo + 7.f;
    const float y_lo = (float)(tile_py + (w >> 1) * TileGeom<PX>::kBlockH) + 0.5f;
    const float y_hi = y_lo + (float)(TileGeom<PX>::kBlockH - 1);
    if (x_lo <= mean.x + ex && x_hi >= mean.x - ex && y_lo <= mean.y + ey &&
        y_hi >= mean.y - ey &&
        !(refine &&
          rect_min_q(co, x_lo - mean.x, x_hi - mean.x, y_lo - mean.y, y_hi - mean.y) > q_cut))
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

// splat_power for the two pixels (dx, dy.x) and (dx, dy.y) of one column,
// with the reference's roundings:
// - the products that only involve dx are shared scalars;
// - the products (c dy) dy and (-b dx) dy are paired operations that round
//   as the scalar ones (mul2_rn);
// - a + b, with one operand a paired product, stays scalar: the code
//   generator was found to contract a paired add fed by a paired product
//   into one rounding;
// - the last step, -0.5 (t1 + t2) - b dx dy, is one paired fused
//   multiply-add. Halving is exact, so the fused product -0.5 s equals its
//   rounded value (s >= 2^-125; a smaller nonzero s needs a conic entry
//   below about 1e-24, a footprint of 1e12 pixels), and the addition of
//   (-b dx) dy = -(b dx dy) equals the subtraction exactly, as rounding to
//   nearest is symmetric.
__device__ __forceinline__ float2 splat_power2(const float4& co, float dx, float2 dy) {
  const float t1 = __fmul_rn(__fmul_rn(co.x, dx), dx);
  const float nbdx = __fmul_rn(-co.y, dx);
  const float2 t2 = mul2_rn(mul2_rn(make_float2(co.z, co.z), dy), dy);
  const float2 s = make_float2(__fadd_rn(t1, t2.x), __fadd_rn(t1, t2.y));
  return fma2_rn(make_float2(-0.5f, -0.5f), s, mul2_rn(make_float2(nbdx, nbdx), dy));
}

// exp(power) for alpha = opacity * exp(power) (SplatRaster.cpp:298), in
// every compositing kernel and its adjoint, so that both take the same
// entries. It is the hardware exponential (__expf): its documented error is
// at most 2 + floor(1.173 |power|) ulp, at most 8 ulp (5e-7 relative) for the
// powers the alpha floor lets through (power >= ln(1/255) - 1e-5 > -5.55),
// against the reference's correctly rounded std::exp. The error moves a pixel's
// colour by a like relative amount, and flips an alpha test only where the
// value lies within that distance of its threshold. It keeps the FP32 range
// handling of expf off the ALU pipe, which compositing and its adjoint are
// bound by (C4 step 17.65 -> 17.22 ms).
__device__ __forceinline__ float splat_exp(float power) { return __expf(power); }

// A power below which opacity * exp(power) is certainly under min_alpha, so
// exp need not be evaluated: ln(min_alpha / opacity) less a 1e-5 margin. The
// quotient and the log are the hardware approximations (at most 3 ulp, under
// 2e-6 in log space for the |ln| <= 5.6 that opacity >= min_alpha allows);
// the margin covers them and the error of splat_exp and the product. -inf
// when min_alpha is 0.
__device__ __forceinline__ float power_floor(float opacity, float min_alpha) {
  return __logf(__fdividef(min_alpha, opacity)) - 1e-5f;
}

}  // namespace pxs
