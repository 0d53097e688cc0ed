// raster_bwd.cu -- the adjoint of front-to-back compositing.
//
// rasterizeSplatsBackward, pixel pass (SplatRaster.cpp:346-433): each pixel
// walks its tile's list back to front from its last contributor (recorded by
// the forward kernel), dividing the transmittance back out rather than storing
// it per pair, and the per-splat screen-space gradients (dL/dmean, dL/dconic,
// dL/dopacity, dL/dcolor, |dL/dmean|) are summed over the tile's pixels:
//   * per warp with a 12-shuffle transpose-reduction of the ten values, which
//     leaves each of ten lanes holding one complete sum;
//   * per CTA in shared memory (eight warps add into the batch's accumulators);
//   * once per (tile, splat) into global memory with three 16-byte vector
//     reductions (red.global.add.v4.f32).
// The branch decisions (power > 0, the alpha floor, the 0.99 cap) are taken
// with the forward kernel's exact rounding (raster_common.cuh); the gradient
// arithmetic itself may use fused multiply-adds.
#include "common.cuh"
#include "kernels.h"
#include "raster_common.cuh"

namespace pxs {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// Sums v[0..9] over the warp. Returns, in ten of the even lanes, one complete
// sum; *idx is the index of that value, or -1 in the other lanes.
__device__ __forceinline__ float warp_reduce10(const float (&v)[10], int lane, int* idx) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
  float w[6];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const float send = b4 ? v[i] : v[i + 5];
    const float keep = b4 ? v[i + 5] : v[i];
    w[i] = keep + __shfl_xor_sync(kFull, send, 16);
  }
  w[5] = 0.f;
  float x[4];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float send = b3 ? w[i] : w[i + 3];
    const float keep = b3 ? w[i + 3] : w[i];
    x[i] = keep + __shfl_xor_sync(kFull, send, 8);
  }
  x[3] = 0.f;
  float y[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float send = b2 ? x[i] : x[i + 2];
    const float keep = b2 ? x[i + 2] : x[i];
    y[i] = keep + __shfl_xor_sync(kFull, send, 4);
  }
  const float send = b1 ? y[0] : y[1];
  const float keep = b1 ? y[1] : y[0];
  float z = keep + __shfl_xor_sync(kFull, send, 2);
  z += __shfl_xor_sync(kFull, z, 1);
  const int q = (b2 ? 2 : 0) + (b1 ? 1 : 0);
  const int p = (b3 ? 3 : 0) + q;
  *idx = ((lane & 1) == 0 && q < 3 && p < 5) ? (b4 ? 5 : 0) + p : -1;
  return z;
}

}  // namespace

template <int PX>
__global__ void __launch_bounds__(TileGeom<PX>::kThreads)
    k_backward(const int2* __restrict__ ranges, const uint32_t* __restrict__ pair_slots,
               const float2* __restrict__ xy, const float4* __restrict__ conic_op,
               const float4* __restrict__ color, const ViewDesc* __restrict__ views,
               int n_views, const float* __restrict__ T_final,
               const int32_t* __restrict__ last_in, const float* __restrict__ dL_drgb,
               ScreenGrad* __restrict__ screen) {
  constexpr int kThreads = TileGeom<PX>::kThreads;
  __shared__ uint32_t s_slot[kBatch];
  __shared__ float2 s_xy[kBatch];
  __shared__ float4 s_co[kBatch];
  __shared__ float4 s_col[kBatch];  // r, g, b, power floor
  __shared__ uint32_t s_mask[kBatch];
  __shared__ float s_acc[kBatch][12];
  __shared__ int s_hi;
  const TileInfo<PX> info = tile_info<PX>(views, n_views, ranges);
  const ViewDesc& vd = views[info.view];
  const float min_alpha = vd.min_alpha;
  const float fx = (float)info.px + 0.5f;
  const float bg0 = vd.background[0], bg1 = vd.background[1], bg2 = vd.background[2];
  // per pixel: dL/drgb, the final and the running transmittance, the suffix
  // colour, the previous contributor's alpha and colour, the last contributor
  float fy[PX], dLp0[PX], dLp1[PX], dLp2[PX], final_T[PX], T[PX], bg_term[PX];
  float suffix0[PX], suffix1[PX], suffix2[PX], last_alpha[PX], lc0[PX], lc1[PX], lc2[PX];
  int my_last[PX];
  int thread_hi = info.range.x;
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    const int py = info.py0 + 4 * p;
    fy[p] = (float)py + 0.5f;
    dLp0[p] = dLp1[p] = dLp2[p] = 0.f;
    final_T[p] = 1.f;
    my_last[p] = info.range.x;
    if (info.px < vd.cam.width && py < vd.cam.height) {
      const int64_t pixel = vd.pixel_offset + (int64_t)py * vd.cam.width + info.px;
      dLp0[p] = dL_drgb[pixel * 3 + 0];
      dLp1[p] = dL_drgb[pixel * 3 + 1];
      dLp2[p] = dL_drgb[pixel * 3 + 2];
      final_T[p] = T_final[pixel];
      my_last[p] = last_in[pixel];
    }
    T[p] = final_T[p];
    bg_term[p] = final_T[p] * (bg0 * dLp0[p] + bg1 * dLp1[p] + bg2 * dLp2[p]);
    suffix0[p] = suffix1[p] = suffix2[p] = 0.f;
    last_alpha[p] = lc0[p] = lc1[p] = lc2[p] = 0.f;
    thread_hi = max(thread_hi, my_last[p]);
  }
  const int lane = lane_id(), warp = warp_id();
  const int warp_hi = __reduce_max_sync(kFull, thread_hi);
  if (threadIdx.x == 0) s_hi = info.range.x;
  __syncthreads();
  if (lane == 0 && warp_hi > info.range.x) atomicMax(&s_hi, warp_hi);
  __syncthreads();
  const int hi = s_hi;

  for (int batch_end = hi; batch_end > info.range.x; batch_end -= kBatch) {
    const int batch_start = max(info.range.x, batch_end - kBatch);
    const int n = batch_end - batch_start;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kThreads) {
      const uint32_t slot = pair_slots[batch_start + i];
      const float4 co = conic_op[slot];
      const float2 mean = xy[slot];
      float4 c = color[slot];
      c.w = power_floor(co.w, min_alpha);
      s_slot[i] = slot;
      s_xy[i] = mean;
      s_co[i] = co;
      s_col[i] = c;
      s_mask[i] = warp_mask<PX>(mean, co, c.w, info.tile_px, info.tile_py);
#pragma unroll
      for (int k = 0; k < 12; ++k) s_acc[i][k] = 0.f;
    }
    __syncthreads();
    const int j_top = min(n, warp_hi - batch_start) - 1;  // warp-uniform
    for (int j = j_top; j >= 0; --j) {
      if (!((s_mask[j] >> warp) & 1u)) continue;  // the splat cannot reach this warp's pixels
      const int e = batch_start + j;
      const float2 m = s_xy[j];
      const float4 co = s_co[j];
      const float4 c = s_col[j];
      const float dx = fx - m.x;
      float v[10];
#pragma unroll
      for (int k = 0; k < 10; ++k) v[k] = 0.f;
      bool contrib = false, touched = false;
#pragma unroll
      for (int p = 0; p < PX; ++p) {
        if (e < my_last[p]) {
          const float dy = fy[p] - m.y;
          const float power = splat_power(co, dx, dy);
          if (!(power > 0.f) && !(power < c.w)) {
            const float gw = expf(power);
            const float raw_alpha = __fmul_rn(co.w, gw);
            const float alpha = raw_alpha < kMaxAlpha ? raw_alpha : kMaxAlpha;
            if (!(alpha < min_alpha)) {
              contrib = true;
              const float inv = __fdividef(1.f, 1.f - alpha);
              T[p] *= inv;
              const float weight = alpha * T[p];
              v[6] += weight * dLp0[p];
              v[7] += weight * dLp1[p];
              v[8] += weight * dLp2[p];
              const float la = last_alpha[p];
              suffix0[p] = la * lc0[p] + (1.f - la) * suffix0[p];
              suffix1[p] = la * lc1[p] + (1.f - la) * suffix1[p];
              suffix2[p] = la * lc2[p] + (1.f - la) * suffix2[p];
              lc0[p] = c.x;
              lc1[p] = c.y;
              lc2[p] = c.z;
              last_alpha[p] = alpha;
              float dL_dalpha = ((c.x - suffix0[p]) * dLp0[p] + (c.y - suffix1[p]) * dLp1[p] +
                                 (c.z - suffix2[p]) * dLp2[p]) * T[p];
              dL_dalpha -= inv * bg_term[p];
              if (raw_alpha < kMaxAlpha) {  // the cap flattens the gradient
                touched = true;
                v[5] += gw * dL_dalpha;  // dopacity
                const float dL_dweight = co.w * dL_dalpha;
                const float gx = gw * dx, gy = gw * dy;
                const float dm0 = dL_dweight * (-gx * co.x - gy * co.y);
                const float dm1 = dL_dweight * (-gy * co.z - gx * co.y);
                v[0] -= dm0;  // d(mean) = -d(delta)
                v[1] -= dm1;
                v[9] += sqrtf(dm0 * dm0 + dm1 * dm1);
                v[2] += -0.5f * dL_dweight * gx * dx;
                v[3] += -dL_dweight * gx * dy;
                v[4] += -0.5f * dL_dweight * gy * dy;
              }
            }
          }
        }
      }
      if (__any_sync(kFull, contrib)) {
        const bool any_touched = __any_sync(kFull, touched);
        int idx;
        const float sum = warp_reduce10(v, lane, &idx);
        float* a = s_acc[j];
        if (idx >= 0) atomicAdd(&a[idx], sum);
        if (lane == 1) {
          if (any_touched) atomicAdd(&a[10], 1.f);
          a[11] = 1.f;
        }
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kThreads) {
      const float* a = s_acc[i];
      if (a[11] != 0.f) {
        float* dst = reinterpret_cast<float*>(&screen[s_slot[i]]);
        red_add_v4(dst + 0, a[0], a[1], a[2], a[3]);
        red_add_v4(dst + 4, a[4], a[5], a[6], a[7]);
        red_add_v4(dst + 8, a[8], a[9], a[10], 0.f);
      }
    }
  }
}

namespace {

template <int PX>
void backward_px(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                 const float4* conic_op, const float4* color, const ViewDesc* views, int n_views,
                 int total_tiles, const float* T_final, const int32_t* last,
                 const float* dL_drgb, ScreenGrad* screen, cudaStream_t stream) {
  k_backward<PX><<<total_tiles, TileGeom<PX>::kThreads, 0, stream>>>(
      ranges, pair_slots, xy, conic_op, color, views, n_views, T_final, last, dL_drgb, screen);
}

}  // namespace

void launch_backward(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                     const float4* conic_op, const float4* color, const ViewDesc* views,
                     int n_views, int total_tiles, const float* T_final, const int32_t* last,
                     const float* dL_drgb, ScreenGrad* screen, cudaStream_t stream) {
  if (total_tiles <= 0) return;
  count_launch();
  switch (raster_config().backward_px) {
    case 1:
      backward_px<1>(ranges, pair_slots, xy, conic_op, color, views, n_views, total_tiles,
                     T_final, last, dL_drgb, screen, stream);
      break;
    case 4:
      backward_px<4>(ranges, pair_slots, xy, conic_op, color, views, n_views, total_tiles,
                     T_final, last, dL_drgb, screen, stream);
      break;
    default:
      backward_px<2>(ranges, pair_slots, xy, conic_op, color, views, n_views, total_tiles,
                     T_final, last, dL_drgb, screen, stream);
  }
}

}  // namespace pxs
