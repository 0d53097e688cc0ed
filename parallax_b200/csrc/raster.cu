// raster.cu -- front-to-back alpha compositing and its adjoint.
//
// One CTA per (view, 16x16 tile), one thread per pixel. Each tile's key list
// is walked in batches of 256 entries staged through shared memory; the CTA
// stops as soon as every pixel has reached the transmittance cutoff
// (__syncthreads_and). Arithmetic follows rasterizeSplats
// (SplatRaster.cpp:285-310) and rasterizeSplatsBackward (:346-433) term for
// term, rounded the same way (the file is compiled with -fmad=false); exp is
// CUDA's expf.
#include "common.cuh"
#include "kernels.h"

namespace pxs {
namespace {

constexpr int kBatch = 256;

struct TileInfo {
  int view;
  int px, py;  // this thread's pixel
  bool inside;
  int2 range;
};

__device__ __forceinline__ TileInfo tile_info(const ViewDesc* __restrict__ views, int n_views,
                                              const int2* __restrict__ ranges) {
  TileInfo info;
  const int tile = blockIdx.x;
  info.view = view_of_tile(views, n_views, tile);
  const ViewDesc& vd = views[info.view];
  const int local = tile - vd.tile_offset;
  const int tx = local % vd.tiles_x, ty = local / vd.tiles_x;
  info.px = tx * kTile + (threadIdx.x % kTile);
  info.py = ty * kTile + (threadIdx.x / kTile);
  info.inside = info.px < vd.cam.width && info.py < vd.cam.height;
  info.range = ranges[tile];
  return info;
}

}  // namespace

// rasterizeSplats (SplatRaster.cpp:265-315). Writes rgb (+ T * background),
// the final transmittance and, for the adjoint, one past the index of the
// last entry that contributed (the `last` of SplatRaster.cpp:363-376).
// With kCount it also counts the (pixel, entry) pairs the loop evaluates and
// those that pass both alpha tests into counts[0] and counts[1].
template <bool kCount>
__global__ void __launch_bounds__(kTilePixels)
    k_forward(const int2* __restrict__ ranges, const uint32_t* __restrict__ pair_slots,
              const float2* __restrict__ xy, const float4* __restrict__ conic_op,
              const float4* __restrict__ color, const ViewDesc* __restrict__ views, int n_views,
              float* __restrict__ rgb_out, float* __restrict__ T_out,
              int32_t* __restrict__ last_out, unsigned long long* __restrict__ counts) {
  __shared__ float2 s_xy[kBatch];
  __shared__ float4 s_co[kBatch];
  __shared__ float4 s_col[kBatch];
  const TileInfo info = tile_info(views, n_views, ranges);
  const ViewDesc& vd = views[info.view];
  const float min_alpha = vd.min_alpha, cutoff = vd.transmittance_cutoff;
  const float fx = (float)info.px + 0.5f, fy = (float)info.py + 0.5f;
  float T = 1.f;
  float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f;
  int last = info.range.x;
  bool done = !info.inside;
  unsigned long long evaluated = 0, contributing = 0;
  for (int base = info.range.x; base < info.range.y; base += kBatch) {
    if (__syncthreads_and(done)) break;
    const int idx = base + (int)threadIdx.x;
    if (idx < info.range.y) {
      const uint32_t slot = pair_slots[idx];
      s_xy[threadIdx.x] = xy[slot];
      s_co[threadIdx.x] = conic_op[slot];
      s_col[threadIdx.x] = color[slot];
    }
    __syncthreads();
    const int n = min(kBatch, info.range.y - base);
    if (!done) {
      for (int j = 0; j < n; ++j) {
        const float2 m = s_xy[j];
        const float4 co = s_co[j];
        const float dx = fx - m.x, dy = fy - m.y;
        const float power = -0.5f * (co.x * dx * dx + co.z * dy * dy) - co.y * dx * dy;
        if (kCount) ++evaluated;
        if (power > 0.f) continue;
        float alpha = co.w * expf(power);
        alpha = alpha < kMaxAlpha ? alpha : kMaxAlpha;
        if (alpha < min_alpha) continue;
        if (kCount) ++contributing;
        const float4 c = s_col[j];
        const float ta = T * alpha;
        acc0 += ta * c.x;
        acc1 += ta * c.y;
        acc2 += ta * c.z;
        T *= 1.f - alpha;
        last = base + j + 1;
        if (T < cutoff) {
          done = true;
          break;
        }
      }
    }
  }
  if (info.inside) {
    const int64_t pixel = vd.pixel_offset + (int64_t)info.py * vd.cam.width + info.px;
    rgb_out[pixel * 3 + 0] = acc0 + T * vd.background[0];
    rgb_out[pixel * 3 + 1] = acc1 + T * vd.background[1];
    rgb_out[pixel * 3 + 2] = acc2 + T * vd.background[2];
    if (T_out != nullptr) T_out[pixel] = T;
    last_out[pixel] = last;
  }
  if (kCount) {
    for (int o = 16; o > 0; o >>= 1) {
      evaluated += __shfl_xor_sync(0xffffffffu, evaluated, o);
      contributing += __shfl_xor_sync(0xffffffffu, contributing, o);
    }
    if (lane_id() == 0) {
      atomicAdd(&counts[0], evaluated);
      atomicAdd(&counts[1], contributing);
    }
  }
}

// rasterizeSplatsBackward, pixel pass (SplatRaster.cpp:346-433). Walks each
// pixel's list back to front from its last contributor, dividing the
// transmittance back out, and adds the per-splat screen-space gradients into
// `screen` (one ScreenGrad per slot): per warp by shuffles, per CTA in shared
// memory, then one vector reduction per (tile, splat) into global memory.
__global__ void __launch_bounds__(kTilePixels)
    k_backward(const int2* __restrict__ ranges, const uint32_t* __restrict__ pair_slots,
               const float2* __restrict__ xy, const float4* __restrict__ conic_op,
               const float4* __restrict__ color, const ViewDesc* __restrict__ views,
               int n_views, const float* __restrict__ T_final,
               const int32_t* __restrict__ last_in, const float* __restrict__ dL_drgb,
               ScreenGrad* __restrict__ screen) {
  __shared__ uint32_t s_slot[kBatch];
  __shared__ float2 s_xy[kBatch];
  __shared__ float4 s_co[kBatch];
  __shared__ float4 s_col[kBatch];
  __shared__ float s_acc[kBatch][12];
  __shared__ int s_hi;
  const TileInfo info = tile_info(views, n_views, ranges);
  const ViewDesc& vd = views[info.view];
  const float min_alpha = vd.min_alpha;
  const float fx = (float)info.px + 0.5f, fy = (float)info.py + 0.5f;
  float dLp0 = 0.f, dLp1 = 0.f, dLp2 = 0.f, final_T = 1.f;
  int my_last = info.range.x;
  if (info.inside) {
    const int64_t pixel = vd.pixel_offset + (int64_t)info.py * vd.cam.width + info.px;
    dLp0 = dL_drgb[pixel * 3 + 0];
    dLp1 = dL_drgb[pixel * 3 + 1];
    dLp2 = dL_drgb[pixel * 3 + 2];
    final_T = T_final[pixel];
    my_last = last_in[pixel];
  }
  if (threadIdx.x == 0) s_hi = info.range.x;
  __syncthreads();
  if (my_last > info.range.x) atomicMax(&s_hi, my_last);
  __syncthreads();
  const int hi = s_hi;
  float T = final_T;
  float suffix0 = 0.f, suffix1 = 0.f, suffix2 = 0.f;
  float last_alpha = 0.f, lc0 = 0.f, lc1 = 0.f, lc2 = 0.f;
  float background_term = 0.f;
  background_term += vd.background[0] * dLp0;
  background_term += vd.background[1] * dLp1;
  background_term += vd.background[2] * dLp2;
  const int lane = lane_id();

  for (int batch_end = hi; batch_end > info.range.x; batch_end -= kBatch) {
    const int batch_start = max(info.range.x, batch_end - kBatch);
    const int n = batch_end - batch_start;
    __syncthreads();
    if ((int)threadIdx.x < n) {
      const uint32_t slot = pair_slots[batch_start + threadIdx.x];
      s_slot[threadIdx.x] = slot;
      s_xy[threadIdx.x] = xy[slot];
      s_co[threadIdx.x] = conic_op[slot];
      s_col[threadIdx.x] = color[slot];
#pragma unroll
      for (int k = 0; k < 12; ++k) s_acc[threadIdx.x][k] = 0.f;
    }
    __syncthreads();
    for (int j = n - 1; j >= 0; --j) {
      const int e = batch_start + j;
      float v[11];
#pragma unroll
      for (int k = 0; k < 11; ++k) v[k] = 0.f;
      bool contrib = false;
      if (e < my_last) {
        const float2 m = s_xy[j];
        const float4 co = s_co[j];
        const float dx = fx - m.x, dy = fy - m.y;
        const float power = -0.5f * (co.x * dx * dx + co.z * dy * dy) - co.y * dx * dy;
        if (!(power > 0.f)) {
          const float gw = expf(power);
          const float raw_alpha = co.w * gw;
          const float alpha = raw_alpha < kMaxAlpha ? raw_alpha : kMaxAlpha;
          if (!(alpha < min_alpha)) {
            contrib = true;
            const float4 c = s_col[j];
            T /= 1.f - alpha;
            const float weight = alpha * T;
            float dL_dalpha = 0.f;
            v[5] = weight * dLp0;
            suffix0 = last_alpha * lc0 + (1.f - last_alpha) * suffix0;
            lc0 = c.x;
            dL_dalpha += (c.x - suffix0) * T * dLp0;
            v[6] = weight * dLp1;
            suffix1 = last_alpha * lc1 + (1.f - last_alpha) * suffix1;
            lc1 = c.y;
            dL_dalpha += (c.y - suffix1) * T * dLp1;
            v[7] = weight * dLp2;
            suffix2 = last_alpha * lc2 + (1.f - last_alpha) * suffix2;
            lc2 = c.z;
            dL_dalpha += (c.z - suffix2) * T * dLp2;
            last_alpha = alpha;
            dL_dalpha += -final_T / (1.f - alpha) * background_term;
            if (raw_alpha < kMaxAlpha) {
              v[4] = gw * dL_dalpha;                       // dopacity
              const float dL_dweight = co.w * dL_dalpha;
              const float gx = gw * dx, gy = gw * dy;
              const float dm0 = dL_dweight * (-gx * co.x - gy * co.y);
              const float dm1 = dL_dweight * (-gy * co.z - gx * co.y);
              v[0] = -dm0;                                 // dmean (sign flipped)
              v[1] = -dm1;
              v[8] = sqrtf(dm0 * dm0 + dm1 * dm1);         // |dmean|
              v[2] = -0.5f * dL_dweight * gx * dx;         // dconic
              v[3] = -1.0f * dL_dweight * gx * dy;
              v[9] = -0.5f * dL_dweight * gy * dy;
              v[10] = 1.f;                                 // touched
            }
          }
        }
      }
      if (__any_sync(0xffffffffu, contrib)) {
#pragma unroll
        for (int k = 0; k < 11; ++k) v[k] = warp_sum(v[k]);
        if (lane == 0) {
          float* a = s_acc[j];
          atomicAdd(&a[0], v[0]);
          atomicAdd(&a[1], v[1]);
          atomicAdd(&a[2], v[2]);
          atomicAdd(&a[3], v[3]);
          atomicAdd(&a[4], v[9]);
          atomicAdd(&a[5], v[4]);
          atomicAdd(&a[6], v[5]);
          atomicAdd(&a[7], v[6]);
          atomicAdd(&a[8], v[7]);
          atomicAdd(&a[9], v[8]);
          atomicAdd(&a[10], v[10]);
          a[11] = 1.f;  // any contribution: flush this entry
        }
      }
    }
    __syncthreads();
    if ((int)threadIdx.x < n) {
      const float* a = s_acc[threadIdx.x];
      if (a[11] != 0.f) {
        float* dst = reinterpret_cast<float*>(&screen[s_slot[threadIdx.x]]);
        red_add_v4(dst + 0, a[0], a[1], a[2], a[3]);
        red_add_v4(dst + 4, a[4], a[5], a[6], a[7]);
        red_add_v4(dst + 8, a[8], a[9], a[10], 0.f);
      }
    }
  }
}

void launch_forward(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                    const float4* conic_op, const float4* color, const ViewDesc* views,
                    int n_views, int total_tiles, float* rgb, float* T, int32_t* last,
                    cudaStream_t stream, unsigned long long* counts) {
  if (total_tiles > 0) {
    count_launch();
    if (counts != nullptr)
      k_forward<true><<<total_tiles, kTilePixels, 0, stream>>>(
          ranges, pair_slots, xy, conic_op, color, views, n_views, rgb, T, last, counts);
    else
      k_forward<false><<<total_tiles, kTilePixels, 0, stream>>>(
          ranges, pair_slots, xy, conic_op, color, views, n_views, rgb, T, last, nullptr);
  }
}

void launch_backward(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                     const float4* conic_op, const float4* color, const ViewDesc* views,
                     int n_views, int total_tiles, const float* T_final, const int32_t* last,
                     const float* dL_drgb, ScreenGrad* screen, cudaStream_t stream) {
  if (total_tiles > 0) {
    count_launch();
    k_backward<<<total_tiles, kTilePixels, 0, stream>>>(ranges, pair_slots, xy, conic_op, color,
                                                        views, n_views, T_final, last, dL_drgb,
                                                        screen);
  }
}

}  // namespace pxs
