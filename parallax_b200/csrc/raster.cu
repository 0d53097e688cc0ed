// raster.cu -- front-to-back alpha compositing.
//
// One CTA per (view, 16x16 tile), one thread per pixel. Each tile's key list
// is walked in batches of 256 entries staged through shared memory; the CTA
// stops as soon as every pixel has reached the transmittance cutoff
// (__syncthreads_and). Arithmetic follows rasterizeSplats
// (SplatRaster.cpp:285-310) term for term, rounded the same way (the file is
// compiled with -fmad=false); exp is CUDA's expf, skipped only where the
// alpha floor certainly rejects the pair (power_floor).
#include "common.cuh"
#include "kernels.h"
#include "raster_common.cuh"

namespace pxs {

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
  __shared__ float4 s_col[kBatch];  // r, g, b, power floor
  __shared__ uint32_t s_mask[kBatch];
  const TileInfo info = tile_info(views, n_views, ranges);
  const int warp = threadIdx.x >> 5;
  const int tile_px = info.px - (info.px % kTile), tile_py = info.py - (info.py % kTile);
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
      const float4 co = conic_op[slot];
      const float2 mean = xy[slot];
      float4 c = color[slot];
      c.w = power_floor(co.w, min_alpha);
      s_xy[threadIdx.x] = mean;
      s_co[threadIdx.x] = co;
      s_col[threadIdx.x] = c;
      s_mask[threadIdx.x] = warp_mask(mean, co, c.w, tile_px, tile_py);
    }
    __syncthreads();
    const int n = min(kBatch, info.range.y - base);
    if (!done) {
      for (int j = 0; j < n; ++j) {
        if (!((s_mask[j] >> warp) & 1u)) {  // the splat cannot reach this warp's pixels
          if (kCount) ++evaluated;
          continue;
        }
        const float2 m = s_xy[j];
        const float4 co = s_co[j];
        const float dx = fx - m.x, dy = fy - m.y;
        const float power = splat_power(co, dx, dy);
        if (kCount) ++evaluated;
        if (power > 0.f || power < s_col[j].w) continue;
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

}  // namespace pxs
