// raster.cu -- front-to-back alpha compositing.
//
// One CTA per (view, 16x16 tile), PX pixels per thread (1, 2 or 4, chosen by
// the raster configuration; raster_common.cuh). Each tile's key list
// is walked in batches of 256 entries staged through shared memory; the CTA
// stops as soon as every pixel has reached the transmittance cutoff
// (__syncthreads_and). Arithmetic follows rasterizeSplats
// (SplatRaster.cpp:285-310) term for term, rounded the same way (the file is
// compiled with -fmad=false); exp is splat_exp (the hardware exponential,
// raster_common.cuh), skipped only where the alpha floor certainly rejects the
// pair (power_floor).
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "raster_common.cuh"

namespace pxs {

RasterConfig& raster_config() {
  static RasterConfig config;
  return config;
}

// rasterizeSplats (SplatRaster.cpp:265-315). Writes rgb (+ T * background),
// the final transmittance and, for the adjoint, one past the index of the
// last entry that contributed (the `last` of SplatRaster.cpp:363-376).
// Each thread composites PX pixels of one column (TileGeom). With kCount it
// also counts the (pixel, entry) pairs the loop evaluates and those that pass
// both alpha tests into counts[0] and counts[1].
template <bool kCount, int PX>
__global__ void __launch_bounds__(TileGeom<PX>::kThreads)
    k_forward(const int2* __restrict__ ranges, const uint32_t* __restrict__ pair_slots,
              const float2* __restrict__ xy, const float4* __restrict__ conic_op,
              const float4* __restrict__ color, const ViewDesc* __restrict__ views, int n_views,
              float* __restrict__ rgb_out, float* __restrict__ T_out,
              int32_t* __restrict__ last_out, unsigned long long* __restrict__ counts) {
  constexpr int kThreads = TileGeom<PX>::kThreads;
  __shared__ float2 s_xy[kBatch];
  __shared__ float4 s_co[kBatch];
  __shared__ float4 s_col[kBatch];  // r, g, b, power floor
  __shared__ uint32_t s_mask[kBatch];
  const TileInfo<PX> info = tile_info<PX>(views, n_views, ranges);
  const int warp = threadIdx.x >> 5;
  const ViewDesc& vd = views[info.view];
  const float min_alpha = vd.min_alpha, cutoff = vd.transmittance_cutoff;
  const float fx = (float)info.px + 0.5f;
  float fy[PX], T[PX], acc0[PX], acc1[PX], acc2[PX];
  int last[PX];
  bool done[PX];
  bool all_done = true;
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    fy[p] = (float)(info.py0 + p) + 0.5f;
    T[p] = 1.f;
    acc0[p] = acc1[p] = acc2[p] = 0.f;
    last[p] = info.range.x;
    done[p] = !(info.px < vd.cam.width && info.py0 + p < vd.cam.height);
    all_done = all_done && done[p];
  }
  unsigned long long evaluated = 0, contributing = 0;
  for (int base = info.range.x; base < info.range.y; base += kBatch) {
    if (__syncthreads_and(all_done)) break;
    const int n = min(kBatch, info.range.y - base);
    for (int i = threadIdx.x; i < n; i += kThreads) {
      const uint32_t slot = pair_slots[base + i];
      const float4 co = conic_op[slot];
      const float2 mean = xy[slot];
      float4 c = color[slot];
      c.w = power_floor(co.w, min_alpha);
      s_xy[i] = mean;
      s_co[i] = co;
      s_col[i] = c;
      s_mask[i] = warp_mask<PX>(mean, co, c.w, info.tile_px, info.tile_py);
    }
    __syncthreads();
    if (!all_done) {
      for (int j = 0; j < n; ++j) {
        if (!((s_mask[j] >> warp) & 1u)) {  // the splat cannot reach this warp's pixels
          if (kCount) {
#pragma unroll
            for (int p = 0; p < PX; ++p) evaluated += done[p] ? 0 : 1;
          }
          continue;
        }
        const float2 m = s_xy[j];
        const float4 co = s_co[j];
        const float floor = s_col[j].w;
        const float dx = fx - m.x;
        bool now_done = true;
#pragma unroll
        for (int p = 0; p < PX; ++p) {
          if (!done[p]) {
            if (kCount) ++evaluated;
            const float dy = fy[p] - m.y;
            const float power = splat_power(co, dx, dy);
            if (!(power > 0.f || power < floor)) {
              float alpha = co.w * splat_exp(power);
              alpha = alpha < kMaxAlpha ? alpha : kMaxAlpha;
              if (!(alpha < min_alpha)) {
                if (kCount) ++contributing;
                const float4 c = s_col[j];
                const float ta = T[p] * alpha;
                acc0[p] += ta * c.x;
                acc1[p] += ta * c.y;
                acc2[p] += ta * c.z;
                T[p] *= 1.f - alpha;
                last[p] = base + j + 1;
                if (T[p] < cutoff) done[p] = true;
              }
            }
          }
          now_done = now_done && done[p];
        }
        if (now_done) {
          all_done = true;
          break;
        }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < PX; ++p) {
    const int py = info.py0 + p;
    if (info.px < vd.cam.width && py < vd.cam.height) {
      const int64_t pixel = vd.pixel_offset + (int64_t)py * vd.cam.width + info.px;
      rgb_out[pixel * 3 + 0] = acc0[p] + T[p] * vd.background[0];
      rgb_out[pixel * 3 + 1] = acc1[p] + T[p] * vd.background[1];
      rgb_out[pixel * 3 + 2] = acc2[p] + T[p] * vd.background[2];
      if (T_out != nullptr) T_out[pixel] = T[p];
      last_out[pixel] = last[p];
    }
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

// The two-pixel form of k_forward: each thread composites two vertically
// adjacent pixels of one column. Power, alpha and transmittance round as the
// scalar operations of k_forward (so the same entries are taken and T is
// bit-identical); the colour sums of the two pixels are one paired fused
// multiply-add per channel (fma.rn.f32x2), which differs from the separate
// multiply and add by at most one rounding per entry. A pixel that does not
// take an entry adds T * 0 * colour = 0.
// kFwdBatch entries are staged per batch (RasterConfig::forward_batch: 64, 128
// or 256; 128 by default -- a tile stops at saturation, so a smaller batch
// stages fewer entries past it); `schedule` maps CTAs to tiles (for_each_tile).
template <bool kCount, bool kBits, int kFwdBatch>
__global__ void __launch_bounds__(TileGeom<2>::kThreads, 8)
    k_forward_x2(const int2* __restrict__ ranges, const uint32_t* __restrict__ pair_slots,
                 const float2* __restrict__ xy, const float4* __restrict__ conic_op,
                 const float4* __restrict__ color, const ViewDesc* __restrict__ views,
                 int n_views, float* __restrict__ rgb_out, float* __restrict__ T_out,
                 int32_t* __restrict__ last_out, unsigned long long* __restrict__ counts,
                 uint8_t* __restrict__ block_bits, int schedule, const int* __restrict__ order,
                 int* __restrict__ ticket, int total_tiles) {
  constexpr int kThreads = TileGeom<2>::kThreads;
  __shared__ float2 s_xy[kFwdBatch];  // -mean
  __shared__ float4 s_co[kFwdBatch];  // conic, -opacity
  __shared__ float4 s_col[kFwdBatch];  // -r, -g, -b, 0
  __shared__ uint32_t s_mask[kFwdBatch];
  __shared__ uint8_t s_took[TileGeom<2>::kWarps][kFwdBatch];  // warp w = 8x8 block w
  __shared__ uint8_t s_list[TileGeom<2>::kWarps][kFwdBatch];  // a warp's entries of the batch
  static_assert(kFwdBatch <= 256, "batch indices are bytes");
  for_each_tile(schedule, order, ticket, total_tiles, [&](int tile) {
  const TileInfo<2> info = tile_info<2>(views, n_views, ranges, tile);
  const int warp = threadIdx.x >> 5;
  const ViewDesc& vd = views[info.view];
  const float min_alpha = vd.min_alpha, cutoff = vd.transmittance_cutoff;
  const float neg_min_alpha = -min_alpha;
  const float fx = (float)info.px + 0.5f;
  const float2 fy = make_float2((float)info.py0 + 0.5f, (float)(info.py0 + 1) + 0.5f);
  const bool col_in = info.px < vd.cam.width;
  bool done0 = !(col_in && info.py0 < vd.cam.height);
  bool done1 = !(col_in && info.py0 + 1 < vd.cam.height);
  float2 T = make_float2(1.f, 1.f);
  float2 acc0 = make_float2(0.f, 0.f), acc1 = acc0, acc2 = acc0;
  int last0 = info.range.x, last1 = info.range.x;
  unsigned long long evaluated = 0, contributing = 0;
  int prev_base = 0, prev_n = 0;  // the batch whose block bits are pending
  // block bits of the pending batch out to global memory, one byte per entry
  auto write_bits = [&]() {
    for (int i = threadIdx.x; i < prev_n; i += kThreads)
      block_bits[prev_base + i] = (uint8_t)(s_took[0][i] | (s_took[1][i] << 1) |
                                            (s_took[2][i] << 2) | (s_took[3][i] << 3));
  };
  for (int base = info.range.x; base < info.range.y; base += kFwdBatch) {
    const bool all_done = __syncthreads_and(done0 && done1);
    if (kBits) {
      write_bits();
      prev_n = 0;
    }
    if (all_done) break;
    if (kBits) __syncthreads();  // the bits are read before they are cleared
    const int n = min(kFwdBatch, info.range.y - base);
    for (int i = threadIdx.x; i < n; i += kThreads) {
      if (kBits) {
#pragma unroll
        for (int w = 0; w < TileGeom<2>::kWarps; ++w) s_took[w][i] = 0;
      }
      const uint32_t slot = pair_slots[base + i];
      const float4 co = conic_op[slot];
      const float2 mean = xy[slot];
      const float4 c = color[slot];
      // staged negated (see visit): the mean, the opacity and the colour
      s_xy[i] = make_float2(-mean.x, -mean.y);
      s_co[i] = make_float4(co.x, co.y, co.z, -co.w);
      s_col[i] = make_float4(-c.x, -c.y, -c.z, 0.f);
      s_mask[i] = warp_mask<2, true>(mean, co, power_floor(co.w, min_alpha), info.tile_px,
                                     info.tile_py);
    }
    __syncthreads();
    // entry j for this warp's pixels; returns whether both are done. The two
    // pixels' operations run as paired f32x2 instructions with the scalar
    // roundings (mul2_rn, add2_rn). The mean, opacity and colour are staged
    // negated, and each negation is exact and undone exactly: fx + (-mx) is
    // fx - mx; (-o) e is -(o e), so alpha's tests and cap are mirrored;
    // (-T alpha)(-r) is (T alpha) r in the colour FMA; 1 + (-alpha) is
    // 1 - alpha.
    auto visit = [&](int j) -> bool {
      const float2 nm = s_xy[j];
      const float4 co = s_co[j];
      const float dx = fx + nm.x;
      const float2 dy = add2_rn(fy, make_float2(nm.y, nm.y));
      const float2 power = splat_power2(co, dx, dy);
      // (the power floor only spares the exp elsewhere: below it alpha is
      // certainly under min_alpha, so the alpha test decides the same)
      const bool in0 = !done0 && !(power.x > 0.f);
      const bool in1 = !done1 && !(power.y > 0.f);
      // No early return for an entry that misses both pixels: a pixel that
      // does not take the entry adds T * 0 to its colour and keeps T, so the
      // body runs branch-free across the warp (measured 2.8% faster at C4).
      // -alpha, read only where c0 / c1 (which include in0 / in1) hold, so
      // it needs no zeroing outside them
      float2 na = mul2_rn(make_float2(co.w, co.w),
                          make_float2(splat_exp(power.x), splat_exp(power.y)));
      na.x = na.x > -kMaxAlpha ? na.x : -kMaxAlpha;
      na.y = na.y > -kMaxAlpha ? na.y : -kMaxAlpha;
      const bool c0 = in0 && !(na.x > neg_min_alpha);
      const bool c1 = in1 && !(na.y > neg_min_alpha);
      if (kCount) contributing += (c0 ? 1 : 0) + (c1 ? 1 : 0);
      if (kBits && (c0 || c1)) s_took[warp][j] = 1;  // same value from every lane
      const float4 nc = s_col[j];
      // -alpha where the pixel takes the entry, else 0: the colour weight is
      // then T * 0 = 0 and T * (1 + 0) = T is exact, so T needs no select
      const float2 nac = make_float2(c0 ? na.x : 0.f, c1 ? na.y : 0.f);
      const float2 nta = mul2_rn(T, nac);
      acc0 = __ffma2_rn(nta, make_float2(nc.x, nc.x), acc0);
      acc1 = __ffma2_rn(nta, make_float2(nc.y, nc.y), acc1);
      acc2 = __ffma2_rn(nta, make_float2(nc.z, nc.z), acc2);
      T = mul2_rn(T, add2_rn(make_float2(1.f, 1.f), nac));
      last0 = c0 ? base + j + 1 : last0;
      last1 = c1 ? base + j + 1 : last1;
      // T changes only where the pixel takes the entry, and a pixel is done
      // once its T is below the cutoff, so no test of c0 / c1 is needed
      done0 = done0 || T.x < cutoff;
      done1 = done1 || T.y < cutoff;
      return done0 && done1;
    };
    if (kCount) {
      if (!(done0 && done1)) {
        // every entry counts as evaluated for each pixel not yet done
        for (int j = 0; j < n; ++j) {
          evaluated += (done0 ? 0 : 1) + (done1 ? 0 : 1);
          if (!((s_mask[j] >> warp) & 1u)) continue;  // cannot reach this warp's pixels
          if (visit(j)) break;
        }
      }
    } else {
      // the entries whose footprint can reach this warp's block, ascending;
      // built by the whole warp (every lane is here, after the barrier above)
      // before each lane walks it for its own pixels
      const int lane = threadIdx.x & 31;
      int n_mine = 0;
      for (int j0 = 0; j0 < n; j0 += 32) {
        const int jj = j0 + lane;
        const bool mine = jj < n && ((s_mask[jj] >> warp) & 1u);
        const unsigned b = __ballot_sync(0xffffffffu, mine);
        if (mine) s_list[warp][n_mine + __popc(b & lanemask_lt())] = (uint8_t)jj;
        n_mine += __popc(b);
      }
      __syncwarp();
      if (!(done0 && done1))
#pragma unroll 8
        for (int q = 0; q < n_mine; ++q)
          if (visit(s_list[warp][q])) break;
    }
    prev_base = base;
    prev_n = n;
  }
  if (kBits && prev_n > 0) {  // the last batch, when the list ran out
    __syncthreads();
    write_bits();
  }
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const int py = info.py0 + p;
    if (col_in && py < vd.cam.height) {
      const float Tp = p ? T.y : T.x;
      const int64_t pixel = vd.pixel_offset + (int64_t)py * vd.cam.width + info.px;
      rgb_out[pixel * 3 + 0] = (p ? acc0.y : acc0.x) + Tp * vd.background[0];
      rgb_out[pixel * 3 + 1] = (p ? acc1.y : acc1.x) + Tp * vd.background[1];
      rgb_out[pixel * 3 + 2] = (p ? acc2.y : acc2.x) + Tp * vd.background[2];
      if (T_out != nullptr) T_out[pixel] = Tp;
      last_out[pixel] = p ? last1 : last0;
    }
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
  });
}

// ------------------------------------------------ heaviest-first tile order

__device__ __forceinline__ int length_class(int2 r) {
  const int len = r.y - r.x;
  return len > 1 ? 31 - __clz(len) : 0;  // floor(log2), 0 for 0 and 1
}

// work[0..31]: tiles per length class
__global__ void k_tile_class_counts(const int2* __restrict__ ranges, int total_tiles,
                                    int* __restrict__ work) {
  __shared__ int s_count[32];
  if (threadIdx.x < 32) s_count[threadIdx.x] = 0;
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < total_tiles) atomicAdd(&s_count[length_class(ranges[t])], 1);
  __syncthreads();
  if (threadIdx.x < 32 && s_count[threadIdx.x] > 0) atomicAdd(&work[threadIdx.x], s_count[threadIdx.x]);
}

// work[32 + c]: where class c starts, the longest class first
__global__ void k_tile_class_offsets(int* __restrict__ work) {
  const int lane = threadIdx.x;  // one warp
  const int c = 31 - lane;      // lane 0 holds the longest class
  const int n = work[c];
  int x = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  work[32 + c] = x - n;
}

__global__ void k_tile_class_scatter(const int2* __restrict__ ranges, int total_tiles,
                                     int* __restrict__ work, int* __restrict__ order) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total_tiles) return;
  order[atomicAdd(&work[32 + length_class(ranges[t])], 1)] = t;
}

void launch_tile_order(const int2* ranges, int total_tiles, int* order, int* work,
                       cudaStream_t stream) {
  if (total_tiles <= 0) return;
  const int blocks = (total_tiles + 255) / 256;
  cudaMemsetAsync(work, 0, sizeof(int) * 32, stream);
  count_launch();
  k_tile_class_counts<<<blocks, 256, 0, stream>>>(ranges, total_tiles, work);
  count_launch();
  k_tile_class_offsets<<<1, 32, 0, stream>>>(work);
  count_launch();
  k_tile_class_scatter<<<blocks, 256, 0, stream>>>(ranges, total_tiles, work, order);
}

namespace {

template <bool kCount, int PX>
void forward_px(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                const float4* conic_op, const float4* color, const ViewDesc* views, int n_views,
                int total_tiles, float* rgb, float* T, int32_t* last, cudaStream_t stream,
                unsigned long long* counts) {
  k_forward<kCount, PX><<<total_tiles, TileGeom<PX>::kThreads, 0, stream>>>(
      ranges, pair_slots, xy, conic_op, color, views, n_views, rgb, T, last, counts);
}

// The two-pixel kernel at the configured batch and schedule. The counting
// form always runs one CTA per tile in tile order.
template <bool kCount, bool kBits, int B>
void forward_x2_launch(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                       const float4* conic_op, const float4* color, const ViewDesc* views,
                       int n_views, int total_tiles, float* rgb, float* T, int32_t* last,
                       cudaStream_t stream, unsigned long long* counts, uint8_t* bits,
                       const int* order, int* ticket) {
  const RasterConfig& rc = raster_config();
  const int schedule = (kCount || order == nullptr) ? kTileOrder : rc.forward_schedule;
  int grid = total_tiles;
  if (schedule == kPersistent) {
    grid = std::min(total_tiles, resident_ctas(k_forward_x2<kCount, kBits, B>,
                                               TileGeom<2>::kThreads));
    cudaMemsetAsync(ticket, 0, sizeof(int), stream);
  }
  k_forward_x2<kCount, kBits, B><<<grid, TileGeom<2>::kThreads, 0, stream>>>(
      ranges, pair_slots, xy, conic_op, color, views, n_views, rgb, T, last, counts, bits,
      schedule, order, ticket, total_tiles);
}

template <bool kCount>
void forward_x2_dispatch(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                         const float4* conic_op, const float4* color, const ViewDesc* views,
                         int n_views, int total_tiles, float* rgb, float* T, int32_t* last,
                         cudaStream_t stream, unsigned long long* counts, uint8_t* bits,
                         const int* order, int* ticket) {
#define PXS_FWD(BITS, B)                                                                    \
  forward_x2_launch<kCount, BITS, B>(ranges, pair_slots, xy, conic_op, color, views, n_views, \
                                     total_tiles, rgb, T, last, stream, counts, bits, order,  \
                                     ticket)
  const int b = raster_config().forward_batch;
  if (bits != nullptr) {
    if (b == 64) PXS_FWD(true, 64);
    else if (b == 256) PXS_FWD(true, 256);
    else PXS_FWD(true, 128);
  } else {
    if (b == 64) PXS_FWD(false, 64);
    else if (b == 256) PXS_FWD(false, 256);
    else PXS_FWD(false, 128);
  }
#undef PXS_FWD
}

template <bool kCount>
void forward_dispatch(int px, const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                      const float4* conic_op, const float4* color, const ViewDesc* views,
                      int n_views, int total_tiles, float* rgb, float* T, int32_t* last,
                      cudaStream_t stream, unsigned long long* counts, uint8_t* bits,
                      const int* order, int* ticket) {
  switch (px) {
    case 1:
      forward_px<kCount, 1>(ranges, pair_slots, xy, conic_op, color, views, n_views,
                            total_tiles, rgb, T, last, stream, counts);
      break;
    case 4:
      forward_px<kCount, 4>(ranges, pair_slots, xy, conic_op, color, views, n_views,
                            total_tiles, rgb, T, last, stream, counts);
      break;
    default:
      forward_x2_dispatch<kCount>(ranges, pair_slots, xy, conic_op, color, views, n_views,
                                  total_tiles, rgb, T, last, stream, counts, bits, order,
                                  ticket);
  }
}

}  // namespace

bool launch_forward(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                    const float4* conic_op, const float4* color, const ViewDesc* views,
                    int n_views, int total_tiles, float* rgb, float* T, int32_t* last,
                    cudaStream_t stream, unsigned long long* counts, uint8_t* block_bits,
                    const int* tile_order, int* ticket) {
  if (total_tiles <= 0) return false;
  count_launch();
  const int px = raster_config().forward_px;
  uint8_t* bits = (px == 1 || px == 4) ? nullptr : block_bits;
  if (counts != nullptr)
    forward_dispatch<true>(px, ranges, pair_slots, xy, conic_op, color, views, n_views,
                           total_tiles, rgb, T, last, stream, counts, bits, tile_order, ticket);
  else
    forward_dispatch<false>(px, ranges, pair_slots, xy, conic_op, color, views, n_views,
                            total_tiles, rgb, T, last, stream, nullptr, bits, tile_order,
                            ticket);
  return bits != nullptr;
}

}  // namespace pxs
