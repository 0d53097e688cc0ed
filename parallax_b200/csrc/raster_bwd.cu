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
#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "raster_common.cuh"

namespace pxs {
namespace {

constexpr unsigned kFull = 0xffffffffu;
// At most this many contributing lanes: per-lane shared-memory atomics
// instead of the warp-wide transpose reduction.
constexpr int kDirectLanes = 1;

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
    const int py = info.py0 + p;
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
            const float gw = splat_exp(power);
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
                v[9] += sqrt_approx(dm0 * dm0 + dm1 * dm1);
                v[2] += -0.5f * dL_dweight * gx * dx;
                v[3] += -dL_dweight * gx * dy;
                v[4] += -0.5f * dL_dweight * gy * dy;
              }
            }
          }
        }
      }
      const unsigned ballot = __ballot_sync(kFull, contrib);
      if (ballot != 0u) {
        float* a = s_acc[j];
        if (__popc(ballot) <= kDirectLanes) {
          // few lanes: each adds its own sums, cheaper than the warp reduction
          if (contrib) {
#pragma unroll
            for (int k = 0; k < 10; ++k) atomicAdd(&a[k], v[k]);
            if (touched) a[10] = 1.f;
            a[11] = 1.f;
          }
        } else {
          const bool any_touched = __any_sync(kFull, touched);
          int idx;
          const float sum = warp_reduce10(v, lane, &idx);
          if (idx >= 0) atomicAdd(&a[idx], sum);
          if (lane == 1) {
            if (any_touched) a[10] = 1.f;
            a[11] = 1.f;
          }
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

// Warp w's bit in a tile-list entry's mask for the adjoint with PX pixels per
// thread, from the forward's block bits (bit b: some pixel of 8x8 block b of
// the two-pixel layout took the entry). With four pixels per thread warp w
// covers the two-pixel blocks w and w + 2.
template <int PX>
__device__ __forceinline__ uint32_t mask_from_block_bits(uint32_t bits) {
  if constexpr (PX == 2) return bits;
  else return (bits | (bits >> 2)) & 3u;
}

// The paired-FP32 forms of k_backward, with NP pairs of vertically adjacent
// pixels per thread (NP = 1: two pixels, 8x8 blocks per warp; NP = 2: four
// pixels, 8x16 blocks). The gradient arithmetic of a pair runs as the halves
// of paired FP32 instructions (fma/add/mul .f32x2). The branch decisions are
// the forward's, from operations that round as its own (splat_power2, alpha
// = opacity * exp). The body has no branches on them: a pixel that does not
// take an entry runs the paired arithmetic with alpha = 0 and a zero loss
// gradient, so its transmittance (multiplied by 1), its suffix colour (an FMA
// with a zero weight) and its sums are unchanged; almost every warp has some
// lane that takes the entry, so branching around the arithmetic only added
// divergence handling (adjoint 8.87 -> 7.81 ms per C4 step). A thread adds
// its pairs' contributions before the warp reduction, so one reduction serves
// 2 NP pixels per lane.
// kB entries are staged per batch (RasterConfig::backward_batch: 64, 128 or
// 256 with two pixels per thread; 128 with four, where fewer threads share a
// batch); `schedule` maps CTAs to tiles (for_each_tile).
template <int NP, int kB>
__global__ void __launch_bounds__(TileGeom<2 * NP>::kThreads)
    k_backward_pairs(const int2* __restrict__ ranges, const uint32_t* __restrict__ pair_slots,
                     const float2* __restrict__ xy, const float4* __restrict__ conic_op,
                     const float4* __restrict__ color, const ViewDesc* __restrict__ views,
                     int n_views, const float* __restrict__ T_final,
                     const int32_t* __restrict__ last_in, const float* __restrict__ dL_drgb,
                     ScreenGrad* __restrict__ screen, const uint8_t* __restrict__ block_bits,
                     int schedule, const int* __restrict__ order, int* __restrict__ ticket,
                     int total_tiles) {
  constexpr int PX = 2 * NP;
  constexpr int kThreads = TileGeom<PX>::kThreads;
  constexpr int kWarps = TileGeom<PX>::kWarps;
  __shared__ uint32_t s_slot[kB];
  __shared__ float2 s_xy[kB];
  __shared__ float4 s_co[kB];
  __shared__ float4 s_col[kB];  // r, g, b (w unused)
  __shared__ uint32_t s_mask[kB];
  __shared__ float s_acc[kB][12];
  __shared__ uint8_t s_list[kWarps][kB];  // a warp's entries of the batch
  __shared__ int s_hi;
  static_assert(kB <= 256, "batch indices are bytes");
  for_each_tile(schedule, order, ticket, total_tiles, [&](int tile) {
  const TileInfo<PX> info = tile_info<PX>(views, n_views, ranges, tile);
  const ViewDesc& vd = views[info.view];
  const float min_alpha = vd.min_alpha;
  const float fx = (float)info.px + 0.5f;
  const float2 zero2 = make_float2(0.f, 0.f);
  float2 fy[NP], dLp0[NP], dLp1[NP], dLp2[NP], T[NP], bg_term[NP];
  int last0[NP], last1[NP];
  int hi_mine = info.range.x;
#pragma unroll
  for (int q = 0; q < NP; ++q) {
    const int py = info.py0 + 2 * q;
    fy[q] = make_float2((float)py + 0.5f, (float)(py + 1) + 0.5f);
    dLp0[q] = dLp1[q] = dLp2[q] = zero2;
    T[q] = make_float2(1.f, 1.f);
    last0[q] = last1[q] = info.range.x;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      if (info.px < vd.cam.width && py + p < vd.cam.height) {
        const int64_t pixel = vd.pixel_offset + (int64_t)(py + p) * vd.cam.width + info.px;
        const float d0 = dL_drgb[pixel * 3 + 0], d1 = dL_drgb[pixel * 3 + 1];
        const float d2 = dL_drgb[pixel * 3 + 2], tf = T_final[pixel];
        const int l = last_in[pixel];
        if (p == 0) {
          dLp0[q].x = d0; dLp1[q].x = d1; dLp2[q].x = d2; T[q].x = tf; last0[q] = l;
        } else {
          dLp0[q].y = d0; dLp1[q].y = d1; dLp2[q].y = d2; T[q].y = tf; last1[q] = l;
        }
      }
    }
    // final T times the background's share of the loss gradient
    bg_term[q] = __fmul2_rn(
        T[q], __ffma2_rn(make_float2(vd.background[2], vd.background[2]), dLp2[q],
                         __ffma2_rn(make_float2(vd.background[1], vd.background[1]), dLp1[q],
                                    __fmul2_rn(make_float2(vd.background[0],
                                                           vd.background[0]),
                                               dLp0[q]))));
    hi_mine = max(hi_mine, max(last0[q], last1[q]));
  }
  // the colour composited behind the current entry (the reference's
  // accum_rec), updated with each entry once its gradient is taken
  float2 suffix0[NP], suffix1[NP], suffix2[NP];
#pragma unroll
  for (int q = 0; q < NP; ++q) suffix0[q] = suffix1[q] = suffix2[q] = zero2;
  const int lane = lane_id(), warp = warp_id();
  const int warp_hi = __reduce_max_sync(kFull, hi_mine);
  if (threadIdx.x == 0) s_hi = info.range.x;
  __syncthreads();
  if (lane == 0 && warp_hi > info.range.x) atomicMax(&s_hi, warp_hi);
  __syncthreads();
  const int hi = s_hi;

  for (int batch_end = hi; batch_end > info.range.x; batch_end -= kB) {
    const int batch_start = max(info.range.x, batch_end - kB);
    const int n = batch_end - batch_start;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kThreads) {
      const uint32_t slot = pair_slots[batch_start + i];
      const float4 co = conic_op[slot];
      const float2 mean = xy[slot];
      s_slot[i] = slot;
      s_xy[i] = make_float2(-mean.x, -mean.y);  // negated: fx + (-mx) is fx - mx
      s_co[i] = co;
      s_col[i] = color[slot];
      // which warps took the entry in the forward pass (exact), else which
      // ones its footprint can reach
      s_mask[i] = block_bits != nullptr
                      ? mask_from_block_bits<PX>(block_bits[batch_start + i])
                      : warp_mask<PX>(mean, co, power_floor(co.w, min_alpha), info.tile_px,
                                      info.tile_py);
#pragma unroll
      for (int k = 0; k < 12; ++k) s_acc[i][k] = 0.f;
    }
    __syncthreads();
    const int j_top = min(n, warp_hi - batch_start) - 1;  // warp-uniform
    // the entries some pixel of this warp takes (or can reach), ascending;
    // built by the whole warp, which is converged here
    int n_mine = 0;
    for (int j0 = 0; j0 <= j_top; j0 += 32) {
      const int jj = j0 + lane;
      const bool mine = jj <= j_top && ((s_mask[jj] >> warp) & 1u);
      const unsigned b = __ballot_sync(kFull, mine);
      if (mine) s_list[warp][n_mine + __popc(b & lanemask_lt())] = (uint8_t)jj;
      n_mine += __popc(b);
    }
    __syncwarp();
    for (int qi = n_mine - 1; qi >= 0; --qi) {  // back to front
      const int j = s_list[warp][qi];
      const int e = batch_start + j;
      const float2 nm = s_xy[j];
      const float4 co = s_co[j];
      const float4 c = s_col[j];
      const float dx = fx + nm.x;
      bool contrib = false, touched = false;
      float v[10];
#pragma unroll
      for (int k = 0; k < 10; ++k) v[k] = 0.f;
      // pair q's sums into v: assigned by the first pair, added by the next
      auto put = [&](int q, int k, float x) {
        if (q == 0) v[k] = x;
        else v[k] += x;
      };
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        const float2 dy = add2_rn(fy[q], make_float2(nm.y, nm.y));
        const float2 power = splat_power2(co, dx, dy);
        // no power-floor test: below the floor alpha is certainly under
        // min_alpha, so the alpha test below decides the same
        const bool in0 = e < last0[q] && !(power.x > 0.f);
        const bool in1 = e < last1[q] && !(power.y > 0.f);
        // not zeroed outside in0 / in1: every gradient term carries g through
        // z or dLw, which are 0 there, and g is finite (a conic of a positive
        // definite covariance gives power <= 0, so g <= 1)
        const float g0 = splat_exp(power.x);
        const float g1 = splat_exp(power.y);
        const float2 r = mul2_rn(make_float2(co.w, co.w), make_float2(g0, g1));
        const float r0 = r.x, r1 = r.y;
        const float a0 = r0 < kMaxAlpha ? r0 : kMaxAlpha;
        const float a1 = r1 < kMaxAlpha ? r1 : kMaxAlpha;
        const bool c0 = in0 && !(a0 < min_alpha);
        const bool c1 = in1 && !(a1 < min_alpha);
        contrib = contrib || c0 || c1;
        const float2 alpha = make_float2(c0 ? a0 : 0.f, c1 ? a1 : 0.f);
        // the reciprocals for both pixels, then 1 where the pixel does not
        // take the entry (its T stays as it is)
        const float q0 = __fdividef(1.f, 1.f - alpha.x), q1 = __fdividef(1.f, 1.f - alpha.y);
        const float2 inv = make_float2(c0 ? q0 : 1.f, c1 ? q1 : 1.f);
        T[q] = __fmul2_rn(T[q], inv);
        const float2 weight = __fmul2_rn(alpha, T[q]);
        const float2 w6 = __fmul2_rn(weight, dLp0[q]);
        const float2 w7 = __fmul2_rn(weight, dLp1[q]);
        const float2 w8 = __fmul2_rn(weight, dLp2[q]);
        put(q, 6, w6.x + w6.y);
        put(q, 7, w7.x + w7.y);
        put(q, 8, w8.x + w8.y);
        // colour minus what lies behind (SplatRaster.cpp:399-405), then the
        // entry joins what lies behind for the entries in front of it:
        // suffix += alpha (colour - suffix), which leaves a pixel that does
        // not take the entry (alpha 0) unchanged
        const float2 d0 = __fadd2_rn(make_float2(c.x, c.x), make_float2(-suffix0[q].x, -suffix0[q].y));
        const float2 d1 = __fadd2_rn(make_float2(c.y, c.y), make_float2(-suffix1[q].x, -suffix1[q].y));
        const float2 d2c = __fadd2_rn(make_float2(c.z, c.z), make_float2(-suffix2[q].x, -suffix2[q].y));
        float2 dL_dalpha = __fmul2_rn(
            __ffma2_rn(d2c, dLp2[q], __ffma2_rn(d1, dLp1[q], __fmul2_rn(d0, dLp0[q]))), T[q]);
        dL_dalpha = __ffma2_rn(make_float2(-inv.x, -inv.y), bg_term[q], dL_dalpha);
        suffix0[q] = __ffma2_rn(alpha, d0, suffix0[q]);
        suffix1[q] = __ffma2_rn(alpha, d1, suffix1[q]);
        suffix2[q] = __ffma2_rn(alpha, d2c, suffix2[q]);
        // the 0.99 cap flattens the gradient
        const bool t0 = c0 && r0 < kMaxAlpha, t1 = c1 && r1 < kMaxAlpha;
        touched = touched || t0 || t1;
        const float2 z = make_float2(t0 ? dL_dalpha.x : 0.f, t1 ? dL_dalpha.y : 0.f);
        const float2 gw = make_float2(g0, g1);
        const float2 qo = __fmul2_rn(gw, z);  // dL/dopacity per pixel
        const float2 dLw = __fmul2_rn(make_float2(co.w, co.w), z);
        const float2 gx = __fmul2_rn(gw, make_float2(dx, dx));
        const float2 gy = __fmul2_rn(gw, dy);
        // d(mean) = -d(delta): v0 = -dm0, v1 = -dm1
        const float2 dm0 = __fmul2_rn(
            dLw, __ffma2_rn(gy, make_float2(-co.y, -co.y),
                            __fmul2_rn(gx, make_float2(-co.x, -co.x))));
        const float2 dm1 = __fmul2_rn(
            dLw, __ffma2_rn(gx, make_float2(-co.y, -co.y),
                            __fmul2_rn(gy, make_float2(-co.z, -co.z))));
        const float2 sq = __ffma2_rn(dm1, dm1, __fmul2_rn(dm0, dm0));
        const float2 wx = __fmul2_rn(dLw, gx);
        const float2 wy = __fmul2_rn(dLw, gy);
        const float2 d2 = __fmul2_rn(wx, make_float2(-0.5f * dx, -0.5f * dx));
        const float2 d3 = __fmul2_rn(wx, make_float2(-dy.x, -dy.y));
        const float2 d4 = __fmul2_rn(wy, __fmul2_rn(make_float2(-0.5f, -0.5f), dy));
        put(q, 0, -(dm0.x + dm0.y));
        put(q, 1, -(dm1.x + dm1.y));
        put(q, 2, d2.x + d2.y);
        put(q, 3, d3.x + d3.y);
        put(q, 4, d4.x + d4.y);
        put(q, 5, qo.x + qo.y);
        // |d(mean)| for the densification statistic (a sum of per-pixel norms
        // compared against a threshold): the square-root approximation
        put(q, 9, sqrt_approx(sq.x) + sqrt_approx(sq.y));
      }
      const unsigned ballot = __ballot_sync(kFull, contrib);
      if (ballot != 0u) {
        float* a = s_acc[j];
        if (__popc(ballot) <= kDirectLanes) {
          if (contrib) {
#pragma unroll
            for (int k = 0; k < 10; ++k) atomicAdd(&a[k], v[k]);
            if (touched) a[10] = 1.f;
            a[11] = 1.f;
          }
        } else {
          const bool any_touched = __any_sync(kFull, touched);
          int idx;
          const float sum = warp_reduce10(v, lane, &idx);
          if (idx >= 0) atomicAdd(&a[idx], sum);
          if (lane == 1) {
            if (any_touched) a[10] = 1.f;
            a[11] = 1.f;
          }
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
  });
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

template <int NP, int B>
void backward_pairs_launch(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                           const float4* conic_op, const float4* color, const ViewDesc* views,
                           int n_views, int total_tiles, const float* T_final,
                           const int32_t* last, const float* dL_drgb, ScreenGrad* screen,
                           cudaStream_t stream, const uint8_t* block_bits,
                           const int* tile_order, int* ticket) {
  const int schedule = tile_order == nullptr ? kTileOrder : raster_config().backward_schedule;
  int grid = total_tiles;
  if (schedule == kPersistent) {
    grid = std::min(total_tiles, resident_ctas(k_backward_pairs<NP, B>, TileGeom<2 * NP>::kThreads));
    cudaMemsetAsync(ticket, 0, sizeof(int), stream);
  }
  k_backward_pairs<NP, B><<<grid, TileGeom<2 * NP>::kThreads, 0, stream>>>(
      ranges, pair_slots, xy, conic_op, color, views, n_views, T_final, last, dL_drgb, screen,
      block_bits, schedule, tile_order, ticket, total_tiles);
}

void launch_backward(const int2* ranges, const uint32_t* pair_slots, const float2* xy,
                     const float4* conic_op, const float4* color, const ViewDesc* views,
                     int n_views, int total_tiles, const float* T_final, const int32_t* last,
                     const float* dL_drgb, ScreenGrad* screen, cudaStream_t stream,
                     const uint8_t* block_bits, const int* tile_order, int* ticket) {
  if (total_tiles <= 0) return;
  count_launch();
  switch (raster_config().backward_px) {
    case 1:
      backward_px<1>(ranges, pair_slots, xy, conic_op, color, views, n_views, total_tiles,
                     T_final, last, dL_drgb, screen, stream);
      break;
    case 4:
      backward_pairs_launch<2, kBatch / 2>(ranges, pair_slots, xy, conic_op, color, views,
                                           n_views, total_tiles, T_final, last, dL_drgb,
                                           screen, stream, block_bits, tile_order, ticket);
      break;
    default: {
      const int b = raster_config().backward_batch;
#define PXS_BWD(B)                                                                         \
  backward_pairs_launch<1, B>(ranges, pair_slots, xy, conic_op, color, views, n_views,    \
                              total_tiles, T_final, last, dL_drgb, screen, stream, block_bits, \
                              tile_order, ticket)
      if (b == 64) PXS_BWD(64);
      else if (b == 128) PXS_BWD(128);
      else PXS_BWD(256);
#undef PXS_BWD
    }
  }
}

}  // namespace pxs
