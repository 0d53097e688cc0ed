// bin.cu -- per-tile key lists from the depth-sorted splats, by tile rows.
//
// The reference appends each splat, in depth order, to every 16-px tile its
// 3-sigma box touches (buildTiles, SplatRaster.cpp:104-151), so a tile's list
// is near to far. Sorting the (tile, splat) pairs themselves moves every pair
// through memory once per radix pass. Here the rectangle structure is used
// instead:
//   1. each visible splat (in depth order) emits one record per tile row it
//      covers -- (global row id, slot), about one seventh as many as pairs;
//   2. one stable radix pass groups the records by row, keeping depth order;
//   3. one CTA per row counts, per column, the records covering it (per warp,
//      over contiguous eighths of the row's records), which gives every tile's
//      length; an exclusive scan over the tiles gives the tile ranges;
//   4. the same CTA walks its records again, 32 at a time per warp: each lane
//      sets its bit in a per-column bitmap for every column its splat covers,
//      and the pair's place in the tile's list is the column's running base
//      plus the number of earlier lanes in the bitmap.
// The result -- ranges and slot lists -- is exactly the reference's, with
// equal depths in gaussian order (the depth sort is stable over slots).
#include "common.cuh"
#include "kernels.h"

namespace pxs {
namespace {

constexpr int kWarps = 8;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int view_of_row(const ViewDesc* __restrict__ views, int n_views,
                                           int row) {
  int v = 0;
  while (v + 1 < n_views && views[v + 1].row_offset <= row) ++v;
  return v;
}

}  // namespace

// Rows covered by the i-th nearest slot of each view (0 when culled).
__global__ void k_gather_row_counts(const uint32_t* __restrict__ sorted_slots,
                                    const int32_t* __restrict__ tile_count,
                                    const uint2* __restrict__ rect, int64_t n,
                                    int32_t* __restrict__ counts) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t slot = sorted_slots[i];
  int rows = 0;
  if (tile_count[slot] > 0) {
    const uint2 r = rect[slot];
    rows = (int)(r.y >> 16) - (int)(r.y & 0xFFFF) + 1;
  }
  counts[i] = rows;
}

// One record (global row id, slot) per covered row, in depth order. A warp
// emits the records of 32 consecutive slots together (coalesced writes; each
// lane finds the slot owning its output position by a binary search).
__global__ void __launch_bounds__(256)
    k_emit_rows(const uint32_t* __restrict__ sorted_slots, const int32_t* __restrict__ counts,
                const int64_t* __restrict__ offsets, const uint2* __restrict__ rect,
                const ViewDesc* __restrict__ views, int64_t slot_stride, int64_t n,
                uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, int64_t capacity,
                uint32_t sentinel_row, int32_t* __restrict__ overflow) {
  const int lane = lane_id();
  const int64_t first = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) - lane;
  if (first >= n) return;
  const int64_t i = first + lane;
  const bool valid = i < n;
  const int cnt = valid ? counts[i] : 0;
  const int64_t off = valid ? offsets[i] : (int64_t)-1;
  const int64_t warp_begin = __shfl_sync(kFull, off, 0);
  const int last_valid = min(31, (int)(n - 1 - first));
  const int64_t warp_end = __shfl_sync(kFull, off + cnt, last_valid);
  if (__any_sync(kFull, valid && cnt > 0 && off + cnt > capacity) && lane == 0)
    atomicExch(overflow, 1);
  uint32_t slot = 0, row0 = 0;
  if (valid && cnt > 0) {
    slot = sorted_slots[i];
    const uint2 r = rect[slot];
    row0 = (uint32_t)views[slot / slot_stride].row_offset + (r.y & 0xFFFF);
  }
  for (int64_t base = warp_begin; base < warp_end; base += 32) {
    const int64_t out = base + lane;
    int owner = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const int cand = owner + step;
      const int64_t cand_off = __shfl_sync(kFull, off, cand & 31);
      if (cand <= last_valid && cand_off <= out) owner = cand;
    }
    const int64_t o_off = __shfl_sync(kFull, off, owner);
    const int o_cnt = __shfl_sync(kFull, cnt, owner);
    const uint32_t o_slot = __shfl_sync(kFull, slot, owner);
    const uint32_t o_row0 = __shfl_sync(kFull, row0, owner);
    if (out >= warp_end || out >= capacity) continue;
    if (o_off + o_cnt > capacity) {  // does not fit: a sentinel past every row
      keys[out] = sentinel_row;
      vals[out] = 0u;
      continue;
    }
    keys[out] = o_row0 + (uint32_t)(out - o_off);
    vals[out] = o_slot;
  }
}

// Per row: how many of its records cover each column, per warp eighth
// (warp_base, exclusive over warps) and in total (the tile's length).
__global__ void __launch_bounds__(kWarps * 32)
    k_row_counts(const int2* __restrict__ row_ranges, const uint32_t* __restrict__ rec_slots,
                 const uint2* __restrict__ rect, const ViewDesc* __restrict__ views, int n_views,
                 int max_tiles_x, int32_t* __restrict__ warp_base,
                 int32_t* __restrict__ tile_counts) {
  extern __shared__ int32_t s_cnt[];  // [kWarps][max_tiles_x]
  const int row = blockIdx.x;
  const int v = view_of_row(views, n_views, row);
  const ViewDesc& vd = views[v];
  const int tiles_x = vd.tiles_x;
  const int local_row = row - vd.row_offset;
  const int2 range = row_ranges[row];
  for (int i = threadIdx.x; i < kWarps * tiles_x; i += blockDim.x)
    s_cnt[(i / tiles_x) * max_tiles_x + (i % tiles_x)] = 0;
  __syncthreads();
  const int w = warp_id(), lane = lane_id();
  const int len = max(0, range.y - range.x);
  const int per = (len + kWarps - 1) / kWarps;
  const int w_begin = range.x + w * per, w_end = min(range.y, w_begin + per);
  for (int rec = w_begin + lane; rec < w_end; rec += 32) {
    const uint2 r = rect[rec_slots[rec]];
    const int x0 = r.x & 0xFFFF, x1 = r.x >> 16;
    for (int c = x0; c <= x1; ++c) atomicAdd(&s_cnt[w * max_tiles_x + c], 1);
  }
  __syncthreads();
  const int64_t tile0 = (int64_t)vd.tile_offset + (int64_t)local_row * tiles_x;
  for (int c = threadIdx.x; c < tiles_x; c += blockDim.x) {
    int run = 0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) {
      const int t = s_cnt[k * max_tiles_x + c];
      warp_base[((int64_t)row * kWarps + k) * max_tiles_x + c] = run;
      run += t;
    }
    tile_counts[tile0 + c] = run;
  }
}

// ranges[t] = [offset, offset + count); a tile whose list would pass the pair
// capacity is left empty and raises the overflow flag.
__global__ void k_ranges_from_offsets(const int32_t* __restrict__ counts,
                                      const int64_t* __restrict__ offsets, int64_t n_tiles,
                                      int64_t capacity, int2* __restrict__ ranges,
                                      int32_t* __restrict__ overflow) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tiles) return;
  const int64_t begin = offsets[t], end = begin + counts[t];
  if (end > capacity) {
    ranges[t] = make_int2(0, 0);
    atomicExch(overflow, 1);
  } else {
    ranges[t] = make_int2((int)begin, (int)end);
  }
}

// Writes each row's records into its tiles' lists, in record (depth) order.
__global__ void __launch_bounds__(kWarps * 32)
    k_row_expand(const int2* __restrict__ row_ranges, const uint32_t* __restrict__ rec_slots,
                 const uint2* __restrict__ rect, const ViewDesc* __restrict__ views, int n_views,
                 int max_tiles_x, const int32_t* __restrict__ warp_base,
                 const int64_t* __restrict__ tile_offsets, int64_t capacity,
                 uint32_t* __restrict__ tile_slots) {
  extern __shared__ int32_t s_mem[];  // base [kWarps][max_tiles_x], then bitmap, same shape
  const int row = blockIdx.x;
  const int v = view_of_row(views, n_views, row);
  const ViewDesc& vd = views[v];
  const int tiles_x = vd.tiles_x;
  const int local_row = row - vd.row_offset;
  const int2 range = row_ranges[row];
  const int w = warp_id(), lane = lane_id();
  int32_t* base = s_mem + w * max_tiles_x;
  uint32_t* bitmap = reinterpret_cast<uint32_t*>(s_mem + kWarps * max_tiles_x) + w * max_tiles_x;
  const int64_t tile0 = (int64_t)vd.tile_offset + (int64_t)local_row * tiles_x;
  for (int c = lane; c < tiles_x; c += 32) {
    base[c] = (int32_t)tile_offsets[tile0 + c] +
              warp_base[((int64_t)row * kWarps + w) * max_tiles_x + c];
    bitmap[c] = 0u;
  }
  __syncwarp();
  const int len = max(0, range.y - range.x);
  const int per = (len + kWarps - 1) / kWarps;
  const int w_begin = range.x + w * per, w_end = min(range.y, w_begin + per);
  const unsigned lt = lanemask_lt();
  for (int step = w_begin; step < w_end; step += 32) {
    const int rec = step + lane;
    const bool valid = rec < w_end;
    int x0 = 1 << 30, x1 = -1;
    uint32_t slot = 0u;
    if (valid) {
      slot = rec_slots[rec];
      const uint2 r = rect[slot];
      x0 = r.x & 0xFFFF;
      x1 = r.x >> 16;
      for (int c = x0; c <= x1; ++c) atomicOr(&bitmap[c], 1u << lane);
    }
    __syncwarp();
    if (valid) {
      for (int c = x0; c <= x1; ++c) {
        const int64_t pos = (int64_t)base[c] + __popc(bitmap[c] & lt);
        if (pos < capacity) tile_slots[pos] = slot;
      }
    }
    __syncwarp();
    const int lo = __reduce_min_sync(kFull, x0), hi = __reduce_max_sync(kFull, x1);
    for (int c = lo + lane; c <= hi; c += 32) {
      const uint32_t m = bitmap[c];
      if (m != 0u) {
        base[c] += __popc(m);
        bitmap[c] = 0u;
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------ host

void launch_gather_row_counts(const uint32_t* sorted_slots, const int32_t* tile_count,
                              const uint2* rect, int64_t n, int32_t* counts,
                              cudaStream_t stream) {
  if (n <= 0) return;
  count_launch();
  k_gather_row_counts<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(sorted_slots, tile_count,
                                                                       rect, n, counts);
}

void launch_emit_rows(const uint32_t* sorted_slots, const int32_t* counts, const int64_t* offsets,
                      const uint2* rect, const ViewDesc* views, int64_t slot_stride, int64_t n,
                      uint32_t* keys, uint32_t* vals, int64_t capacity, uint32_t sentinel_row,
                      int32_t* overflow, cudaStream_t stream) {
  if (n <= 0) return;
  count_launch();
  k_emit_rows<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(
      sorted_slots, counts, offsets, rect, views, slot_stride, n, keys, vals, capacity,
      sentinel_row, overflow);
}

size_t row_counts_smem(int max_tiles_x) { return sizeof(int32_t) * kWarps * max_tiles_x; }
size_t row_expand_smem(int max_tiles_x) { return 2 * sizeof(int32_t) * kWarps * max_tiles_x; }

void configure_bin_kernels() {
  cudaFuncSetAttribute(k_row_counts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)row_counts_smem(kMaxTilesX));
  cudaFuncSetAttribute(k_row_expand, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)row_expand_smem(kMaxTilesX));
}

void launch_row_counts(const int2* row_ranges, const uint32_t* rec_slots, const uint2* rect,
                       const ViewDesc* views, int n_views, int total_rows, int max_tiles_x,
                       int32_t* warp_base, int32_t* tile_counts, cudaStream_t stream) {
  if (total_rows <= 0) return;
  count_launch();
  k_row_counts<<<total_rows, kWarps * 32, row_counts_smem(max_tiles_x), stream>>>(
      row_ranges, rec_slots, rect, views, n_views, max_tiles_x, warp_base, tile_counts);
}

void launch_ranges_from_offsets(const int32_t* counts, const int64_t* offsets, int64_t n_tiles,
                                int64_t capacity, int2* ranges, int32_t* overflow,
                                cudaStream_t stream) {
  if (n_tiles <= 0) return;
  count_launch();
  k_ranges_from_offsets<<<(unsigned)((n_tiles + 255) / 256), 256, 0, stream>>>(
      counts, offsets, n_tiles, capacity, ranges, overflow);
}

void launch_row_expand(const int2* row_ranges, const uint32_t* rec_slots, const uint2* rect,
                       const ViewDesc* views, int n_views, int total_rows, int max_tiles_x,
                       const int32_t* warp_base, const int64_t* tile_offsets, int64_t capacity,
                       uint32_t* tile_slots, cudaStream_t stream) {
  if (total_rows <= 0) return;
  count_launch();
  k_row_expand<<<total_rows, kWarps * 32, row_expand_smem(max_tiles_x), stream>>>(
      row_ranges, rec_slots, rect, views, n_views, max_tiles_x, warp_base, tile_offsets,
      capacity, tile_slots);
}

}  // namespace pxs
