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
//   3. each row is cut into chunks of 1024 records; one CTA per chunk counts,
//      per column, the records covering it; a per-row pass turns those into
//      each chunk's base within every tile of the row and the tiles' lengths;
//      an exclusive scan over the tiles gives the tile ranges;
//   4. one CTA per chunk walks its records again, 32 at a time per warp: each
//      lane sets its bit in a per-column bitmap for every column its splat
//      covers, and the pair's place among the chunk's pairs of that column is
//      the column's running base plus the number of earlier lanes in the
//      bitmap; the chunk's pairs are grouped by column in shared memory and
//      copied out to the lists with consecutive stores.
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

// Rows are cut into chunks of at most kChunk records so the work balances
// whatever the rows' lengths. chunks[c] = (row, begin, end); n_chunks[0] is
// the count. One CTA builds the table with a block-wide scan over the rows.
constexpr int kChunk = 1024;
constexpr int kStage = 8192;  // pairs a chunk can stage in shared memory
constexpr int kPerLane = kChunk / (kWarps * 32);  // records per lane per chunk

__global__ void __launch_bounds__(1024)
    k_row_chunks(const int2* __restrict__ row_ranges, int total_rows, int max_chunks,
                 int4* __restrict__ chunks, int32_t* __restrict__ n_chunks) {
  __shared__ int warp_sums[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < total_rows; base += blockDim.x) {
    const int row = base + threadIdx.x;
    int len = 0;
    int2 range = make_int2(0, 0);
    if (row < total_rows) {
      range = row_ranges[row];
      len = max(0, range.y - range.x);
    }
    const int count = (len + kChunk - 1) / kChunk;
    // block-wide inclusive scan of count
    int x = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int n = __shfl_up_sync(kFull, x, o);
      if (lane_id() >= o) x += n;
    }
    if (lane_id() == 31) warp_sums[warp_id()] = x;
    __syncthreads();
    if (warp_id() == 0) {
      int y = lane_id() < (int)(blockDim.x / 32) ? warp_sums[lane_id()] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int n = __shfl_up_sync(kFull, y, o);
        if (lane_id() >= o) y += n;
      }
      warp_sums[lane_id()] = y;
    }
    __syncthreads();
    const int first = carry + (warp_id() > 0 ? warp_sums[warp_id() - 1] : 0) + x - count;
    for (int j = 0; j < count; ++j) {
      const int c = first + j;
      if (c < max_chunks)
        chunks[c] = make_int4(row, range.x + j * kChunk, min(range.y, range.x + (j + 1) * kChunk), 0);
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = first + count;
    __syncthreads();
  }
  if (threadIdx.x == 0) n_chunks[0] = min(carry, max_chunks);
}

// Per-warp column counts of one chunk into s_cnt [kWarps][max_tiles_x]
// (zeroed by the caller): each record adds +1 at its first column and -1 past
// its last (two shared-memory atomics however wide it is), then each warp's
// row is prefix-summed over the columns. Lanes prefetch their records' rects.
__device__ __forceinline__ void chunk_column_counts(const int4& ch, const uint32_t* __restrict__ rec_slots,
                                                    const uint2* __restrict__ rect, int max_tiles_x,
                                                    int tiles_x, int32_t* s_cnt,
                                                    uint32_t (&slot)[kPerLane],
                                                    uint32_t (&xr)[kPerLane]) {
  const int w = warp_id(), lane = lane_id();
  const int w_begin = ch.y + w * (kChunk / kWarps);
#pragma unroll
  for (int k = 0; k < kPerLane; ++k) {
    const int rec = w_begin + k * 32 + lane;
    slot[k] = 0u;
    xr[k] = 1u;  // x0 = 1 > x1 = 0: covers nothing
    if (rec < ch.z) {
      slot[k] = rec_slots[rec];
      xr[k] = rect[slot[k]].x;
    }
  }
  int32_t* row = s_cnt + w * max_tiles_x;
#pragma unroll
  for (int k = 0; k < kPerLane; ++k) {
    const int x0 = xr[k] & 0xFFFF, x1 = xr[k] >> 16;
    if (x1 >= x0) {
      atomicAdd(&row[x0], 1);
      if (x1 + 1 < tiles_x) atomicAdd(&row[x1 + 1], -1);
    }
  }
  __syncwarp();
  int carry = 0;
  for (int c0 = 0; c0 < tiles_x; c0 += 32) {
    const int c = c0 + lane;
    int v = c < tiles_x ? row[c] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int n = __shfl_up_sync(kFull, v, o);
      if (lane >= o) v += n;
    }
    if (c < tiles_x) row[c] = carry + v;
    carry += __shfl_sync(kFull, v, 31);
  }
  __syncwarp();
}

// Per chunk: how many of its records cover each column.
__global__ void __launch_bounds__(kWarps * 32)
    k_chunk_counts(const int4* __restrict__ chunks, const int32_t* __restrict__ n_chunks,
                   const uint32_t* __restrict__ rec_slots, const uint2* __restrict__ rect,
                   const ViewDesc* __restrict__ views, int n_views, int max_tiles_x,
                   int32_t* __restrict__ chunk_counts) {
  extern __shared__ int32_t s_cnt[];  // [kWarps][max_tiles_x]
  if ((int)blockIdx.x >= n_chunks[0]) return;
  const int4 ch = chunks[blockIdx.x];
  const ViewDesc& vd = views[view_of_row(views, n_views, ch.x)];
  const int tiles_x = vd.tiles_x;
  for (int i = threadIdx.x; i < kWarps * tiles_x; i += blockDim.x)
    s_cnt[(i / tiles_x) * max_tiles_x + (i % tiles_x)] = 0;
  __syncthreads();
  uint32_t slot[kPerLane], xr[kPerLane];
  chunk_column_counts(ch, rec_slots, rect, max_tiles_x, tiles_x, s_cnt, slot, xr);
  __syncthreads();
  for (int c = threadIdx.x; c < tiles_x; c += blockDim.x) {
    int total = 0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) total += s_cnt[k * max_tiles_x + c];
    chunk_counts[(int64_t)blockIdx.x * max_tiles_x + c] = total;
  }
}

// Per row: each chunk's base within each tile of the row (exclusive over the
// row's chunks, in order) and the tile's length. The row's chunks are
// consecutive in the table, found from the first one by a binary search.
__global__ void __launch_bounds__(256)
    k_row_tiles(const int4* __restrict__ chunks, const int32_t* __restrict__ n_chunks,
                const ViewDesc* __restrict__ views, int n_views, int max_tiles_x,
                const int32_t* __restrict__ chunk_counts, int32_t* __restrict__ chunk_base,
                int32_t* __restrict__ tile_counts) {
  const int row = blockIdx.x;
  const int v = view_of_row(views, n_views, row);
  const ViewDesc& vd = views[v];
  const int tiles_x = vd.tiles_x;
  const int nc = n_chunks[0];
  // first chunk with chunks[c].x >= row
  int lo = 0, hi = nc;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (chunks[mid].x < row) lo = mid + 1;
    else hi = mid;
  }
  const int64_t tile0 = (int64_t)vd.tile_offset + (int64_t)(row - vd.row_offset) * tiles_x;
  for (int c = threadIdx.x; c < tiles_x; c += blockDim.x) {
    int run = 0;
    for (int k = lo; k < nc && chunks[k].x == row; ++k) {
      const int t = chunk_counts[(int64_t)k * max_tiles_x + c];
      chunk_base[(int64_t)k * max_tiles_x + c] = run;
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

// Block-wide exclusive scan of v (one value per thread); returns the prefix
// and writes the total to *total.
__device__ __forceinline__ int block_exclusive_scan(int v, int* s_warp, int* total) {
  const int lane = lane_id(), w = warp_id();
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int n = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += n;
  }
  if (lane == 31) s_warp[w] = x;
  __syncthreads();
  if (w == 0) {
    int y = lane < kWarps ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < kWarps; o <<= 1) {
      const int n = __shfl_up_sync(kFull, y, o);
      if (lane >= o) y += n;
    }
    if (lane < kWarps) s_warp[lane] = y;
  }
  __syncthreads();
  const int before = (w > 0 ? s_warp[w - 1] : 0) + x - v;
  *total = s_warp[kWarps - 1];
  __syncthreads();
  return before;
}

// Writes each chunk's records into its row's tile lists, in record (depth)
// order: 32 records at a time per warp, a per-column bitmap giving each pair
// its place among the lanes. The chunk's pairs are staged in shared memory
// grouped by column, then copied out column by column, so each tile's run of
// the chunk is written with consecutive stores; a chunk with more pairs than
// the stage holds stores them straight into the lists instead.
__global__ void __launch_bounds__(kWarps * 32)
    k_chunk_expand(const int4* __restrict__ chunks, const int32_t* __restrict__ n_chunks,
                   const uint32_t* __restrict__ rec_slots, const uint2* __restrict__ rect,
                   const ViewDesc* __restrict__ views, int n_views, int max_tiles_x,
                   const int32_t* __restrict__ chunk_base,
                   const int64_t* __restrict__ tile_offsets, int64_t capacity,
                   uint32_t* __restrict__ tile_slots) {
  // [kWarps][max_tiles_x] counts then bases, the same shape of bitmaps,
  // per column: stage start, pair count and list position; then the stage
  extern __shared__ __align__(16) int32_t s_mem[];
  __shared__ int s_warp[kWarps];
  if ((int)blockIdx.x >= n_chunks[0]) return;
  const int4 ch = chunks[blockIdx.x];
  const ViewDesc& vd = views[view_of_row(views, n_views, ch.x)];
  const int tiles_x = vd.tiles_x;
  const int w = warp_id(), lane = lane_id();
  int32_t* s_cnt = s_mem;
  uint32_t* bitmap_all = reinterpret_cast<uint32_t*>(s_mem + kWarps * max_tiles_x);
  int32_t* col_start = s_mem + 2 * kWarps * max_tiles_x;
  int32_t* col_count = col_start + max_tiles_x;
  // at byte 72 * max_tiles_x of the 16-byte aligned block: 8-byte aligned
  int64_t* col_dst = reinterpret_cast<int64_t*>(col_count + max_tiles_x);
  uint32_t* stage = reinterpret_cast<uint32_t*>(col_dst + max_tiles_x);
  for (int i = threadIdx.x; i < kWarps * tiles_x; i += blockDim.x) {
    s_cnt[(i / tiles_x) * max_tiles_x + (i % tiles_x)] = 0;
    bitmap_all[(i / tiles_x) * max_tiles_x + (i % tiles_x)] = 0u;
  }
  __syncthreads();
  uint32_t slot[kPerLane], xr[kPerLane];
  chunk_column_counts(ch, rec_slots, rect, max_tiles_x, tiles_x, s_cnt, slot, xr);
  __syncthreads();
  // per-column totals, then their exclusive scan: each column's stage start
  const int per = (tiles_x + blockDim.x - 1) / blockDim.x;
  const int c_begin = min(tiles_x, (int)threadIdx.x * per);
  const int c_end = min(tiles_x, c_begin + per);
  int mine = 0;
  for (int c = c_begin; c < c_end; ++c) {
    int t = 0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) t += s_cnt[k * max_tiles_x + c];
    col_count[c] = t;
    mine += t;
  }
  int total = 0;
  int run_start = block_exclusive_scan(mine, s_warp, &total);
  const bool staged = total <= kStage;  // block-uniform
  const int64_t tile0 = (int64_t)vd.tile_offset + (int64_t)(ch.x - vd.row_offset) * tiles_x;
  for (int c = c_begin; c < c_end; ++c) {
    col_start[c] = run_start;
    col_dst[c] = tile_offsets[tile0 + c] + chunk_base[(int64_t)blockIdx.x * max_tiles_x + c];
    // per warp, where its pairs of this column begin among the chunk's pairs
    int run = run_start;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) {
      const int t = s_cnt[k * max_tiles_x + c];
      s_cnt[k * max_tiles_x + c] = run;
      run += t;
    }
    run_start += col_count[c];
  }
  __syncthreads();
  int32_t* base = s_cnt + w * max_tiles_x;
  uint32_t* bitmap = bitmap_all + w * max_tiles_x;
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int k = 0; k < kPerLane; ++k) {
    const int x0 = xr[k] & 0xFFFF, x1 = xr[k] >> 16;
    for (int c = x0; c <= x1; ++c) atomicOr(&bitmap[c], 1u << lane);
    __syncwarp();
    for (int c = x0; c <= x1; ++c) {
      const int pos = base[c] + __popc(bitmap[c] & lt);  // among the chunk's pairs
      if (staged) {
        stage[pos] = slot[k];
      } else {
        const int64_t dst = col_dst[c] + (pos - col_start[c]);
        if (dst < capacity) tile_slots[dst] = slot[k];
      }
    }
    __syncwarp();
    const int lo = __reduce_min_sync(kFull, x1 >= x0 ? x0 : (1 << 30));
    const int hi = __reduce_max_sync(kFull, x1 >= x0 ? x1 : -1);
    for (int c = lo + lane; c <= hi; c += 32) {
      const uint32_t m = bitmap[c];
      if (m != 0u) {
        base[c] += __popc(m);
        bitmap[c] = 0u;
      }
    }
    __syncwarp();
  }
  if (!staged) return;
  __syncthreads();
  // copy out: one warp per column, consecutive entries per lane
  for (int c = w; c < tiles_x; c += kWarps) {
    const int n = col_count[c], src = col_start[c];
    const int64_t dst = col_dst[c];  // >= 0: offsets and bases are counts
    for (int i = lane; i < n; i += 32)
      if (dst + i < capacity) tile_slots[dst + i] = stage[src + i];
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

size_t chunk_counts_smem(int max_tiles_x) { return sizeof(int32_t) * kWarps * max_tiles_x; }
size_t chunk_expand_smem(int max_tiles_x) {
  return sizeof(int32_t) * ((2 * kWarps + 2) * (size_t)max_tiles_x + kStage) +
         sizeof(int64_t) * (size_t)max_tiles_x;
}

void configure_bin_kernels() {
  cudaFuncSetAttribute(k_chunk_counts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)chunk_counts_smem(kMaxTilesX));
  cudaFuncSetAttribute(k_chunk_expand, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)chunk_expand_smem(kMaxTilesX));
}

int64_t max_row_chunks(int64_t records, int total_rows) { return records / kChunk + total_rows + 1; }

void launch_tile_lists(const int2* row_ranges, const uint32_t* rec_slots, const uint2* rect,
                       const ViewDesc* views, int n_views, int total_rows, int max_tiles_x,
                       int64_t max_chunks, int4* chunks, int32_t* n_chunks,
                       int32_t* chunk_counts, int32_t* chunk_base, int32_t* tile_counts,
                       cudaStream_t stream) {
  if (total_rows <= 0) return;
  count_launch();
  k_row_chunks<<<1, 1024, 0, stream>>>(row_ranges, total_rows, (int)max_chunks, chunks, n_chunks);
  count_launch();
  k_chunk_counts<<<(unsigned)max_chunks, kWarps * 32, chunk_counts_smem(max_tiles_x), stream>>>(
      chunks, n_chunks, rec_slots, rect, views, n_views, max_tiles_x, chunk_counts);
  count_launch();
  k_row_tiles<<<total_rows, 256, 0, stream>>>(chunks, n_chunks, views, n_views, max_tiles_x,
                                              chunk_counts, chunk_base, tile_counts);
}

void launch_ranges_from_offsets(const int32_t* counts, const int64_t* offsets, int64_t n_tiles,
                                int64_t capacity, int2* ranges, int32_t* overflow,
                                cudaStream_t stream) {
  if (n_tiles <= 0) return;
  count_launch();
  k_ranges_from_offsets<<<(unsigned)((n_tiles + 255) / 256), 256, 0, stream>>>(
      counts, offsets, n_tiles, capacity, ranges, overflow);
}

void launch_chunk_expand(const int4* chunks, const int32_t* n_chunks, const uint32_t* rec_slots,
                         const uint2* rect, const ViewDesc* views, int n_views, int max_tiles_x,
                         int64_t max_chunks, const int32_t* chunk_base,
                         const int64_t* tile_offsets, int64_t capacity, uint32_t* tile_slots,
                         cudaStream_t stream) {
  if (max_chunks <= 0) return;
  count_launch();
  k_chunk_expand<<<(unsigned)max_chunks, kWarps * 32, chunk_expand_smem(max_tiles_x), stream>>>(
      chunks, n_chunks, rec_slots, rect, views, n_views, max_tiles_x, chunk_base, tile_offsets,
      capacity, tile_slots);
}

}  // namespace pxs
