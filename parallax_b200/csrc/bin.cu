// bin.cu -- per-tile key lists from the depth-sorted splats, by tile rows.
//
// The reference appends each splat, in depth order, to every 16-px tile its
// 3-sigma box touches (buildTiles, SplatRaster.cpp:104-151), so a tile's list
// is near to far. Sorting the (tile, splat) pairs themselves moves every pair
// through memory once per radix pass. Here the rectangle structure is used
// instead:
//   1. each visible splat has one record per tile row it covers (about one
//      seventh as many as pairs), wanted grouped by row and near to far
//      within a row: each view's depth-sorted slots are cut into chunks of
//      1024; a CTA per chunk counts, per tile row, the splats covering it; an
//      exclusive scan of the counts in (row, chunk) order gives each chunk
//      its base in each row, and the chunk writes its records there (the
//      ranking of step 3 with rows for columns) -- a stable counting sort by
//      row with no sort pass;
//   2. each row is cut into chunks of 1024 records; one CTA per chunk counts,
//      per column, the records covering it; a per-row pass turns those into
//      each chunk's base within every tile of the row and the tiles' lengths;
//      an exclusive scan over the tiles gives the tile ranges;
//   3. one CTA per chunk walks its records again, 32 at a time per warp: each
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

// Rows are cut into chunks of at most kChunk records so the work balances
// whatever the rows' lengths. chunks[c] = (row, begin, end); n_chunks[0] is
// the count. One CTA builds the table with a block-wide scan over the rows.
constexpr int kChunk = 1024;
constexpr int kStage = 10240;  // pairs a chunk can stage in shared memory
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

// Per-warp counts of the lanes' ranges range[k] = lo | hi << 16 (empty when
// hi < lo) over the columns of `row` (zeroed by the caller, `extent` wide):
// each range adds +1 at lo and -1 past hi (two shared-memory atomics however
// wide it is), then the warp prefix-sums its row.
template <int K>
__device__ __forceinline__ void warp_range_counts(const uint32_t (&range)[K], int extent,
                                                  int32_t* row) {
  const int lane = lane_id();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int lo = range[k] & 0xFFFF, hi = range[k] >> 16;
    if (hi >= lo) {
      atomicAdd(&row[lo], 1);
      if (hi + 1 < extent) atomicAdd(&row[hi + 1], -1);
    }
  }
  __syncwarp();
  int carry = 0;
  for (int c0 = 0; c0 < extent; c0 += 32) {
    const int c = c0 + lane;
    int v = c < extent ? row[c] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int n = __shfl_up_sync(kFull, v, o);
      if (lane >= o) v += n;
    }
    if (c < extent) row[c] = carry + v;
    carry += __shfl_sync(kFull, v, 31);
  }
  __syncwarp();
}

// Per-warp column counts of one chunk of row records into s_cnt
// [kWarps][max_tiles_x] (zeroed by the caller). Each record's column range
// was stored beside it when the records were written (rec_xr), so it is read
// with the record instead of gathered through the record's slot.
__device__ __forceinline__ void chunk_column_counts(const int4& ch, const uint32_t* __restrict__ rec_slots,
                                                    const uint32_t* __restrict__ rec_xr, int max_tiles_x,
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
      xr[k] = rec_xr[rec];
    }
  }
  warp_range_counts(xr, tiles_x, s_cnt + w * max_tiles_x);
}

// Per chunk: how many of its records cover each column.
__global__ void __launch_bounds__(kWarps * 32)
    k_chunk_counts(const int4* __restrict__ chunks, const int32_t* __restrict__ n_chunks,
                   const uint32_t* __restrict__ rec_slots, const uint32_t* __restrict__ rec_xr,
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
  chunk_column_counts(ch, rec_slots, rec_xr, max_tiles_x, tiles_x, s_cnt, slot, xr);
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

// The chunk's layout from the per-warp counts in s_cnt [kWarps][stride] over
// `extent` columns: per column its pair total (col_count), its start among
// the chunk's staged pairs (col_start) and the list position of its first
// pair (col_dst = dst_of(c)); the per-warp counts become per-warp bases in
// place. Returns whether the chunk's pairs fit a stage of `stage_cap`.
template <typename DstOf>
__device__ __forceinline__ bool chunk_layout(int32_t* s_cnt, int stride, int extent,
                                             int stage_cap, int* s_warp, int32_t* col_count,
                                             int32_t* col_start, int64_t* col_dst,
                                             DstOf dst_of) {
  const int per = (extent + blockDim.x - 1) / blockDim.x;
  const int c_begin = min(extent, (int)threadIdx.x * per);
  const int c_end = min(extent, c_begin + per);
  int mine = 0;
  for (int c = c_begin; c < c_end; ++c) {
    int t = 0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) t += s_cnt[k * stride + c];
    col_count[c] = t;
    mine += t;
  }
  int total = 0;
  int run_start = block_exclusive_scan(mine, s_warp, &total);
  for (int c = c_begin; c < c_end; ++c) {
    col_start[c] = run_start;
    col_dst[c] = dst_of(c);
    // per warp, where its pairs of this column begin among the chunk's pairs
    int run = run_start;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) {
      const int t = s_cnt[k * stride + c];
      s_cnt[k * stride + c] = run;
      run += t;
    }
    run_start += col_count[c];
  }
  __syncthreads();
  return total <= stage_cap;  // block-uniform
}

// Each warp places its lanes' payloads, 32 at a time, on every column of their
// ranges: a lane sets its bit in the warp's per-column bitmap, and its place
// among the chunk's pairs of the column is the warp's running base there plus
// the number of earlier lanes in the bitmap. Staged pairs go to `stage`,
// grouped by column; otherwise straight to out[col_dst + rank] below capacity.
template <int K>
__device__ __forceinline__ void warp_range_expand(const uint32_t (&range)[K],
                                                  const uint32_t (&payload)[K], int32_t* base,
                                                  uint32_t* bitmap, bool staged,
                                                  uint32_t* stage, const int32_t* col_start,
                                                  const int64_t* col_dst, int64_t capacity,
                                                  uint32_t* __restrict__ out,
                                                  const uint32_t (*extra)[K] = nullptr,
                                                  uint32_t* __restrict__ out_extra = nullptr) {
  const int lane = lane_id();
  const unsigned lt = lanemask_lt();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int lo = range[k] & 0xFFFF, hi = range[k] >> 16;
    for (int c = lo; c <= hi; ++c) atomicOr(&bitmap[c], 1u << lane);
    __syncwarp();
    for (int c = lo; c <= hi; ++c) {
      const int pos = base[c] + __popc(bitmap[c] & lt);  // among the chunk's pairs
      if (staged) {
        stage[pos] = payload[k];
      } else {
        const int64_t dst = col_dst[c] + (pos - col_start[c]);
        if (dst < capacity) {
          out[dst] = payload[k];
          if (out_extra != nullptr) out_extra[dst] = (*extra)[k];
        }
      }
    }
    __syncwarp();
    const int wlo = __reduce_min_sync(kFull, hi >= lo ? lo : (1 << 30));
    const int whi = __reduce_max_sync(kFull, hi >= lo ? hi : -1);
    for (int c = wlo + lane; c <= whi; c += 32) {
      const uint32_t m = bitmap[c];
      if (m != 0u) {
        base[c] += __popc(m);
        bitmap[c] = 0u;
      }
    }
    __syncwarp();
  }
}

// The staged pairs out to their lists: one warp per column, consecutive
// entries per lane.
// With `rect` and `out_x` the records also get their slot's column range.
__device__ __forceinline__ void copy_out_staged(int extent, const int32_t* col_count,
                                                const int32_t* col_start,
                                                const int64_t* col_dst, const uint32_t* stage,
                                                int64_t capacity, uint32_t* __restrict__ out,
                                                const uint2* __restrict__ rect = nullptr,
                                                uint32_t* __restrict__ out_x = nullptr) {
  const int w = warp_id(), lane = lane_id();
  for (int c = w; c < extent; c += kWarps) {
    const int n = col_count[c], src = col_start[c];
    const int64_t dst = col_dst[c];  // >= 0: offsets and bases are counts
    for (int i = lane; i < n; i += 32)
      if (dst + i < capacity) {
        const uint32_t v = stage[src + i];
        out[dst + i] = v;
        if (out_x != nullptr) out_x[dst + i] = rect[v].x;
      }
  }
}

// Shared memory of an expansion over `extent` columns: [kWarps][extent]
// counts then bases, the same shape of bitmaps, per column stage start, pair
// count and list position, then the stage.
struct ExpandSmem {
  int32_t* cnt;
  uint32_t* bitmap;
  int32_t* col_start;
  int32_t* col_count;
  int64_t* col_dst;
  uint32_t* stage;
};

__device__ __forceinline__ ExpandSmem expand_smem(int32_t* s_mem, int max_extent) {
  ExpandSmem e;
  e.cnt = s_mem;
  e.bitmap = reinterpret_cast<uint32_t*>(s_mem + kWarps * max_extent);
  e.col_start = s_mem + 2 * kWarps * max_extent;
  e.col_count = e.col_start + max_extent;
  // at byte 72 * max_extent of the 16-byte aligned block: 8-byte aligned
  e.col_dst = reinterpret_cast<int64_t*>(e.col_count + max_extent);
  e.stage = reinterpret_cast<uint32_t*>(e.col_dst + max_extent);
  return e;
}

// Writes each chunk's records into its row's tile lists, in record (depth)
// order: 32 records at a time per warp, a per-column bitmap giving each pair
// its place among the lanes. The chunk's pairs are staged in shared memory
// grouped by column, then copied out column by column, so each tile's run of
// the chunk is written with consecutive stores; a chunk with more pairs than
// the stage holds stores them straight into the lists instead.
__global__ void __launch_bounds__(kWarps * 32)
    k_chunk_expand(const int4* __restrict__ chunks, const int32_t* __restrict__ n_chunks,
                   const uint32_t* __restrict__ rec_slots, const uint32_t* __restrict__ rec_xr,
                   const ViewDesc* __restrict__ views, int n_views, int max_tiles_x,
                   const int32_t* __restrict__ chunk_base,
                   const int64_t* __restrict__ tile_offsets, int64_t capacity,
                   uint32_t* __restrict__ tile_slots) {
  extern __shared__ __align__(16) int32_t s_mem[];
  __shared__ int s_warp[kWarps];
  if ((int)blockIdx.x >= n_chunks[0]) return;
  const int4 ch = chunks[blockIdx.x];
  const ViewDesc& vd = views[view_of_row(views, n_views, ch.x)];
  const int tiles_x = vd.tiles_x;
  const int w = warp_id();
  const ExpandSmem e = expand_smem(s_mem, max_tiles_x);
  for (int i = threadIdx.x; i < kWarps * tiles_x; i += blockDim.x) {
    e.cnt[(i / tiles_x) * max_tiles_x + (i % tiles_x)] = 0;
    e.bitmap[(i / tiles_x) * max_tiles_x + (i % tiles_x)] = 0u;
  }
  __syncthreads();
  uint32_t slot[kPerLane], xr[kPerLane];
  chunk_column_counts(ch, rec_slots, rec_xr, max_tiles_x, tiles_x, e.cnt, slot, xr);
  __syncthreads();
  const int64_t tile0 = (int64_t)vd.tile_offset + (int64_t)(ch.x - vd.row_offset) * tiles_x;
  const bool staged = chunk_layout(
      e.cnt, max_tiles_x, tiles_x, kStage, s_warp, e.col_count, e.col_start, e.col_dst,
      [&](int c) {
        return tile_offsets[tile0 + c] + chunk_base[(int64_t)blockIdx.x * max_tiles_x + c];
      });
  warp_range_expand(xr, slot, e.cnt + w * max_tiles_x, e.bitmap + w * max_tiles_x, staged,
                    e.stage, e.col_start, e.col_dst, capacity, tile_slots);
  if (!staged) return;
  __syncthreads();
  copy_out_staged(tiles_x, e.col_count, e.col_start, e.col_dst, e.stage, capacity, tile_slots);
}

// ------------------------------------------------------------ tile-row records
//
// The records -- one (tile row, slot) per row a visible splat covers -- are
// wanted grouped by row (rows of every view one after another) and, within a
// row, in depth order. Each view's depth-sorted slots are cut into chunks of
// kSlotChunk; a chunk counts, per tile row of its view, the splats covering
// it; an exclusive scan of those counts in (row, chunk) order gives every
// chunk its base in every row; the chunk then writes its records there with
// the same bitmap ranking and staging as the tile lists (rows for columns).
// This is the stable counting sort of the records by row, with no sort pass.
constexpr int kSlotChunk = 1024;
constexpr int kSlotPerLane = kSlotChunk / (kWarps * 32);  // slots per lane per chunk

// Lane slots of a chunk starting at `begin` of the depth-sorted slots, and
// their tile-row ranges and (with xr) tile-column ranges, empty for a culled
// slot. A culled slot is known by its sorted key (kCulledKey, read beside the
// slot), so the only gather by slot is its rectangle; a visible slot's
// rectangle is never empty (its footprint meets the image).
__device__ __forceinline__ void chunk_slot_rows(const uint32_t* __restrict__ sorted_slots,
                                                const uint32_t* __restrict__ sorted_keys,
                                                const uint2* __restrict__ rect, int64_t begin,
                                                uint32_t (&slot)[kSlotPerLane],
                                                uint32_t (&yr)[kSlotPerLane],
                                                uint32_t (*xr)[kSlotPerLane] = nullptr) {
  const int w = warp_id(), lane = lane_id();
  bool live[kSlotPerLane];
#pragma unroll
  for (int k = 0; k < kSlotPerLane; ++k) {
    const int64_t i = begin + w * (kSlotChunk / kWarps) + k * 32 + lane;
    slot[k] = sorted_slots[i];
    live[k] = sorted_keys[i] != kCulledKey;
    yr[k] = 1u;  // y0 = 1 > y1 = 0: no rows
    if (xr != nullptr) (*xr)[k] = 1u;
  }
#pragma unroll
  for (int k = 0; k < kSlotPerLane; ++k)
    if (live[k]) {
      const uint2 r = rect[slot[k]];
      yr[k] = r.y;
      if (xr != nullptr) (*xr)[k] = r.x;
    }
}

// counts[(row_offset + y) * cpv + c]: splats of chunk c of view v (block
// v * cpv + c) covering tile row y of the view.
__global__ void __launch_bounds__(kWarps * 32)
    k_slot_row_counts(const uint32_t* __restrict__ sorted_slots,
                      const uint32_t* __restrict__ sorted_keys, const uint2* __restrict__ rect,
                      const ViewDesc* __restrict__ views, int64_t slot_stride, int cpv,
                      int max_tiles_y, int32_t* __restrict__ counts) {
  extern __shared__ int32_t s_cnt[];  // [kWarps][max_tiles_y]
  const int v = blockIdx.x / cpv, c = blockIdx.x % cpv;
  const ViewDesc& vd = views[v];
  const int tiles_y = vd.tiles_y;
  for (int i = threadIdx.x; i < kWarps * tiles_y; i += blockDim.x)
    s_cnt[(i / tiles_y) * max_tiles_y + (i % tiles_y)] = 0;
  __syncthreads();
  uint32_t slot[kSlotPerLane], yr[kSlotPerLane];
  chunk_slot_rows(sorted_slots, sorted_keys, rect,
                  (int64_t)v * slot_stride + (int64_t)c * kSlotChunk, slot, yr);
  warp_range_counts(yr, tiles_y, s_cnt + warp_id() * max_tiles_y);
  __syncthreads();
  for (int y = threadIdx.x; y < tiles_y; y += blockDim.x) {
    int total = 0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) total += s_cnt[k * max_tiles_y + y];
    counts[(int64_t)(vd.row_offset + y) * cpv + c] = total;
  }
}

// The chunk's records at offsets[(row_offset + y) * cpv + c] onwards in each
// row y, in slot order; nothing at or past `capacity`.
__global__ void __launch_bounds__(kWarps * 32)
    k_slot_row_expand(const uint32_t* __restrict__ sorted_slots,
                      const uint32_t* __restrict__ sorted_keys, const uint2* __restrict__ rect,
                      const ViewDesc* __restrict__ views, int64_t slot_stride, int cpv,
                      int max_tiles_y, const int64_t* __restrict__ offsets, int64_t capacity,
                      uint32_t* __restrict__ rec_slots, uint32_t* __restrict__ rec_xr) {
  extern __shared__ __align__(16) int32_t s_mem[];
  __shared__ int s_warp[kWarps];
  const int v = blockIdx.x / cpv, c = blockIdx.x % cpv;
  const ViewDesc& vd = views[v];
  const int tiles_y = vd.tiles_y;
  const int w = warp_id();
  const ExpandSmem e = expand_smem(s_mem, max_tiles_y);
  for (int i = threadIdx.x; i < kWarps * tiles_y; i += blockDim.x) {
    e.cnt[(i / tiles_y) * max_tiles_y + (i % tiles_y)] = 0;
    e.bitmap[(i / tiles_y) * max_tiles_y + (i % tiles_y)] = 0u;
  }
  __syncthreads();
  uint32_t slot[kSlotPerLane], yr[kSlotPerLane];
  uint32_t xr[kSlotPerLane];  // the column ranges, written beside the records
  chunk_slot_rows(sorted_slots, sorted_keys, rect,
                  (int64_t)v * slot_stride + (int64_t)c * kSlotChunk, slot, yr, &xr);
  warp_range_counts(yr, tiles_y, e.cnt + w * max_tiles_y);
  __syncthreads();
  const bool staged = chunk_layout(
      e.cnt, max_tiles_y, tiles_y, kStage, s_warp, e.col_count, e.col_start, e.col_dst,
      [&](int y) { return offsets[(int64_t)(vd.row_offset + y) * cpv + c]; });
  warp_range_expand(yr, slot, e.cnt + w * max_tiles_y, e.bitmap + w * max_tiles_y, staged,
                    e.stage, e.col_start, e.col_dst, capacity, rec_slots, &xr, rec_xr);
  if (!staged) return;
  __syncthreads();
  copy_out_staged(tiles_y, e.col_count, e.col_start, e.col_dst, e.stage, capacity, rec_slots,
                  rect, rec_xr);
}

// row_ranges[r] = [offsets[r * cpv], offsets[(r + 1) * cpv]) (the total for the
// last row), clamped to the capacity; records past it raise the overflow flag.
__global__ void k_row_ranges_from_chunks(const int64_t* __restrict__ offsets, int total_rows,
                                         int cpv, const int64_t* __restrict__ total,
                                         int64_t capacity, int2* __restrict__ row_ranges,
                                         int32_t* __restrict__ overflow) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= total_rows) return;
  int64_t b = offsets[(int64_t)r * cpv];
  int64_t e = r + 1 < total_rows ? offsets[(int64_t)(r + 1) * cpv] : *total;
  if (e > capacity) atomicExch(overflow, 1);
  b = b < capacity ? b : capacity;
  e = e < capacity ? e : capacity;
  row_ranges[r] = make_int2((int)b, (int)e);
}

// ------------------------------------------------------------------ host

size_t chunk_counts_smem(int max_tiles_x) { return sizeof(int32_t) * kWarps * max_tiles_x; }
size_t chunk_expand_smem(int max_tiles_x) {
  return sizeof(int32_t) * ((2 * kWarps + 2) * (size_t)max_tiles_x + kStage) +
         sizeof(int64_t) * (size_t)max_tiles_x;
}

size_t slot_row_counts_smem(int max_tiles_y) { return sizeof(int32_t) * kWarps * max_tiles_y; }

void configure_bin_kernels() {
  cudaFuncSetAttribute(k_chunk_counts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)chunk_counts_smem(kMaxTilesX));
  cudaFuncSetAttribute(k_chunk_expand, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)chunk_expand_smem(kMaxTilesX));
  cudaFuncSetAttribute(k_slot_row_counts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)slot_row_counts_smem(kMaxTilesY));
  cudaFuncSetAttribute(k_slot_row_expand, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)chunk_expand_smem(kMaxTilesY));
}

int slot_chunks_per_view(int64_t slot_stride) { return (int)(slot_stride / kSlotChunk); }

void launch_slot_row_counts(const uint32_t* sorted_slots, const uint32_t* sorted_keys,
                            const uint2* rect, const ViewDesc* views, int n_views,
                            int64_t slot_stride, int max_tiles_y, int32_t* counts,
                            cudaStream_t stream) {
  const int cpv = slot_chunks_per_view(slot_stride);
  if (n_views <= 0 || cpv <= 0) return;
  count_launch();
  k_slot_row_counts<<<(unsigned)(n_views * cpv), kWarps * 32, slot_row_counts_smem(max_tiles_y),
                      stream>>>(sorted_slots, sorted_keys, rect, views, slot_stride, cpv,
                                max_tiles_y, counts);
}

void launch_slot_row_expand(const uint32_t* sorted_slots, const uint32_t* sorted_keys,
                            const uint2* rect, const ViewDesc* views, int n_views,
                            int64_t slot_stride, int max_tiles_y, const int64_t* offsets,
                            int64_t capacity, uint32_t* rec_slots, uint32_t* rec_xr,
                            cudaStream_t stream) {
  const int cpv = slot_chunks_per_view(slot_stride);
  if (n_views <= 0 || cpv <= 0) return;
  count_launch();
  k_slot_row_expand<<<(unsigned)(n_views * cpv), kWarps * 32, chunk_expand_smem(max_tiles_y),
                      stream>>>(sorted_slots, sorted_keys, rect, views, slot_stride, cpv,
                                max_tiles_y, offsets, capacity, rec_slots, rec_xr);
}

void launch_row_ranges_from_chunks(const int64_t* offsets, int total_rows, int cpv,
                                   const int64_t* total, int64_t capacity, int2* row_ranges,
                                   int32_t* overflow, cudaStream_t stream) {
  if (total_rows <= 0) return;
  count_launch();
  k_row_ranges_from_chunks<<<(unsigned)((total_rows + 255) / 256), 256, 0, stream>>>(
      offsets, total_rows, cpv, total, capacity, row_ranges, overflow);
}

int64_t max_row_chunks(int64_t records, int total_rows) { return records / kChunk + total_rows + 1; }

void launch_tile_lists(const int2* row_ranges, const uint32_t* rec_slots, const uint32_t* rec_xr,
                       const ViewDesc* views, int n_views, int total_rows, int max_tiles_x,
                       int64_t max_chunks, int4* chunks, int32_t* n_chunks,
                       int32_t* chunk_counts, int32_t* chunk_base, int32_t* tile_counts,
                       cudaStream_t stream) {
  if (total_rows <= 0) return;
  count_launch();
  k_row_chunks<<<1, 1024, 0, stream>>>(row_ranges, total_rows, (int)max_chunks, chunks, n_chunks);
  count_launch();
  k_chunk_counts<<<(unsigned)max_chunks, kWarps * 32, chunk_counts_smem(max_tiles_x), stream>>>(
      chunks, n_chunks, rec_slots, rec_xr, views, n_views, max_tiles_x, chunk_counts);
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
                         const uint32_t* rec_xr, const ViewDesc* views, int n_views, int max_tiles_x,
                         int64_t max_chunks, const int32_t* chunk_base,
                         const int64_t* tile_offsets, int64_t capacity, uint32_t* tile_slots,
                         cudaStream_t stream) {
  if (max_chunks <= 0) return;
  count_launch();
  k_chunk_expand<<<(unsigned)max_chunks, kWarps * 32, chunk_expand_smem(max_tiles_x), stream>>>(
      chunks, n_chunks, rec_slots, rec_xr, views, n_views, max_tiles_x, chunk_base, tile_offsets,
      capacity, tile_slots);
}

}  // namespace pxs
