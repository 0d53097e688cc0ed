// sort.cu -- scans, radix sort and key ranges for the binning path.
//
// Device-wide exclusive scans, a stable segmented LSD radix sort of 32-bit
// keys with 32-bit values, and the range kernel. The binning path uses them
// for the depth sort of every (view, gaussian) slot (segmented per view; ties
// keep gaussian order) and for grouping the tile-row records by row (bin.cu).
#include "common.cuh"
#include "kernels.h"

namespace pxs {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kMaxBins = 512;
constexpr int kSortWarps = kSortThreads / 32;

template <typename T>
__device__ T block_exclusive_scan(T v, T* total, T* smem_warp) {
  // warp inclusive scan
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T n = __shfl_up_sync(0xffffffffu, x, o);
    if (lane_id() >= o) x += n;
  }
  if (lane_id() == 31) smem_warp[warp_id()] = x;
  __syncthreads();
  if (warp_id() == 0) {
    T w = lane_id() < (int)(blockDim.x / 32) ? smem_warp[lane_id()] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T n = __shfl_up_sync(0xffffffffu, w, o);
      if (lane_id() >= o) w += n;
    }
    smem_warp[lane_id()] = w;  // inclusive warp totals
  }
  __syncthreads();
  const T warp_prefix = warp_id() > 0 ? smem_warp[warp_id() - 1] : T(0);
  *total = smem_warp[blockDim.x / 32 - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

template <typename Tin, typename T>
__global__ void __launch_bounds__(kScanThreads)
    k_scan_reduce(const Tin* __restrict__ in, int64_t n, T* __restrict__ block_sums) {
  __shared__ T warp_sums[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  T sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
    if (i < n) sum += (T)in[i];
  }
  T total;
  block_exclusive_scan<T>(sum, &total, warp_sums);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// Exclusive scan of one tile per block, seeded with block_offsets[block] (or 0).
template <typename Tin, typename T>
__global__ void __launch_bounds__(kScanThreads)
    k_scan_tile(const Tin* __restrict__ in, int64_t n, T* __restrict__ out,
                const T* __restrict__ block_offsets, T* __restrict__ total_out) {
  __shared__ T warp_sums[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  // blocked arrangement: thread owns kScanItems consecutive items
  T vals[kScanItems];
  T sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    vals[k] = i < n ? (T)in[i] : T(0);
    sum += vals[k];
  }
  T total;
  T prefix = block_exclusive_scan<T>(sum, &total, warp_sums);
  if (block_offsets != nullptr) prefix += block_offsets[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    if (i < n) out[i] = prefix;
    prefix += vals[k];
  }
  if (total_out != nullptr && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1)
    *total_out = prefix;
}

// ------------------------------------------------------------ radix sort

struct RadixPass {
  int shift;
  int bits;
  int64_t n;                // items (an upper bound when n_device is set)
  const int64_t* n_device;  // optional device-side item count
  int64_t segment_len;      // items per segment (a multiple of kSortTile, or n)
  int blocks_per_segment;
  int segments;
};

__global__ void __launch_bounds__(kSortThreads)
    k_radix_upsweep(const uint32_t* __restrict__ keys, RadixPass p, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[kMaxBins];
  const int bins = 1 << p.bits;
  for (int d = threadIdx.x; d < bins; d += blockDim.x) h[d] = 0;
  __syncthreads();
  const int seg = blockIdx.x / p.blocks_per_segment;
  const int bis = blockIdx.x % p.blocks_per_segment;
  const int64_t n = p.n_device != nullptr ? min(*p.n_device, p.n) : p.n;
  const int64_t seg_begin = (int64_t)seg * p.segment_len;
  const int64_t seg_end = min(seg_begin + p.segment_len, n);
  const int64_t begin = seg_begin + (int64_t)bis * kSortTile;
  const uint32_t mask = (uint32_t)bins - 1u;
  uint32_t key[kSortItemsPerThread];
#pragma unroll
  for (int k = 0; k < kSortItemsPerThread; ++k) {
    const int64_t i = begin + (int64_t)k * kSortThreads + threadIdx.x;
    key[k] = i < seg_end ? keys[i] : 0xFFFFFFFFu;
  }
#pragma unroll
  for (int k = 0; k < kSortItemsPerThread; ++k) {
    const int64_t i = begin + (int64_t)k * kSortThreads + threadIdx.x;
    if (i < seg_end) atomicAdd(&h[(key[k] >> p.shift) & mask], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < bins; d += blockDim.x)
    hist[((int64_t)seg * bins + d) * p.blocks_per_segment + bis] = h[d];
}

// Stable scatter of one block tile. Items are warp-striped (warp w owns
// [w*512, (w+1)*512), item k of a lane at k*32 + lane) and ranked with
// __match_any_sync per digit, then offset by earlier warps. The tile is
// reordered by digit in shared memory and written out digit run by digit run,
// so consecutive threads write consecutive addresses.
__global__ void __launch_bounds__(kSortThreads)
    k_radix_downsweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                      uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                      RadixPass p, const uint32_t* __restrict__ offsets) {
  // per-warp digit counters; reused as the staging buffer once ranks are known
  __shared__ uint32_t counts[kSortWarps * kMaxBins];
  __shared__ uint32_t block_offset[kMaxBins];
  __shared__ uint32_t digit_start[kMaxBins];
  __shared__ uint32_t warp_sums[32];
  static_assert(kSortWarps * kMaxBins >= kSortTile, "staging buffer too small");
  static_assert(2 * kSortThreads >= kMaxBins, "two digits per thread");
  const int bins = 1 << p.bits;
  const uint32_t mask = (uint32_t)bins - 1u;
  const int seg = blockIdx.x / p.blocks_per_segment;
  const int bis = blockIdx.x % p.blocks_per_segment;
  const int64_t n = p.n_device != nullptr ? min(*p.n_device, p.n) : p.n;
  const int64_t seg_begin = (int64_t)seg * p.segment_len;
  const int64_t seg_end = min(seg_begin + p.segment_len, n);
  const int64_t begin = seg_begin + (int64_t)bis * kSortTile;
  const int64_t end = min(begin + kSortTile, seg_end);
  const int items = end > begin ? (int)(end - begin) : 0;
  for (int d = threadIdx.x; d < bins; d += blockDim.x) {
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) counts[w * kMaxBins + d] = 0;
    block_offset[d] = offsets[((int64_t)seg * bins + d) * p.blocks_per_segment + bis];
  }
  __syncthreads();
  const int warp = warp_id(), lane = lane_id();
  const unsigned lt = lanemask_lt();
  uint32_t key[kSortItemsPerThread], val[kSortItemsPerThread], rank[kSortItemsPerThread];
  int digit[kSortItemsPerThread];
#pragma unroll
  for (int k = 0; k < kSortItemsPerThread; ++k) {
    const int local = warp * (kSortItemsPerThread * 32) + k * 32 + lane;
    const bool valid = local < items;
    key[k] = valid ? keys_in[begin + local] : 0u;
    val[k] = valid ? vals_in[begin + local] : 0u;
    digit[k] = valid ? (int)((key[k] >> p.shift) & mask) : kMaxBins;  // sentinel groups invalid
  }
#pragma unroll
  for (int k = 0; k < kSortItemsPerThread; ++k) {
    const int d = digit[k];
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (d < kMaxBins) base = counts[warp * kMaxBins + d];
    __syncwarp();
    if (lane == leader && d < kMaxBins) counts[warp * kMaxBins + d] = base + __popc(peers);
    __syncwarp();
    rank[k] = base + __popc(peers & lt);
  }
  __syncthreads();
  // thread t owns digits 2t and 2t+1: exclusive prefix over warps in place,
  // then the block-local start of each digit by a scan in digit order
  uint32_t total_pair[2] = {0u, 0u};
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int d = 2 * (int)threadIdx.x + r;
    if (d < bins) {
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = counts[w * kMaxBins + d];
        counts[w * kMaxBins + d] = run;
        run += c;
      }
      total_pair[r] = run;
    }
  }
  uint32_t block_total;
  const uint32_t start = block_exclusive_scan<uint32_t>(total_pair[0] + total_pair[1],
                                                         &block_total, warp_sums);
  if (2 * (int)threadIdx.x < bins) digit_start[2 * threadIdx.x] = start;
  if (2 * (int)threadIdx.x + 1 < bins) digit_start[2 * threadIdx.x + 1] = start + total_pair[0];
  __syncthreads();
  uint32_t local_pos[kSortItemsPerThread];
#pragma unroll
  for (int k = 0; k < kSortItemsPerThread; ++k) {
    const int d = digit[k];
    local_pos[k] = d < kMaxBins ? digit_start[d] + counts[warp * kMaxBins + d] + rank[k] : 0u;
  }
  __syncthreads();  // counts is now free: stage the keys by digit
  uint32_t* stage = counts;
#pragma unroll
  for (int k = 0; k < kSortItemsPerThread; ++k)
    if (digit[k] < kMaxBins) stage[local_pos[k]] = key[k];
  __syncthreads();
  uint32_t global_pos[kSortItemsPerThread];
#pragma unroll
  for (int k = 0; k < kSortItemsPerThread; ++k) {
    const int i = k * kSortThreads + threadIdx.x;
    global_pos[k] = 0xFFFFFFFFu;
    if (i < items) {
      const uint32_t kk = stage[i];
      const int d = (int)((kk >> p.shift) & mask);
      global_pos[k] = block_offset[d] + ((uint32_t)i - digit_start[d]);
      keys_out[global_pos[k]] = kk;
    }
  }
  __syncthreads();  // stage the values the same way
#pragma unroll
  for (int k = 0; k < kSortItemsPerThread; ++k)
    if (digit[k] < kMaxBins) stage[local_pos[k]] = val[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kSortItemsPerThread; ++k) {
    const int i = k * kSortThreads + threadIdx.x;
    if (i < items) vals_out[global_pos[k]] = stage[i];
  }
}

__global__ void k_iota(uint32_t* __restrict__ out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (uint32_t)i;
}


}  // namespace

// --------------------------------------------------------------- host side

template <typename Tin, typename T>
static void scan_impl(const Tin* in, T* out, int64_t n, T* total, ScanScratch& scratch, int level,
                      cudaStream_t stream) {
  const int64_t blocks = (n + kScanTile - 1) / kScanTile;
  if (blocks <= 1) {
    count_launch();
    k_scan_tile<Tin, T><<<1, kScanThreads, 0, stream>>>(in, n, out, nullptr, total);
    return;
  }
  T* sums = reinterpret_cast<T*>(scratch.level[level]);
  T* sums_scanned = reinterpret_cast<T*>(scratch.level[level]) + blocks;
  count_launch();
  k_scan_reduce<Tin, T><<<(unsigned)blocks, kScanThreads, 0, stream>>>(in, n, sums);
  scan_impl<T, T>(sums, sums_scanned, blocks, total, scratch, level + 1, stream);
  count_launch();
  k_scan_tile<Tin, T><<<(unsigned)blocks, kScanThreads, 0, stream>>>(in, n, out, sums_scanned,
                                                                      nullptr);
}

size_t scan_scratch_bytes(int64_t n, int level) {
  const int64_t blocks = (n + kScanTile - 1) / kScanTile;
  if (blocks <= 1) return 0;
  return (size_t)blocks * 2 * sizeof(int64_t) + scan_scratch_bytes(blocks, level + 1);
}

void scan_scratch_assign(ScanScratch& s, char* base, int64_t n) {
  int level = 0;
  int64_t m = n;
  while (level < ScanScratch::kLevels) {
    const int64_t blocks = (m + kScanTile - 1) / kScanTile;
    if (blocks <= 1) break;
    s.level[level] = base;
    base += blocks * 2 * sizeof(int64_t);
    m = blocks;
    ++level;
  }
}

void exclusive_scan_i32_to_i64(const int32_t* in, int64_t* out, int64_t n, int64_t* total,
                               ScanScratch& scratch, cudaStream_t stream) {
  if (n <= 0) {
    cudaMemsetAsync(total, 0, sizeof(int64_t), stream);
    return;
  }
  scan_impl<int32_t, int64_t>(in, out, n, total, scratch, 0, stream);
}

void exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, ScanScratch& scratch,
                        cudaStream_t stream) {
  if (n <= 0) return;
  scan_impl<uint32_t, uint32_t>(in, out, n, nullptr, scratch, 0, stream);
}

size_t radix_hist_entries(int64_t n, int64_t segment_len, int max_bits) {
  const int64_t seg_len = segment_len > 0 ? segment_len : n;
  const int segments = (int)((n + seg_len - 1) / seg_len);
  const int bps = (int)((seg_len + kSortTile - 1) / kSortTile);
  return (size_t)segments * ((size_t)1 << max_bits) * (size_t)bps;
}

int radix_sort_pairs(uint32_t*& keys, uint32_t*& vals, uint32_t*& keys_alt,
                     uint32_t*& vals_alt, int64_t n, int64_t segment_len, int total_bits,
                     uint32_t* hist, uint32_t* hist_scanned, ScanScratch& scratch,
                     cudaStream_t stream, const int64_t* n_device) {
  if (n <= 0 || total_bits <= 0) return 0;
  const int64_t seg_len = segment_len > 0 ? segment_len : n;
  const int passes = (total_bits + 8) / 9 > 0 ? (total_bits + 8) / 9 : 1;
  RadixPass p;
  p.n = n;
  p.n_device = n_device;
  p.segment_len = seg_len;
  p.segments = (int)((n + seg_len - 1) / seg_len);
  p.blocks_per_segment = (int)((seg_len + kSortTile - 1) / kSortTile);
  const int blocks = p.segments * p.blocks_per_segment;
  int shift = 0;
  for (int pass = 0; pass < passes; ++pass) {
    const int remaining = total_bits - shift;
    const int bits = (remaining + (passes - pass) - 1) / (passes - pass);
    p.shift = shift;
    p.bits = bits;
    count_launch();
    k_radix_upsweep<<<blocks, kSortThreads, 0, stream>>>(keys, p, hist);
    const int64_t entries = (int64_t)p.segments * ((int64_t)1 << bits) * p.blocks_per_segment;
    exclusive_scan_u32(hist, hist_scanned, entries, scratch, stream);
    count_launch();
    k_radix_downsweep<<<blocks, kSortThreads, 0, stream>>>(keys, vals, keys_alt, vals_alt, p,
                                                           hist_scanned);
    std::swap(keys, keys_alt);
    std::swap(vals, vals_alt);
    shift += bits;
  }
  return passes;
}

void launch_iota(uint32_t* out, int64_t n, cudaStream_t stream) {
  if (n > 0) {
    count_launch();
    k_iota<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(out, n);
  }
}

}  // namespace pxs
