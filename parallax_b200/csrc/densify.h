// densify.h -- device-side densify/prune and finish().
#pragma once

#include <cstdint>

#include "runtime.h"

namespace pxs {

// Powers M^(2^k) of the xorshift32 step kept for jumping ahead; 40 covers
// 12 draws for each of 2^31 split parents.
constexpr int kJumpPowers = 40;

struct DensifyArgs {
  float grad_threshold;     // densify_grad_threshold
  float size_threshold;     // percent_dense * extent
  float max_scale;          // prune_scale_fraction * extent
  float prune_opacity;
  float log_split_divider;  // logf(split_scale_divider), host libm
  int32_t prune_oversized;  // iteration > opacity_reset_interval
  int32_t has_room;         // count < max_gaussians
  int32_t max_gaussians;
  uint32_t rng_state;
};

struct DensifyResult {
  int64_t count = 0;
  int cloned = 0, split = 0, pruned = 0;
  uint32_t rng_state = 0;
};

struct DensifyWork {
  DeviceArray<int32_t> keep, n_add, split, prunable, not_prunable;
  DeviceArray<int64_t> keep_offset, add_offset, split_rank, np_rank, totals;
  DeviceArray<float> adds;
  DeviceArray<char> scan;
  DeviceArray<uint32_t> jump_cols, sort_a, sort_b, sort_c, sort_d, hist, hist_scanned;
  uint32_t host_cols[32 * kJumpPowers];
};

void xorshift_jump_tables(uint32_t* cols);
uint32_t xorshift_jump_host(const uint32_t* cols, uint32_t state, uint64_t steps);

// densifyAndPrune on device arrays (stride N in, stride result.count out).
// out_m/out_v/source may be null. Synchronises the stream (it needs the new
// count on the host).
DensifyResult densify_device(DensifyWork& w, const float* params, const float* m, const float* v,
                             int N, int S, const float* acc_gradient, const int32_t* acc_views,
                             const DensifyArgs& args, float* out_params, float* out_m,
                             float* out_v, int32_t* source, int64_t out_capacity,
                             cudaStream_t stream);

// SplatTrainer::finish: prune(min_opacity) then stable sort by descending
// opacity logit into `out` (stride = returned count).
int64_t finish_device(DensifyWork& w, const float* params, int N, int S, float min_opacity,
                      float* out, cudaStream_t stream);

}  // namespace pxs
