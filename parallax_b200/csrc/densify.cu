// densify.cu -- adaptive density control as stream compaction, and finish().
//
// densifyAndPrune (SplatDensify.cpp:28-109) visits gaussians in index order:
// clone or split the ones whose mean screen gradient reaches the threshold,
// drop split parents and prunable originals, then append the additions in
// order until max_gaussians. Here that is: a classify kernel (one thread per
// gaussian), exclusive scans for the kept originals, the additions and the
// split ranks, an additions kernel that draws each split child's normals from
// the reference's xorshift32 stream jumped ahead to that parent's draws
// (xorshift is linear over GF(2), so 12*rank steps are a product of
// precomputed matrix powers), a scan over the non-prunable additions, and one
// compaction kernel that writes the new cloud and carries the Adam moments of
// kept gaussians (new ones start at zero, SplatTrainer.cpp:267-288).
//
// Compiled with -fmad=false. exp, log and cos are correctly rounded (computed
// in double); glibc's expf/logf/cosf differ from that in the last bit for a
// small fraction of inputs, which is the only way this can differ from the
// reference.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "densify.h"
#include "kernels.h"

namespace pxs {
namespace {

__device__ __forceinline__ float exp_cr(float x) { return __double2float_rn(exp((double)x)); }
__device__ __forceinline__ float log_cr(float x) { return __double2float_rn(log((double)x)); }
__device__ __forceinline__ float cos_cr(float x) { return __double2float_rn(cos((double)x)); }

__device__ __forceinline__ float largest_scale(const float* __restrict__ params, int64_t N,
                                               int64_t g) {
  float best = exp_cr(params[(int64_t)PXS_C_LOG_SCALE * N + g]);
  for (int a = 1; a < 3; ++a) {
    const float s = exp_cr(params[(int64_t)(PXS_C_LOG_SCALE + a) * N + g]);
    if (s > best) best = s;
  }
  return best;
}

__device__ __forceinline__ float opacity_of(float logit) {
  return 1.0f / (1.0f + exp_cr(-logit));
}

// Applies the linear map whose columns are cols[0..31] to x.
__device__ __forceinline__ uint32_t gf2_apply(const uint32_t* cols, uint32_t x) {
  uint32_t y = 0;
#pragma unroll 8
  for (int i = 0; i < 32; ++i)
    if ((x >> i) & 1u) y ^= cols[i];
  return y;
}

__device__ __forceinline__ uint32_t xorshift32(uint32_t& s) {
  uint32_t x = s;
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  s = x == 0u ? 1u : x;
  return s;
}

// nextNormal (SplatDensify.cpp:11-24).
__device__ __forceinline__ float next_normal(uint32_t& s) {
  float u1 = __uint2float_rn(xorshift32(s)) / 4294967296.f;
  u1 = u1 < 1e-7f ? 1e-7f : u1;  // std::max(1e-7f, u1)
  const float u2 = __uint2float_rn(xorshift32(s)) / 4294967296.f;
  return sqrtf(-2.f * log_cr(u1)) * cos_cr(2.f * 3.14159265358979f * u2);
}

}  // namespace

__global__ void k_densify_classify(const float* __restrict__ params, int N,
                                   const float* __restrict__ acc_gradient,
                                   const int32_t* __restrict__ acc_views, DensifyArgs a,
                                   int32_t* __restrict__ keep, int32_t* __restrict__ n_add,
                                   int32_t* __restrict__ is_split) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N) return;
  const int64_t n = N;
  int action = 0;  // 0 none, 1 clone, 2 split
  const float largest = largest_scale(params, n, g);
  if (a.has_room) {
    const int views = acc_views[g];
    if (views > 0) {
      const float mean_gradient = acc_gradient[g] / (float)views;
      if (!(mean_gradient < a.grad_threshold)) action = largest <= a.size_threshold ? 1 : 2;
    }
  }
  const bool prunable = opacity_of(params[(int64_t)PXS_C_OPACITY * n + g]) < a.prune_opacity ||
                        (a.prune_oversized && largest > a.max_scale);
  keep[g] = (action != 2 && !prunable) ? 1 : 0;
  n_add[g] = action == 1 ? 1 : (action == 2 ? 2 : 0);
  is_split[g] = action == 2 ? 1 : 0;
}

// Materialises every addition (clones copy the parent; split children are
// drawn from the parent's distribution) into `adds` (P x A, stride A) and
// flags the prunable ones.
__global__ void k_densify_additions(const float* __restrict__ params, int N, int P,
                                    const int32_t* __restrict__ n_add,
                                    const int64_t* __restrict__ add_offset,
                                    const int64_t* __restrict__ split_rank, DensifyArgs a,
                                    const uint32_t* __restrict__ jump_cols, int64_t A,
                                    float* __restrict__ adds, int32_t* __restrict__ prunable) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N) return;
  const int count = n_add[g];
  if (count == 0) return;
  const int64_t n = N;
  const int64_t base = add_offset[g];
  if (count == 1) {
    for (int c = 0; c < P; ++c) adds[(int64_t)c * A + base] = params[(int64_t)c * n + g];
    const float largest = largest_scale(params, n, g);
    prunable[base] = (opacity_of(params[(int64_t)PXS_C_OPACITY * n + g]) < a.prune_opacity ||
                      (a.prune_oversized && largest > a.max_scale))
                         ? 1
                         : 0;
    return;
  }
  // split: the state after 12 * rank draws of the densify stream
  uint32_t state = a.rng_state;
  uint64_t jump = 12ull * (uint64_t)split_rank[g];
  for (int k = 0; jump != 0 && k < kJumpPowers; ++k, jump >>= 1)
    if (jump & 1ull) state = gf2_apply(jump_cols + 32 * k, state);
  float s[3];
  for (int ax = 0; ax < 3; ++ax) s[ax] = exp_cr(params[(int64_t)(PXS_C_LOG_SCALE + ax) * n + g]);
  // rotation of the normalised quaternion (Quaternion::toRotationMatrix)
  float w = params[(int64_t)(PXS_C_ROTATION + 0) * n + g];
  float x = params[(int64_t)(PXS_C_ROTATION + 1) * n + g];
  float y = params[(int64_t)(PXS_C_ROTATION + 2) * n + g];
  float z = params[(int64_t)(PXS_C_ROTATION + 3) * n + g];
  const float sq = (x * x + z * z) + (y * y + w * w);
  if (sq > 0.f) {
    const float norm = sqrtf(sq);
    w = w / norm;
    x = x / norm;
    y = y / norm;
    z = z / norm;
  }
  const float tx = 2.f * x, ty = 2.f * y, tz = 2.f * z;
  const float twx = tx * w, twy = ty * w, twz = tz * w;
  const float txx = tx * x, txy = ty * x, txz = tz * x;
  const float tyy = ty * y, tyz = tz * y, tzz = tz * z;
  const float R[9] = {1.f - (tyy + tzz), txy - twz, txz + twy, txy + twz, 1.f - (txx + tzz),
                      tyz - twx, txz - twy, tyz + twx, 1.f - (txx + tyy)};
  const float opacity = opacity_of(params[(int64_t)PXS_C_OPACITY * n + g]);
  for (int child = 0; child < 2; ++child) {
    // Vec3f(n()*sx, n()*sy, n()*sz): the compiled reference draws the last
    // argument first
    const float nz = next_normal(state);
    const float ny = next_normal(state);
    const float nx = next_normal(state);
    const float sample[3] = {nx * s[0], ny * s[1], nz * s[2]};
    const int64_t dst = base + child;
    for (int c = 0; c < P; ++c) adds[(int64_t)c * A + dst] = params[(int64_t)c * n + g];
    for (int i = 0; i < 3; ++i) {
      const float p = params[(int64_t)(PXS_C_POSITION + i) * n + g];
      adds[(int64_t)(PXS_C_POSITION + i) * A + dst] =
          p + (R[i * 3 + 0] * sample[0] + (R[i * 3 + 1] * sample[1] + R[i * 3 + 2] * sample[2]));
    }
    float largest = 0.f;
    for (int ax = 0; ax < 3; ++ax) {
      const float ls = params[(int64_t)(PXS_C_LOG_SCALE + ax) * n + g] - a.log_split_divider;
      adds[(int64_t)(PXS_C_LOG_SCALE + ax) * A + dst] = ls;
      const float e = exp_cr(ls);
      largest = ax == 0 ? e : (e > largest ? e : largest);
    }
    prunable[dst] = (opacity < a.prune_opacity || (a.prune_oversized && largest > a.max_scale))
                        ? 1
                        : 0;
  }
}

__global__ void k_not(const int32_t* __restrict__ in, int64_t n, int32_t* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] ? 0 : 1;
}

// Writes the new cloud (stride N_new) and its Adam moments; `source` gets the
// old index or -1.
__global__ void k_densify_compact(const float* __restrict__ params, const float* __restrict__ m,
                                  const float* __restrict__ v, int N, int P,
                                  const int32_t* __restrict__ keep,
                                  const int64_t* __restrict__ keep_offset,
                                  const float* __restrict__ adds,
                                  const int32_t* __restrict__ prunable,
                                  const int64_t* __restrict__ np_rank, int64_t A, int64_t kept,
                                  int64_t n_new, float* __restrict__ out_params,
                                  float* __restrict__ out_m, float* __restrict__ out_v,
                                  int32_t* __restrict__ source) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) {
    if (keep[i]) {
      const int64_t dst = keep_offset[i];
      for (int c = 0; c < P; ++c) {
        const int64_t from = (int64_t)c * N + i, to = (int64_t)c * n_new + dst;
        out_params[to] = params[from];
        if (out_m != nullptr) {
          out_m[to] = m[from];
          out_v[to] = v[from];
        }
      }
      if (source != nullptr) source[dst] = (int32_t)i;
    }
  } else if (i - N < A) {
    const int64_t a = i - N;
    if (prunable[a]) return;
    const int64_t dst = kept + np_rank[a];
    if (dst >= n_new) return;
    for (int c = 0; c < P; ++c) {
      const int64_t to = (int64_t)c * n_new + dst;
      out_params[to] = adds[(int64_t)c * A + a];
      if (out_m != nullptr) {
        out_m[to] = 0.f;
        out_v[to] = 0.f;
      }
    }
    if (source != nullptr) source[dst] = -1;
  }
}

// Prunable additions the reference visits before it stops at max_gaussians
// (it counts those as pruned).
__global__ void k_count_pruned_additions(const int32_t* __restrict__ prunable,
                                         const int64_t* __restrict__ np_rank, int64_t A,
                                         int64_t room, unsigned long long* __restrict__ count) {
  const int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (a < A && prunable[a] && np_rank[a] < room) atomicAdd(count, 1ull);
}

// ---------------------------------------------------------------- finish

// GaussianCloud::prune (GaussianCloud.cpp:177-190): opacity below min_opacity,
// or a largest scale exp(max log sigma) that is non-finite or above max_scale.
__global__ void k_finish_keep(const float* __restrict__ params, int N, float min_opacity,
                              float max_scale, int32_t* __restrict__ keep) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N) return;
  const int64_t n = N;
  float ls = params[(int64_t)PXS_C_LOG_SCALE * n + g];
  for (int a = 1; a < 3; ++a) {
    const float x = params[(int64_t)(PXS_C_LOG_SCALE + a) * n + g];
    ls = ls < x ? x : ls;  // Eigen maxCoeff
  }
  const float largest = exp_cr(ls);
  const bool drop = opacity_of(params[(int64_t)PXS_C_OPACITY * n + g]) < min_opacity ||
                    !isfinite(largest) || largest > max_scale;
  keep[g] = drop ? 0 : 1;
}

// Sort key for descending opacity logit with a stable ascending radix sort.
__global__ void k_finish_keys(const float* __restrict__ params, int N,
                              const int32_t* __restrict__ keep,
                              const int64_t* __restrict__ keep_offset,
                              uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N || !keep[g]) return;
  float x = -params[(int64_t)PXS_C_OPACITY * N + g];
  if (x == 0.f) x = 0.f;  // -0 and +0 compare equal
  uint32_t b = __float_as_uint(x);
  b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  const int64_t dst = keep_offset[g];
  keys[dst] = b;
  vals[dst] = (uint32_t)g;
}

__global__ void k_gather_params(const float* __restrict__ params, int N, int P,
                                const uint32_t* __restrict__ order, int64_t n_new,
                                float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_new) return;
  const int64_t g = order[i];
  for (int c = 0; c < P; ++c) out[(int64_t)c * n_new + i] = params[(int64_t)c * N + g];
}

// --------------------------------------------------------------- host side

void xorshift_jump_tables(uint32_t* cols) {
  // column i of the one-step map is the step applied to bit i
  uint32_t base[32];
  for (int i = 0; i < 32; ++i) {
    uint32_t x = 1u << i;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    base[i] = x;
  }
  auto apply = [](const uint32_t* c, uint32_t x) {
    uint32_t y = 0;
    for (int i = 0; i < 32; ++i)
      if ((x >> i) & 1u) y ^= c[i];
    return y;
  };
  for (int i = 0; i < 32; ++i) cols[i] = base[i];
  for (int k = 1; k < kJumpPowers; ++k) {
    const uint32_t* prev = cols + 32 * (k - 1);
    for (int i = 0; i < 32; ++i) cols[32 * k + i] = apply(prev, prev[i]);
  }
}

uint32_t xorshift_jump_host(const uint32_t* cols, uint32_t state, uint64_t steps) {
  for (int k = 0; steps != 0 && k < kJumpPowers; ++k, steps >>= 1) {
    if (steps & 1ull) {
      uint32_t y = 0;
      for (int i = 0; i < 32; ++i)
        if ((state >> i) & 1u) y ^= cols[32 * k + i];
      state = y;
    }
  }
  return state;
}

DensifyResult densify_device(DensifyWork& w, const float* params, const float* m, const float* v,
                             int N, int S, const float* acc_gradient, const int32_t* acc_views,
                             const DensifyArgs& args_in, float* out_params, float* out_m,
                             float* out_v, int32_t* source, int64_t out_capacity,
                             cudaStream_t stream) {
  DensifyResult r;
  const int P = 14 + 3 * S;
  if (N == 0) return r;
  DensifyArgs args = args_in;
  const size_t n = static_cast<size_t>(N);
  int32_t* keep = w.keep.reserve(n);
  int32_t* n_add = w.n_add.reserve(n);
  int32_t* split = w.split.reserve(n);
  int64_t* keep_off = w.keep_offset.reserve(n);
  int64_t* add_off = w.add_offset.reserve(n);
  int64_t* split_rank = w.split_rank.reserve(n);
  int64_t* totals = w.totals.reserve(4);
  const size_t scratch = scan_scratch_bytes(static_cast<int64_t>(2 * n + 2));
  char* base = w.scan.reserve(scratch + 64);
  ScanScratch ss;
  scan_scratch_assign(ss, base, static_cast<int64_t>(2 * n + 2));
  if (w.jump_cols.get() == nullptr) {
    uint32_t cols[32 * kJumpPowers];
    xorshift_jump_tables(cols);
    w.jump_cols.reserve(32 * kJumpPowers);
    PXS_CUDA(cudaMemcpy(w.jump_cols.get(), cols, sizeof(cols), cudaMemcpyHostToDevice));
    std::memcpy(w.host_cols, cols, sizeof(cols));
  }
  const unsigned blocks = (N + 255) / 256;
  count_launch();
  k_densify_classify<<<blocks, 256, 0, stream>>>(params, N, acc_gradient, acc_views, args, keep,
                                                 n_add, split);
  exclusive_scan_i32_to_i64(keep, keep_off, N, totals + 0, ss, stream);
  exclusive_scan_i32_to_i64(n_add, add_off, N, totals + 1, ss, stream);
  exclusive_scan_i32_to_i64(split, split_rank, N, totals + 2, ss, stream);
  int64_t host_totals[3] = {0, 0, 0};
  PXS_CUDA(cudaMemcpyAsync(host_totals, totals, sizeof(host_totals), cudaMemcpyDeviceToHost,
                           stream));
  PXS_CUDA(cudaStreamSynchronize(stream));
  const int64_t kept = host_totals[0], A = host_totals[1], splits = host_totals[2];
  float* adds = w.adds.reserve(static_cast<size_t>(P) * static_cast<size_t>(std::max<int64_t>(A, 1)));
  int32_t* prunable = w.prunable.reserve(static_cast<size_t>(std::max<int64_t>(A, 1)));
  int32_t* not_prunable = w.not_prunable.reserve(static_cast<size_t>(std::max<int64_t>(A, 1)));
  int64_t* np_rank = w.np_rank.reserve(static_cast<size_t>(std::max<int64_t>(A, 1)));
  int64_t n_np = 0;
  if (A > 0) {
    count_launch();
    k_densify_additions<<<blocks, 256, 0, stream>>>(params, N, P, n_add, add_off, split_rank,
                                                    args, w.jump_cols.get(), A, adds, prunable);
    count_launch();
    k_not<<<(unsigned)((A + 255) / 256), 256, 0, stream>>>(prunable, A, not_prunable);
    exclusive_scan_i32_to_i64(not_prunable, np_rank, A, totals + 3, ss, stream);
    PXS_CUDA(cudaMemcpyAsync(&n_np, totals + 3, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
    PXS_CUDA(cudaStreamSynchronize(stream));
  }
  const int64_t room = std::max<int64_t>(0, static_cast<int64_t>(args.max_gaussians) - kept);
  const int64_t accepted = std::min(n_np, room);
  const int64_t n_new = kept + accepted;
  if (n_new > out_capacity) throw Error(PXS_ERR_CAPACITY, "densified cloud exceeds the output");
  // counts as the reference reports them
  r.cloned = static_cast<int>(A - 2 * splits);
  r.split = static_cast<int>(splits);
  unsigned long long* d_count = reinterpret_cast<unsigned long long*>(totals + 3);
  PXS_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), stream));
  if (A > 0) {
    count_launch();
    k_count_pruned_additions<<<(unsigned)((A + 255) / 256), 256, 0, stream>>>(prunable, np_rank,
                                                                            A, room, d_count);
  }
  const int64_t total_threads = static_cast<int64_t>(N) + A;
  count_launch();
  k_densify_compact<<<(unsigned)((total_threads + 255) / 256), 256, 0, stream>>>(
      params, m, v, N, P, keep, keep_off, adds, prunable, np_rank, A, kept, n_new, out_params,
      out_m, out_v, source);
  unsigned long long pruned_adds = 0;
  PXS_CUDA(cudaMemcpyAsync(&pruned_adds, d_count, sizeof(pruned_adds), cudaMemcpyDeviceToHost,
                           stream));
  PXS_CUDA(cudaStreamSynchronize(stream));
  PXS_CUDA(cudaGetLastError());
  // originals removed without being split, plus the prunable additions visited
  r.pruned = static_cast<int>(static_cast<int64_t>(N) - splits - kept) + static_cast<int>(pruned_adds);
  r.count = n_new;
  r.rng_state = xorshift_jump_host(w.host_cols, args.rng_state, 12ull * (uint64_t)splits);
  return r;
}

int64_t finish_device(DensifyWork& w, const float* params, int N, int S, float min_opacity,
                      float* out, cudaStream_t stream) {
  const int P = 14 + 3 * S;
  if (N == 0) return 0;
  const size_t n = static_cast<size_t>(N);
  int32_t* keep = w.keep.reserve(n);
  int64_t* keep_off = w.keep_offset.reserve(n);
  int64_t* totals = w.totals.reserve(4);
  const size_t scratch =
      std::max(scan_scratch_bytes(static_cast<int64_t>(n)),
               scan_scratch_bytes(static_cast<int64_t>(radix_hist_entries(N, 0, 9))));
  char* base = w.scan.reserve(scratch + 64);
  ScanScratch ss;
  scan_scratch_assign(ss, base, std::max<int64_t>(N, radix_hist_entries(N, 0, 9)));
  const unsigned blocks = (N + 255) / 256;
  count_launch();
  k_finish_keep<<<blocks, 256, 0, stream>>>(params, N, min_opacity, 1e3f, keep);
  exclusive_scan_i32_to_i64(keep, keep_off, N, totals, ss, stream);
  int64_t kept = 0;
  PXS_CUDA(cudaMemcpyAsync(&kept, totals, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
  PXS_CUDA(cudaStreamSynchronize(stream));
  if (kept == 0) return 0;
  uint32_t* keys = w.sort_a.reserve(n);
  uint32_t* vals = w.sort_b.reserve(n);
  uint32_t* keys_alt = w.sort_c.reserve(n);
  uint32_t* vals_alt = w.sort_d.reserve(n);
  const size_t hist_n = radix_hist_entries(kept, 0, 9);
  uint32_t* hist = w.hist.reserve(hist_n);
  uint32_t* hist_scanned = w.hist_scanned.reserve(hist_n);
  count_launch();
  k_finish_keys<<<blocks, 256, 0, stream>>>(params, N, keep, keep_off, keys, vals);
  radix_sort_pairs(keys, vals, keys_alt, vals_alt, kept, 0, 32, hist, hist_scanned, ss, stream);
  count_launch();
  k_gather_params<<<(unsigned)((kept + 255) / 256), 256, 0, stream>>>(params, N, P, vals, kept,
                                                                      out);
  PXS_CUDA(cudaGetLastError());
  return kept;
}

}  // namespace pxs
