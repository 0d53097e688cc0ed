// loss.cu -- photometric loss L = (1-w) mean|r-t| + w (1 - mean SSIM) and its
// gradient, fused into one shared-memory tiled kernel.
//
// photometricLoss / meanSsim (SplatRaster.cpp:582-738) run 13 separable
// blurs per channel over whole-image planes. Here a CTA owns a 32x32 output
// tile and stages each channel of the rendered and target images over a
// 10-pixel halo (two stacked 11-tap blurs): it blurs the five statistic
// planes (x, y, xx, yy, xy) onto a 5-pixel halo, forms the SSIM map and its
// partials there (zero outside the image, as the reference's zero-padded
// adjoint requires), blurs them back onto the tile and writes dL/drgb. The
// reference blurs five partial planes back; by linearity of the blur the three
// without a pixel factor are summed first, so three planes are blurred (equal
// in exact arithmetic, within FP32 rounding otherwise). Each blur pass is
// register-blocked: a thread loads a strip once and slides the 11 taps along
// it. Sums run in the reference's tap order (fused multiply-adds allowed);
// the scalar totals are accumulated in double.
#include <cstdio>
#include <exception>
#include <mutex>

#include "common.cuh"
#include "kernels.h"
#include "runtime.h"

namespace pxs {
namespace {

constexpr int TW = 32, TH = 32;
constexpr int IW = TW + 20, IH = TH + 20;  // input region
constexpr int SW = TW + 10, SH = TH + 10;  // statistics region
constexpr int kThreads = 320;  // every blur pass below is one round of items

struct LossSmem {
  float in_r[IH][IW];      // rendered, the current channel
  float in_t[IH][IW];      // target
  float hb[5][IH][SW];     // horizontal blur of the five products / of the three partials
  float st[3][SH][SW];     // the three partial planes
};

}  // namespace

// mode 0: dL/drgb of photometricLoss; mode 1: d(mean SSIM)/drgb (meanSsim).
// With `flat`, the grid is one-dimensional over every view's own output tiles,
// view after view (views of different sizes waste no CTAs); otherwise the
// grid is (tiles across, tiles down, view) for the largest view.
__global__ void __launch_bounds__(kThreads, 2)
    k_loss(const float* __restrict__ rendered, const float* __restrict__ target,
           const ViewDesc* __restrict__ views, int n_views, LossParams lp,
           float* __restrict__ grad_out, double* __restrict__ sums, int flat) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LossSmem& sm = *reinterpret_cast<LossSmem*>(smem_raw);
  int v = blockIdx.z, ox = blockIdx.x * TW, oy = blockIdx.y * TH;
  if (flat) {
    // the last view whose first tile is at or before this CTA's
    const int t = blockIdx.x;
    int lo = 0, hi = n_views - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (views[mid].loss_tile_offset <= t) lo = mid;
      else hi = mid - 1;
    }
    v = lo;
    const int local = t - views[v].loss_tile_offset;
    const int across = (views[v].cam.width + TW - 1) / TW;
    if (across == 0) return;
    ox = (local % across) * TW;
    oy = (local / across) * TH;
  }
  const ViewDesc& vd = views[v];
  const int W = vd.cam.width, H = vd.cam.height;
  if (ox >= W || oy >= H) return;
  const int64_t pix0 = vd.pixel_offset;
  const float* rimg = rendered + pix0 * 3;
  const float* timg = target + vd.target_offset * 3;
  const int tid = threadIdx.x;


  const float w = lp.ssim_weight;
  // 1 / values and 1 / (pixels * 3) of photometricLoss and meanSsim: equal
  const float inv = 1.f / (float)((int64_t)W * H * 3);
  const float scale = inv;
  const float c1 = 0.01f * 0.01f, c2 = 0.03f * 0.03f;
  double l1_sum = 0.0, ssim_sum = 0.0;
  const bool want_ssim = lp.mode == 1 || w > 0.f;

  for (int c = 0; c < 3; ++c) {
    // stage channel c of both images over the input region, zero outside
    // (one channel at a time keeps three CTAs per SM; the other channels'
    // bytes of the same lines come back from L2)
    for (int q = tid; q < IH * IW; q += kThreads) {
      const int lx = q % IW, ly = q / IW;
      const int X = ox - 10 + lx, Y = oy - 10 + ly;
      float a = 0.f, b = 0.f;
      if (X >= 0 && X < W && Y >= 0 && Y < H) {
        const int64_t o = ((int64_t)Y * W + X) * 3 + c;
        a = rimg[o];
        b = timg[o];
      }
      sm.in_r[ly][lx] = a;
      sm.in_t[ly][lx] = b;
    }
    __syncthreads();
    if (want_ssim) {
      // horizontal blur of the five products over every input row, onto the
      // statistics columns; a thread slides the 11 taps over 7 outputs
      constexpr int HS = 7;
      for (int item = tid; item < IH * (SW / HS); item += kThreads) {
        const int r = item / (SW / HS), col0 = (item % (SW / HS)) * HS;
        float xs[HS + 10], ys[HS + 10], xx[HS + 10], yy[HS + 10], xy[HS + 10];
#pragma unroll
        for (int k = 0; k < HS + 10; ++k) {
          xs[k] = sm.in_r[r][col0 + k];
          ys[k] = sm.in_t[r][col0 + k];
          xx[k] = xs[k] * xs[k];
          yy[k] = ys[k] * ys[k];
          xy[k] = xs[k] * ys[k];
        }
#pragma unroll
        for (int o = 0; o < HS; ++o) {
          float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f, s4 = 0.f;
#pragma unroll
          for (int k = 0; k < 11; ++k) {
            const float kk = lp.kernel[k];
            s0 += kk * xs[o + k];
            s1 += kk * ys[o + k];
            s2 += kk * xx[o + k];
            s3 += kk * yy[o + k];
            s4 += kk * xy[o + k];
          }
          sm.hb[0][r][col0 + o] = s0;
          sm.hb[1][r][col0 + o] = s1;
          sm.hb[2][r][col0 + o] = s2;
          sm.hb[3][r][col0 + o] = s3;
          sm.hb[4][r][col0 + o] = s4;
        }
      }
      __syncthreads();
      // vertical blur -> statistics, then the SSIM map and its partials in
      // place; a thread takes one column and 7 consecutive rows
      constexpr int VS = 7;
      constexpr int VSEG = (SH + VS - 1) / VS;
      for (int item = tid; item < SW * VSEG; item += kThreads) {
        const int col = item % SW, r0 = (item / SW) * VS;
        float m[5][VS];
#pragma unroll
        for (int p = 0; p < 5; ++p) {
          float hv[VS + 10];
#pragma unroll
          for (int k = 0; k < VS + 10; ++k) hv[k] = (r0 + k < IH) ? sm.hb[p][r0 + k][col] : 0.f;
#pragma unroll
          for (int o = 0; o < VS; ++o) {
            float acc = 0.f;
#pragma unroll
            for (int k = 0; k < 11; ++k) acc += lp.kernel[k] * hv[o + k];
            m[p][o] = acc;
          }
        }
#pragma unroll
        for (int o = 0; o < VS; ++o) {
          const int r = r0 + o;
          if (r >= SH) break;
          const int X = ox - 5 + col, Y = oy - 5 + r;
          float t_mu = 0.f, t_var = 0.f, t_cov = 0.f, mu_x = m[0][o], mu_y = m[1][o];
          if (X >= 0 && X < W && Y >= 0 && Y < H) {
            const float var_x = m[2][o] - mu_x * mu_x;
            const float var_y = m[3][o] - mu_y * mu_y;
            const float cov = m[4][o] - mu_x * mu_y;
            const float a = 2.f * mu_x * mu_y + c1;
            const float b = 2.f * cov + c2;
            const float cc = mu_x * mu_x + mu_y * mu_y + c1;
            const float d = var_x + var_y + c2;
            // hardware reciprocal approximations (relative error ~1e-7, far
            // inside the 1e-5 loss tolerance; cc >= C1 and d >= C2 - rounding)
            const float rc = __fdividef(1.f, cc), rd = __fdividef(1.f, d);
            const float r_ccd = rc * rd;  // 1 / (cc d)
            const float ssim = (a * b) * r_ccd;
            if (col >= 5 && col < 5 + TW && r >= 5 && r < 5 + TH) ssim_sum += (double)ssim;
            t_mu = scale * (2.f * b * r_ccd) * (mu_y - mu_x * a * rc);
            t_var = -scale * ssim * rd;
            t_cov = scale * (2.f * a * r_ccd);
          } else {
            mu_x = 0.f;
            mu_y = 0.f;
          }
          // dL/dx = blur(t_mu) + 2x blur(t_var) - 2 blur(t_var mu_x)
          //        + y blur(t_cov) - blur(t_cov mu_y); the blur is linear, so
          // the three terms without a pixel factor are blurred as one plane
          sm.st[0][r][col] = t_mu - 2.f * t_var * mu_x - t_cov * mu_y;
          sm.st[1][r][col] = t_var;
          sm.st[2][r][col] = t_cov;
        }
      }
      __syncthreads();
      // horizontal blur of the partials onto the tile's columns, 16 per thread
      constexpr int HS2 = 16;
      for (int item = tid; item < 3 * SH * (TW / HS2); item += kThreads) {
        const int p = item / (SH * (TW / HS2));
        const int rem = item % (SH * (TW / HS2));
        const int r = rem / (TW / HS2), col0 = (rem % (TW / HS2)) * HS2;
        float tv[HS2 + 10];
#pragma unroll
        for (int k = 0; k < HS2 + 10; ++k) tv[k] = sm.st[p][r][col0 + k];
#pragma unroll
        for (int o = 0; o < HS2; ++o) {
          float acc = 0.f;
#pragma unroll
          for (int k = 0; k < 11; ++k) acc += lp.kernel[k] * tv[o + k];
          sm.hb[p][r][col0 + o] = acc;
        }
      }
      __syncthreads();
    }
    // vertical blur and the gradient, one column and 4 rows per thread
    constexpr int VS2 = 4;
    for (int item = tid; item < TW * (TH / VS2); item += kThreads) {
      const int col = item % TW, r0 = (item / TW) * VS2;
      float B[3][VS2];
      if (want_ssim) {
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          float hv[VS2 + 10];
#pragma unroll
          for (int k = 0; k < VS2 + 10; ++k) hv[k] = sm.hb[p][r0 + k][col];
#pragma unroll
          for (int o = 0; o < VS2; ++o) {
            float acc = 0.f;
#pragma unroll
            for (int k = 0; k < 11; ++k) acc += lp.kernel[k] * hv[o + k];
            B[p][o] = acc;
          }
        }
      }
#pragma unroll
      for (int o = 0; o < VS2; ++o) {
        const int r = r0 + o;
        const int X = ox + col, Y = oy + r;
        if (X >= W || Y >= H) continue;
        const float x = sm.in_r[r + 10][col + 10];
        const float y = sm.in_t[r + 10][col + 10];
        float d = 0.f;
        if (want_ssim) {
          d = B[0][o];
          d += 2.f * x * B[1][o];
          d += y * B[2][o];
        }
        const int64_t oidx = (pix0 + (int64_t)Y * W + X) * 3 + c;
        if (lp.mode == 1) {
          grad_out[oidx] = d;
        } else {
          const float diff = x - y;
          l1_sum += (double)fabsf(diff);
          const float sign = diff > 0.f ? 1.f : (diff < 0.f ? -1.f : 0.f);
          float g = (1.f - w) * sign * inv;
          if (w > 0.f) g -= w * d;
          if (grad_out != nullptr) grad_out[oidx] = g;
        }
      }
    }
    __syncthreads();
  }
  // block sums -> per-view totals
  __shared__ double red[2][kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    l1_sum += __shfl_xor_sync(0xffffffffu, l1_sum, o);
    ssim_sum += __shfl_xor_sync(0xffffffffu, ssim_sum, o);
  }
  if (lane_id() == 0) {
    red[0][warp_id()] = l1_sum;
    red[1][warp_id()] = ssim_sum;
  }
  __syncthreads();
  if (tid == 0) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < kThreads / 32; ++k) {
      a += red[0][k];
      b += red[1][k];
    }
    atomicAdd(&sums[2 * v + 0], a);
    atomicAdd(&sums[2 * v + 1], b);
  }
}

// loss = (1-w) * l1 + w * (1 - ssim) per view (SplatRaster.cpp:737); the
// batch loss is the mean over views. mode 1 reports mean SSIM instead.
__global__ void k_loss_finalize(const double* __restrict__ sums, const ViewDesc* views,
                                int n_views, float ssim_weight, int mode,
                                float* __restrict__ per_view, float* __restrict__ total) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float sum = 0.f;
  for (int v = 0; v < n_views; ++v) {
    const double values = 3.0 * (double)views[v].cam.width * (double)views[v].cam.height;
    float loss;
    const float ssim = (float)(sums[2 * v + 1] / values);
    if (mode == 1) {
      loss = ssim;
    } else {
      const float l1 = (float)(sums[2 * v + 0] / values);
      loss = ssim_weight <= 0.f ? l1 : (1.f - ssim_weight) * l1 + ssim_weight * (1.f - ssim);
    }
    if (per_view != nullptr) per_view[v] = loss;
    sum += loss;
  }
  if (total != nullptr) *total = n_views > 0 ? sum / (float)n_views : 0.f;
}

size_t loss_smem_bytes() { return sizeof(LossSmem); }

void configure_loss_kernel() {
  cudaFuncSetAttribute(k_loss, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(LossSmem));
}

int64_t loss_tiles(int width, int height) {
  return (int64_t)((width + TW - 1) / TW) * ((height + TH - 1) / TH);
}

void launch_loss(const float* rendered, const float* target, const ViewDesc* views, int n_views,
                 int max_width, int max_height, const LossParams& lp, float* grad_out,
                 double* sums, float* per_view, float* total, cudaStream_t stream,
                 int64_t flat_tiles) {
  if (n_views <= 0) return;
  cudaMemsetAsync(sums, 0, sizeof(double) * 2 * n_views, stream);
  count_launch();
  if (flat_tiles >= 0) {
    if (flat_tiles > 0)
      k_loss<<<(unsigned)flat_tiles, kThreads, sizeof(LossSmem), stream>>>(
          rendered, target, views, n_views, lp, grad_out, sums, 1);
  } else {
    dim3 grid((max_width + TW - 1) / TW, (max_height + TH - 1) / TH, n_views);
    k_loss<<<grid, kThreads, sizeof(LossSmem), stream>>>(rendered, target, views, n_views, lp,
                                                         grad_out, sums, 0);
  }
  count_launch();
  k_loss_finalize<<<1, 32, 0, stream>>>(sums, views, n_views, lp.ssim_weight, lp.mode,
                                        per_view, total);
}

}  // namespace pxs

// ------------------------------------------------ allocation-free entry point
//
// pxs_photometric_loss_static serves callers that cannot allocate device
// memory (a host framework whose caching allocator owns the GPU's memory, or
// a loop that must not pay cudaFree's device-wide synchronisation). The loss
// kernel's scratch -- the per-image descriptors it reads and the two double
// sums per image it accumulates into -- lives here, in one file-scope array
// that every GPU loading the library holds until the process exits. Its name
// in host code stands in for the symbol only; the device address comes from
// cudaGetSymbolAddress, looked up once per device on the first call there.
// Every call shares the array and finds the previous call's contents in it:
// the descriptors are rewritten and the sums cleared before each kernel runs,
// and calls that overlap on the GPU race.

namespace pxs {
namespace {

struct StaticLossScratch {
  ViewDesc views[PXS_STATIC_LOSS_MAX_VIEWS];
  double sums[2 * PXS_STATIC_LOSS_MAX_VIEWS];
};
static_assert(sizeof(StaticLossScratch) <= PXS_STATIC_LOSS_SCRATCH_BYTES,
              "the static loss scratch does not hold its views");

static __device__ __align__(256) unsigned char g_loss_scratch[PXS_STATIC_LOSS_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
StaticLossScratch* g_scratch_addr[kMaxDevices] = {};

// Image v of a batch of same-sized images laid out one after another.
__global__ void k_static_loss_views(StaticLossScratch* scratch, int width, int height,
                                    int n_views) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n_views) return;
  ViewDesc d;
  memset(&d, 0, sizeof(d));
  d.cam.width = width;
  d.cam.height = height;
  d.pixel_offset = (int64_t)v * width * height;
  d.target_offset = d.pixel_offset;
  scratch->views[v] = d;
}

struct StaticError {
  int status;
  const char* what;
};

// The scratch's device address on the current device; the first call on a
// device looks it up and raises the loss kernel's shared-memory limit.
StaticLossScratch* static_scratch(int device) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_addr[device] == nullptr) {
    void* ptr = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&ptr, g_loss_scratch);
    if (err != cudaSuccess) throw StaticError{PXS_ERR_CUDA, cudaGetErrorString(err)};
    err = cudaFuncSetAttribute(k_loss, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(LossSmem));
    if (err != cudaSuccess) throw StaticError{PXS_ERR_CUDA, cudaGetErrorString(err)};
    g_scratch_addr[device] = static_cast<StaticLossScratch*>(ptr);
  }
  return g_scratch_addr[device];
}

int static_fail(int status, const char* what, char* error, size_t error_len) {
  if (error != nullptr && error_len > 0) std::snprintf(error, error_len, "%s", what);
  return status;
}

}  // namespace
}  // namespace pxs

extern "C" int pxs_photometric_loss_static(const float* rendered, const float* target,
                                           int32_t width, int32_t height, int32_t n_views,
                                           float ssim_weight, float* dL_drgb,
                                           float* per_view_loss, float* loss, void* stream,
                                           char* error, size_t error_len) {
  using namespace pxs;
  char why[160];
  if (width < 0 || height < 0 || n_views < 0)
    return static_fail(PXS_ERR_INVALID, "negative image size or count", error, error_len);
  if (n_views > PXS_STATIC_LOSS_MAX_VIEWS) {
    std::snprintf(why, sizeof(why),
                  "n_views = %d exceeds the static scratch limit of %d images per call",
                  (int)n_views, PXS_STATIC_LOSS_MAX_VIEWS);
    return static_fail(PXS_ERR_INVALID, why, error, error_len);
  }
  const bool empty = n_views == 0 || width == 0 || height == 0;
  if (!empty && (rendered == nullptr || target == nullptr))
    return static_fail(PXS_ERR_INVALID, "image is null", error, error_len);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  try {
    if (empty) {  // nothing to score: every loss is 0
      if (loss != nullptr) {
        const cudaError_t err = cudaMemsetAsync(loss, 0, sizeof(float), s);
        if (err != cudaSuccess) throw StaticError{PXS_ERR_CUDA, cudaGetErrorString(err)};
      }
      if (per_view_loss != nullptr && n_views > 0) {
        const cudaError_t err = cudaMemsetAsync(per_view_loss, 0, sizeof(float) * n_views, s);
        if (err != cudaSuccess) throw StaticError{PXS_ERR_CUDA, cudaGetErrorString(err)};
      }
      return PXS_OK;
    }
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) throw StaticError{PXS_ERR_CUDA, cudaGetErrorString(err)};
    if (device < 0 || device >= kMaxDevices)
      throw StaticError{PXS_ERR_UNAVAILABLE, "device ordinal beyond the supported range"};
    StaticLossScratch* scratch = static_scratch(device);
    cudaGetLastError();  // an earlier, unrelated failure is not this call's
    count_launch();
    k_static_loss_views<<<(n_views + 63) / 64, 64, 0, s>>>(scratch, width, height, n_views);
    LossParams lp;
    ssim_kernel_weights(lp.kernel);
    lp.ssim_weight = ssim_weight;
    lp.mode = 0;
    // launch_loss clears scratch->sums on `s` before the kernel adds into them.
    launch_loss(rendered, target, scratch->views, n_views, width, height, lp, dL_drgb,
                scratch->sums, per_view_loss, loss, s);
    err = cudaGetLastError();
    if (err != cudaSuccess) throw StaticError{PXS_ERR_CUDA, cudaGetErrorString(err)};
    return PXS_OK;
  } catch (const StaticError& e) {
    return static_fail(e.status, e.what, error, error_len);
  } catch (const std::exception& e) {
    return static_fail(PXS_ERR_CUDA, e.what(), error, error_len);
  }
}
