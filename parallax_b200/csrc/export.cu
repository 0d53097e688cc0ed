// export.cu -- the trained cloud packed into the reference's file formats on
// the device, so one device-to-host copy carries the file's body.
//
//   PLY    writeGaussianPly (GaussianCloud.cpp:259-306): per gaussian, x y z,
//          three zero normals, f_dc_0..2, f_rest_*, opacity, scale_0..2,
//          rot_0..3 (w first), float32 little-endian. One CTA transposes 64
//          gaussians through shared memory, so both the component-major reads
//          and the record writes are contiguous.
//   .splat writeSplat (:414-443): 32-byte records: position, linear sigma,
//          RGBA bytes (base colour, opacity), quaternion bytes (w first).
//   .spz   writeSpz (:493-550): the attribute planes after the 16-byte header
//          (24-bit fixed-point positions, scale, rotation x y z, alpha,
//          colour and SH bytes); the host adds the header and the gzip
//          wrapper.
//
// Compiled with -fmad=false: every quantisation rounds like the reference's
// (products and sums separately, roundf / lroundf half away from zero as
// std::round / std::lround). exp is correctly rounded here; where glibc's expf
// is not (about 0.06% of inputs) a linear sigma or an opacity byte can differ.
#include "common.cuh"
#include "kernels.h"

namespace pxs {
namespace {

constexpr int kPlyTile = 64;  // gaussians per CTA in the PLY transpose

__device__ __forceinline__ float exp_cr(float x) { return __double2float_rn(exp((double)x)); }

// max(0, min(255, round(x))) as a byte, with std::min / std::max's handling
// of the comparisons (a NaN becomes 255)
__device__ __forceinline__ uint8_t clamp_byte(float x) {
  const float r = roundf(x);
  const float hi = r < 255.f ? r : 255.f;  // std::min(255.f, r)
  return (uint8_t)(0.f < hi ? hi : 0.f);   // std::max(0.f, ...)
}

// quantizeUnit (GaussianCloud.cpp:28-30)
__device__ __forceinline__ uint8_t quantize_unit(float v) { return clamp_byte(v * 255.f); }

// gaussianOpacity (GaussianCloud.h:81-83)
__device__ __forceinline__ float opacity_of(float logit) { return 1.0f / (1.0f + exp_cr(-logit)); }

// Quaternion::normalized over (x, y, z, w) storage: each coefficient divided
// by the square root of the squared norm (left alone when it is zero).
__device__ __forceinline__ void normalized(const float* __restrict__ params, int64_t n, int g,
                                           float q[4]) {
  const float w = params[(int64_t)(PXS_C_ROTATION + 0) * n + g];
  const float x = params[(int64_t)(PXS_C_ROTATION + 1) * n + g];
  const float y = params[(int64_t)(PXS_C_ROTATION + 2) * n + g];
  const float z = params[(int64_t)(PXS_C_ROTATION + 3) * n + g];
  const float sq = (x * x + z * z) + (y * y + w * w);
  q[0] = w;
  q[1] = x;
  q[2] = y;
  q[3] = z;
  if (sq > 0.f) {
    const float norm = sqrtf(sq);
#pragma unroll
    for (int a = 0; a < 4; ++a) q[a] = q[a] / norm;
  }
}

}  // namespace

// PLY body: record field f of gaussian g comes from parameter component
// field_src[f] (or zero when it is -1).
__global__ void __launch_bounds__(256)
    k_pack_ply(const float* __restrict__ params, int n, const int* __restrict__ field_src,
               int fields, float* __restrict__ out) {
  extern __shared__ float tile[];  // [fields][kPlyTile + 1]
  const int g0 = blockIdx.x * kPlyTile;
  const int count = min(kPlyTile, n - g0);
  for (int i = threadIdx.x; i < fields * kPlyTile; i += blockDim.x) {
    const int f = i / kPlyTile, k = i % kPlyTile;
    const int src = field_src[f];
    tile[f * (kPlyTile + 1) + k] =
        (k < count && src >= 0) ? params[(int64_t)src * n + g0 + k] : 0.f;
  }
  __syncthreads();
  float* dst = out + (int64_t)g0 * fields;
  for (int i = threadIdx.x; i < count * fields; i += blockDim.x) {
    const int k = i / fields, f = i % fields;
    dst[i] = tile[f * (kPlyTile + 1) + k];
  }
}

// .splat records, one thread per gaussian.
__global__ void __launch_bounds__(256)
    k_pack_splat(const float* __restrict__ params, int n, uint8_t* __restrict__ out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  float rec[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    rec[a] = params[(int64_t)(PXS_C_POSITION + a) * n + g];
    rec[3 + a] = exp_cr(params[(int64_t)(PXS_C_LOG_SCALE + a) * n + g]);  // linear sigma
  }
  uint8_t bytes[8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {  // gaussianBaseColor (GaussianCloud.h:75-79)
    const float v = 0.5f + kShC0 * params[(int64_t)(PXS_C_DC + c) * n + g];
    const float lo = v < 1.f ? v : 1.f;  // std::min(1.f, v)
    bytes[c] = quantize_unit(0.f < lo ? lo : 0.f);
  }
  bytes[3] = quantize_unit(opacity_of(params[(int64_t)PXS_C_OPACITY * n + g]));
  float q[4];
  normalized(params, n, g, q);
#pragma unroll
  for (int a = 0; a < 4; ++a) bytes[4 + a] = clamp_byte(q[a] * 128.0f + 128.0f);
  uint8_t* dst = out + (int64_t)g * 32;
  float4* d4 = reinterpret_cast<float4*>(dst);
  d4[0] = make_float4(rec[0], rec[1], rec[2], rec[3]);
  uint32_t w0 = bytes[0] | (bytes[1] << 8) | (bytes[2] << 16) | ((uint32_t)bytes[3] << 24);
  uint32_t w1 = bytes[4] | (bytes[5] << 8) | (bytes[6] << 16) | ((uint32_t)bytes[7] << 24);
  d4[1] = make_float4(rec[4], rec[5], __uint_as_float(w0), __uint_as_float(w1));
}

// .spz attribute planes (everything after the header), one thread per gaussian.
__global__ void __launch_bounds__(256)
    k_pack_spz(const float* __restrict__ params, int n, int fractional_bits, int rest_stored,
               int rest_degree, uint8_t* __restrict__ out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const int64_t N = n;
  uint8_t* pos = out;
  uint8_t* scl = pos + 9 * N;
  uint8_t* rot = scl + 3 * N;
  uint8_t* alp = rot + 3 * N;
  uint8_t* col = alp + N;
  uint8_t* sh = col + 3 * N;
  const float scale = (float)(1 << fractional_bits);
#pragma unroll
  for (int a = 0; a < 3; ++a) {  // 24-bit signed fixed point, little-endian
    // std::lround into a long, kept to its low 32 bits as the int32 cast does,
    // then clamped into the 24-bit signed range
    const long long rounded = lroundf(params[(int64_t)(PXS_C_POSITION + a) * N + g] * scale);
    int32_t fixed = (int32_t)(uint32_t)(unsigned long long)rounded;
    fixed = fixed < -(1 << 23) ? -(1 << 23) : (fixed > (1 << 23) - 1 ? (1 << 23) - 1 : fixed);
    const uint32_t bits = (uint32_t)fixed & 0xFFFFFFu;
    pos[g * 9 + a * 3 + 0] = (uint8_t)(bits & 0xFF);
    pos[g * 9 + a * 3 + 1] = (uint8_t)((bits >> 8) & 0xFF);
    pos[g * 9 + a * 3 + 2] = (uint8_t)((bits >> 16) & 0xFF);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)  // log sigma: (x + 10) * 16 onto a byte
    scl[g * 3 + a] = clamp_byte((params[(int64_t)(PXS_C_LOG_SCALE + a) * N + g] + 10.0f) * 16.0f);
  float q[4];
  normalized(params, N, g, q);
  if (q[0] < 0.f) {  // the hemisphere with w >= 0; w is implied on read
#pragma unroll
    for (int a = 0; a < 4; ++a) q[a] = q[a] * -1.f;
  }
#pragma unroll
  for (int a = 1; a < 4; ++a) rot[g * 3 + a - 1] = clamp_byte(q[a] * 127.5f + 127.5f);
  alp[g] = quantize_unit(opacity_of(params[(int64_t)PXS_C_OPACITY * N + g]));
#pragma unroll
  for (int c = 0; c < 3; ++c)
    col[g * 3 + c] = quantize_unit(0.5f + kShC0 * params[(int64_t)(PXS_C_DC + c) * N + g]);
  // SH bytes with the colour channel fastest; the coefficient of (channel c,
  // band k) is stored element c * rest_degree + k of the gaussian's sh_rest
  const int stored = 3 * rest_stored;
  for (int k = 0; k < rest_degree; ++k) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int index = c * rest_degree + k;
      const float v = index < stored ? params[(int64_t)(PXS_C_SH_REST + index) * N + g] : 0.f;
      sh[(int64_t)g * 3 * rest_degree + k * 3 + c] = clamp_byte(v * 128.0f + 128.0f);
    }
  }
}

size_t ply_pack_smem(int fields) { return sizeof(float) * (size_t)fields * (kPlyTile + 1); }

void launch_pack_ply(const float* params, int n, const int* field_src, int fields, float* out,
                     cudaStream_t stream) {
  if (n <= 0) return;
  count_launch();
  k_pack_ply<<<(n + kPlyTile - 1) / kPlyTile, 256, ply_pack_smem(fields), stream>>>(
      params, n, field_src, fields, out);
}

void launch_pack_splat(const float* params, int n, uint8_t* out, cudaStream_t stream) {
  if (n <= 0) return;
  count_launch();
  k_pack_splat<<<(n + 255) / 256, 256, 0, stream>>>(params, n, out);
}

void launch_pack_spz(const float* params, int n, int fractional_bits, int rest_stored,
                     int rest_degree, uint8_t* out, cudaStream_t stream) {
  if (n <= 0) return;
  count_launch();
  k_pack_spz<<<(n + 255) / 256, 256, 0, stream>>>(params, n, fractional_bits, rest_stored,
                                                  rest_degree, out);
}

}  // namespace pxs

// ------------------------------------------------- initializeFromPointCloud
//
// GaussianCloud.cpp:199-257. The spacing estimate's O(samples^2) nearest-
// neighbour search runs on the device, one thread per sampled point, with the
// reference's arithmetic: float differences, the squared norm summed as
// x^2 + (y^2 + z^2) (Eigen's unrolled 3-term reduction), its float square root
// widened to double. The host sums the distances in order and takes the logs.
namespace pxs {

__global__ void __launch_bounds__(256)
    k_seed_nearest(const float* __restrict__ points, int n, int stride, int samples,
                   double* __restrict__ nearest) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= samples) return;
  const int64_t i = (int64_t)s * stride;
  const float xi = points[i * 3], yi = points[i * 3 + 1], zi = points[i * 3 + 2];
  double best = 1e30;
  for (int64_t j = 0; j < n; j += stride) {
    if (j == i) continue;
    const float dx = xi - points[j * 3], dy = yi - points[j * 3 + 1], dz = zi - points[j * 3 + 2];
    const double d = (double)sqrtf(dx * dx + (dy * dy + dz * dz));
    best = d < best ? d : best;  // std::min(best, d)
  }
  nearest[s] = best;
}

// One gaussian per point: position, isotropic log sigma, identity rotation,
// the opacity logit, the DC colour from the point's 8-bit colour (or zero),
// zero higher SH. Component-major with n gaussians per component.
__global__ void __launch_bounds__(256)
    k_seed_points(const float* __restrict__ points, const uint8_t* __restrict__ colors, int n,
                  int S, float log_sigma, float logit, float* __restrict__ params) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const int64_t N = n;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    params[(PXS_C_POSITION + a) * N + g] = points[(int64_t)g * 3 + a];
    params[(PXS_C_LOG_SCALE + a) * N + g] = log_sigma;
    params[(PXS_C_DC + a) * N + g] =
        colors != nullptr ? ((float)colors[(int64_t)g * 3 + a] / 255.0f - 0.5f) / kShC0 : 0.f;
  }
  params[(PXS_C_ROTATION + 0) * N + g] = 1.f;  // w
  params[(PXS_C_ROTATION + 1) * N + g] = 0.f;
  params[(PXS_C_ROTATION + 2) * N + g] = 0.f;
  params[(PXS_C_ROTATION + 3) * N + g] = 0.f;
  params[PXS_C_OPACITY * N + g] = logit;
  for (int k = 0; k < 3 * S; ++k) params[(PXS_C_SH_REST + k) * N + g] = 0.f;
}

void launch_seed_nearest(const float* points, int n, int stride, int samples, double* nearest,
                         cudaStream_t stream) {
  if (samples <= 0) return;
  count_launch();
  k_seed_nearest<<<(samples + 255) / 256, 256, 0, stream>>>(points, n, stride, samples, nearest);
}

void launch_seed_points(const float* points, const uint8_t* colors, int n, int S,
                        float log_sigma, float logit, float* params, cudaStream_t stream) {
  if (n <= 0) return;
  count_launch();
  k_seed_points<<<(n + 255) / 256, 256, 0, stream>>>(points, colors, n, S, log_sigma, logit,
                                                     params);
}

}  // namespace pxs
