// ingest.cu -- training images from 8-bit camera frames, on the device.
//
// Pipeline::Impl::runSplatTraining (Pipeline.cpp:1892-1917) downscales each
// frame with downscaleToWidth (ImageIo.cpp:300-337) and divides every byte by
// 255 into the float image the trainer fits. Here one thread per output pixel
// averages its box of source pixels with the same integer arithmetic (box
// edges from 64-bit products, the sum rounded by adding half the count) and
// writes the byte and / or the float; the 8-bit frame crosses PCIe instead of
// the four times larger float image.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace pxs {

__global__ void __launch_bounds__(256)
    k_downscale(const uint8_t* __restrict__ src, int width, int height, int out_width,
                int out_height, uint8_t* __restrict__ out_bytes, float* __restrict__ out_linear) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)out_width * out_height) return;
  const int x = (int)(i % out_width), y = (int)(i / out_width);
  const int y0 = (int)((int64_t)y * height / out_height);
  const int y1 = max(y0 + 1, (int)((int64_t)(y + 1) * height / out_height));
  const int x0 = (int)((int64_t)x * width / out_width);
  const int x1 = max(x0 + 1, (int)((int64_t)(x + 1) * width / out_width));
  int sums[3] = {0, 0, 0};
  int taken = 0;
  for (int sy = y0; sy < y1 && sy < height; ++sy) {
    for (int sx = x0; sx < x1 && sx < width; ++sx) {
      const uint8_t* p = src + ((int64_t)sy * width + sx) * 3;
      sums[0] += p[0];
      sums[1] += p[1];
      sums[2] += p[2];
      ++taken;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const uint8_t b = (uint8_t)(taken > 0 ? (sums[c] + taken / 2) / taken : 0);
    if (out_bytes != nullptr) out_bytes[i * 3 + c] = b;
    if (out_linear != nullptr) out_linear[i * 3 + c] = (float)b / 255.f;
  }
}

// A frame already at the target size (downscaleToWidth returns it unchanged,
// ImageIo.cpp:301-303): every byte divided by 255, 16 bytes per thread with
// 16-byte loads and stores. The same float as k_downscale writes for a box of
// one pixel.
__global__ void __launch_bounds__(256)
    k_bytes_to_linear16(const uint4* __restrict__ src, float4* __restrict__ out, int64_t n16) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n16) return;
  const uint4 w = src[i];
  const uint32_t words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t v = words[k];
    out[i * 4 + k] = make_float4((float)(v & 0xFFu) / 255.f, (float)((v >> 8) & 0xFFu) / 255.f,
                                 (float)((v >> 16) & 0xFFu) / 255.f, (float)(v >> 24) / 255.f);
  }
}

__global__ void __launch_bounds__(256)
    k_bytes_to_linear(const uint8_t* __restrict__ src, uint8_t* __restrict__ out_bytes,
                      float* __restrict__ out_linear, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t b = src[i];
  if (out_bytes != nullptr) out_bytes[i] = b;
  if (out_linear != nullptr) out_linear[i] = (float)b / 255.f;
}

// Several frames already at their view's size in one launch: thread i
// converts 16-byte group i of the frames laid end to end (frame j holds
// groups [start[j], start[j + 1])), with the arithmetic of k_bytes_to_linear16.
struct LinearFrames {
  const uint4* src[kMaxLinearFrames];
  float4* out[kMaxLinearFrames];
  int64_t start[kMaxLinearFrames + 1];
  int count;
};

__global__ void __launch_bounds__(256) k_bytes_to_linear16_frames(LinearFrames f) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.start[f.count]) return;
  int j = 0;
  while (j + 1 < f.count && f.start[j + 1] <= i) ++j;
  const int64_t g = i - f.start[j];
  const uint4 w = f.src[j][g];
  const uint32_t words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t v = words[k];
    f.out[j][g * 4 + k] = make_float4((float)(v & 0xFFu) / 255.f, (float)((v >> 8) & 0xFFu) / 255.f,
                                      (float)((v >> 16) & 0xFFu) / 255.f, (float)(v >> 24) / 255.f);
  }
}

bool linear_frame_ok(const uint8_t* src, const float* out, int64_t bytes) {
  return bytes > 0 && bytes % 16 == 0 && (reinterpret_cast<uintptr_t>(src) & 15u) == 0 &&
         (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
}

void launch_bytes_to_linear_frames(const uint8_t* const* src, float* const* out,
                                   const int64_t* bytes, int n, cudaStream_t stream) {
  for (int first = 0; first < n; first += kMaxLinearFrames) {
    LinearFrames f;
    f.count = std::min(kMaxLinearFrames, n - first);
    f.start[0] = 0;
    for (int j = 0; j < f.count; ++j) {
      f.src[j] = reinterpret_cast<const uint4*>(src[first + j]);
      f.out[j] = reinterpret_cast<float4*>(out[first + j]);
      f.start[j + 1] = f.start[j] + bytes[first + j] / 16;
    }
    const int64_t groups = f.start[f.count];
    if (groups <= 0) continue;
    count_launch();
    k_bytes_to_linear16_frames<<<(unsigned)((groups + 255) / 256), 256, 0, stream>>>(f);
  }
}

void launch_downscale(const uint8_t* src, int width, int height, int out_width, int out_height,
                      uint8_t* out_bytes, float* out_linear, cudaStream_t stream) {
  const int64_t n = (int64_t)out_width * out_height;
  if (n <= 0) return;
  count_launch();
  if (out_width == width && out_height == height) {
    const int64_t bytes = n * 3;
    const bool wide = out_bytes == nullptr && out_linear != nullptr && bytes % 16 == 0 &&
                      (reinterpret_cast<uintptr_t>(src) & 15u) == 0 &&
                      (reinterpret_cast<uintptr_t>(out_linear) & 15u) == 0;
    if (wide) {
      const int64_t n16 = bytes / 16;
      k_bytes_to_linear16<<<(unsigned)((n16 + 255) / 256), 256, 0, stream>>>(
          reinterpret_cast<const uint4*>(src), reinterpret_cast<float4*>(out_linear), n16);
    } else {
      k_bytes_to_linear<<<(unsigned)((bytes + 255) / 256), 256, 0, stream>>>(src, out_bytes,
                                                                             out_linear, bytes);
    }
    return;
  }
  k_downscale<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(src, width, height, out_width,
                                                               out_height, out_bytes, out_linear);
}

}  // namespace pxs
