// ingest.cu -- training images from 8-bit camera frames, on the device.
//
// Pipeline::Impl::runSplatTraining (Pipeline.cpp:1892-1917) downscales each
// frame with downscaleToWidth (ImageIo.cpp:300-337) and divides every byte by
// 255 into the float image the trainer fits. Here one thread per output pixel
// averages its box of source pixels with the same integer arithmetic (box
// edges from 64-bit products, the sum rounded by adding half the count) and
// writes the byte and / or the float; the 8-bit frame crosses PCIe instead of
// the four times larger float image.
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

void launch_downscale(const uint8_t* src, int width, int height, int out_width, int out_height,
                      uint8_t* out_bytes, float* out_linear, cudaStream_t stream) {
  const int64_t n = (int64_t)out_width * out_height;
  if (n <= 0) return;
  count_launch();
  k_downscale<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(src, width, height, out_width,
                                                               out_height, out_bytes, out_linear);
}

}  // namespace pxs
