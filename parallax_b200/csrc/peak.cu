// peak.cu -- FP32 fused multiply-add throughput of this device, measured.
//
// The compositing kernels are bound by FP32 arithmetic, not by HBM or the
// tensor cores, so their roofline needs the FP32 peak; this microkernel runs
// independent FMA chains on every SM and reports the achieved TFLOP/s.
#include "common.cuh"
#include "kernels.h"
#include "runtime.h"

namespace pxs {

__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iterations, float seed) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 1e-7f + k;
  const float m = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iterations; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains live
}

float measure_fp32_peak_tflops(cudaStream_t stream) {
  int device = 0, sms = 0;
  PXS_CUDA(cudaGetDevice(&device));
  PXS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  float* out = nullptr;
  PXS_CUDA(cudaMalloc(&out, sizeof(float) * sms * 16));
  cudaEvent_t a, b;
  PXS_CUDA(cudaEventCreate(&a));
  PXS_CUDA(cudaEventCreate(&b));
  const int blocks = sms * 8, threads = 256, iterations = 1 << 14;
  float best = 0.f;
  for (int rep = 0; rep < 4; ++rep) {
    PXS_CUDA(cudaEventRecord(a, stream));
    count_launch();
    k_fma_peak<<<blocks, threads, 0, stream>>>(out, iterations, 1.0f + rep);
    PXS_CUDA(cudaEventRecord(b, stream));
    PXS_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    PXS_CUDA(cudaEventElapsedTime(&ms, a, b));
    const double flops = 2.0 * 8.0 * iterations * (double)blocks * threads;
    const float tflops = (float)(flops / (ms * 1e-3) / 1e12);
    if (rep > 0 && tflops > best) best = tflops;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  return best;
}

}  // namespace pxs
