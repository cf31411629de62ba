// FMA issue-rate microbenchmarks: the roofline denominators for the ERI
// kernels, which run on the FP64 CUDA-core pipe (plain form) and partly on
// the FP32 pipe (precision form).  Eight independent FMA chains per thread
// keep the pipe full; the result is stored so the chains are not eliminated.
#include <cuda_runtime.h>

#include <string>

#include "../../include/hfgpu.h"

namespace {

constexpr int kIters = 4096;

template <class T>
__global__ void fma_chains(T *out, T a, T b) {
  T x0 = T(threadIdx.x * 1e-9), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3), x4 = x0 + T(4), x5 = x0 + T(5),
    x6 = x0 + T(6), x7 = x0 + T(7);
#pragma unroll 16
  for (int i = 0; i < kIters; ++i) {
    x0 = fma(x0, a, b);
    x1 = fma(x1, a, b);
    x2 = fma(x2, a, b);
    x3 = fma(x3, a, b);
    x4 = fma(x4, a, b);
    x5 = fma(x5, a, b);
    x6 = fma(x6, a, b);
    x7 = fma(x7, a, b);
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

template <class T>
hfg_status measure_peak(int32_t device, double *tflops) {
  if (!tflops) return HFG_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return HFG_NO_DEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int threads = 256, blocks = sms * 8;
  T *out = nullptr;
  if (cudaMalloc(&out, sizeof(T) * threads * blocks) != cudaSuccess) return HFG_OOM_BUDGET;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_chains<T><<<blocks, threads>>>(out, T(0.999999), T(1e-7));  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0);
    fma_chains<T><<<blocks, threads>>>(out, T(0.999999), T(1e-7));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return HFG_DEVICE_ERROR;
  const double flops = 2.0 * 8.0 * kIters * (double)threads * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return HFG_OK;
}

}  // namespace

extern "C" hfg_status hfg_measure_fp64_peak(int32_t device, double *tflops) { return measure_peak<double>(device, tflops); }

extern "C" hfg_status hfg_measure_fp32_peak(int32_t device, double *tflops) { return measure_peak<float>(device, tflops); }
