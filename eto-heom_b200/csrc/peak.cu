// Measured CUDA-core FMA throughput of the current GPU (the roofline denominator of the
// propagation kernels, which run on the FP32/FP64 FMA pipes, not on the tensor cores).
#include <cuda_runtime.h>

#include "../../include/heom.h"

namespace {

template <typename T>
__global__ void __launch_bounds__(512) fma_loop(T *out, int iters, T seed) {
  // 8 independent chains per thread keep the FMA pipe full.
  T a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const T m = (T)0.9999999, c = (T)1e-7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
      a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
      a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
  }
  const T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == (T)-1) out[blockIdx.x] = s; // never true; keeps the chains live
}

template <typename T> int measure(int device, double *tflops) {
  if (cudaSetDevice(device) != cudaSuccess) return HEOM_ERR_CUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  T *out = nullptr;
  if (cudaMalloc(&out, sizeof(T) * sms * 8) != cudaSuccess) return HEOM_ERR_NOMEM;
  const int blocks = sms * 4, threads = 512, iters = sizeof(T) == 4 ? 4096 : 1024;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_loop<T><<<blocks, threads>>>(out, 64, (T)1);
  cudaEventRecord(e0);
  fma_loop<T><<<blocks, threads>>>(out, iters, (T)1);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess || ms <= 0) return HEOM_ERR_CUDA;
  const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return HEOM_OK;
}

} // namespace

extern "C" int heom_measure_fma_peak(int device, int fp64, double *tflops) {
  if (!tflops) return HEOM_ERR_ARG;
  return fp64 ? measure<double>(device, tflops) : measure<float>(device, tflops);
}
