// Compute-pipe peaks of the device, measured with CUDA events, for the
// roofline of the render (FP32 CUDA-core multiply-adds and exp2f on the
// special-function unit) and of the float64 solves:
//   out[0]  FP32 multiply-add rate, TFLOP/s (2 flops per FMA)
//   out[1]  exp2f rate, 10^12 evaluations/s (the render's exponential)
//   out[2]  FP64 multiply-add rate, TFLOP/s
// Each kernel runs independent dependency chains in every thread of a grid
// of 8 CTAs of 256 threads per SM, a few ms per launch so that launch
// overhead is negligible; the best of three timed launches after a warm-up
// is kept.
#include <cuda_runtime.h>

#include <algorithm>

#include "uph_internal.cuh"

namespace {

constexpr int PK_THREADS = 256;
constexpr int PK_CHAINS = 8;

__global__ void __launch_bounds__(PK_THREADS) k_peak_fma(int iters, float* out) {
  float a[PK_CHAINS];
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) a[j] = 1.0f + 1e-3f * (threadIdx.x + j);
  const float m = 0.99999f, c = 1e-5f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int j = 0; j < PK_CHAINS; ++j) a[j] = fmaf(a[j], m, c);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) s += a[j];
  if (s == -1.0f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;   // never true
}

__global__ void __launch_bounds__(PK_THREADS) k_peak_exp2(int iters, float* out) {
  float a[PK_CHAINS];
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) a[j] = -1e-3f * (threadIdx.x + j);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int j = 0; j < PK_CHAINS; ++j) a[j] = exp2f(-a[j]) - 1.5f;   // stays within (-1.5, 1.5)
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) s += a[j];
  if (s == -1.0f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(PK_THREADS) k_peak_dfma(int iters, double* out) {
  double a[PK_CHAINS];
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) a[j] = 1.0 + 1e-3 * (threadIdx.x + j);
  const double m = 0.99999, c = 1e-5;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int j = 0; j < PK_CHAINS; ++j) a[j] = fma(a[j], m, c);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < PK_CHAINS; ++j) s += a[j];
  if (s == -1.0) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <class F>
float best_ms(F&& launch, cudaEvent_t e0, cudaEvent_t e1, cudaStream_t s) {
  launch();   // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0, s);
    launch();
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  return best;
}

}  // namespace

int measure_peaks(cudaStream_t s, int sms, double* out) {
  const int blocks = sms * 8;
  const size_t threads = (size_t)blocks * PK_THREADS;
  void* sink = nullptr;
  cudaError_t err = cudaMalloc(&sink, threads * sizeof(double));
  if (err != cudaSuccess) return (int)err;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int it_fma = 4096, it_exp = 2048, it_dfma = 1024;
  const float ms_fma = best_ms([&] {
    k_peak_fma<<<blocks, PK_THREADS, 0, s>>>(it_fma, (float*)sink);
  }, e0, e1, s);
  const float ms_exp = best_ms([&] {
    k_peak_exp2<<<blocks, PK_THREADS, 0, s>>>(it_exp, (float*)sink);
  }, e0, e1, s);
  const float ms_dfma = best_ms([&] {
    k_peak_dfma<<<blocks, PK_THREADS, 0, s>>>(it_dfma, (double*)sink);
  }, e0, e1, s);
  err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess) return (int)err;
  const double n = (double)threads * PK_CHAINS;
  out[0] = 2.0 * n * it_fma * 16 / (ms_fma * 1e-3) / 1e12;
  out[1] = n * it_exp * 4 / (ms_exp * 1e-3) / 1e12;
  out[2] = 2.0 * n * it_dfma * 4 / (ms_dfma * 1e-3) / 1e12;
  return 0;
}
