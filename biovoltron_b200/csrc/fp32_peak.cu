// fp32_peak.cu -- measures the device's achievable FP32 and FP64 FMA
// throughput.
//
// The PairHMM kernels are bound by the CUDA-core FP32 pipe (the FP64 rescue
// kernel by the FP64 pipe), not by HBM or the tensor cores, so their roofline
// denominators are the chip's non-tensor FP32 and FP64 peaks.  This probe runs
// independent FMA chains (8 per thread, enough warps to saturate every SM
// sub-partition) and times them with CUDA events.
#include <cuda_runtime.h>

#include <algorithm>

#include "bv_pairhmm.h"

namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_ffma(T* out, int iters, T a, T b) {
  T x0 = threadIdx.x * T(1e-7), x1 = x0 + T(1e-7), x2 = x0 + T(2e-7), x3 = x0 + T(3e-7);
  T x4 = x0 + T(4e-7), x5 = x0 + T(5e-7), x6 = x0 + T(6e-7), x7 = x0 + T(7e-7);
  for (int k = 0; k < iters; ++k) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == T(1.2345)) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

// Best of five timed runs, in TFLOP/s (an FMA counts two flops).
template <typename T>
int measure_peak(int device, int iters, double* tflops) {
  if (!tflops) return BV_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return BV_ERR_NO_DEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  T* out = nullptr;
  const int threads = 256, blocks = sms * 8;
  if (cudaMalloc(&out, sizeof(T) * threads * blocks) != cudaSuccess) return BV_ERR_OOM;
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_ffma<T><<<blocks, threads, 0, st>>>(out, iters / 16, T(0.999), T(1e-3));  // warm-up
  double best = 0;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0, st);
    k_ffma<T><<<blocks, threads, 0, st>>>(out, iters, T(0.999), T(1e-3));
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    if (ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  cudaFree(out);
  if (err != cudaSuccess) return BV_ERR_CUDA;
  *tflops = best;
  return BV_OK;
}

}  // namespace

extern "C" int bv_phmm_measure_fp32_peak(int device, double* tflops) { return measure_peak<float>(device, 4096, tflops); }

extern "C" int bv_phmm_measure_fp64_peak(int device, double* tflops) { return measure_peak<double>(device, 1024, tflops); }
