// fp32_peak.cu -- measures the device's achievable FP32 FMA throughput.
//
// The PairHMM kernels are bound by the CUDA-core FP32 pipe, not by HBM or the
// tensor cores, so their roofline denominator is the chip's non-tensor FP32
// peak.  This probe runs independent FMA chains (8 per thread, enough warps
// to saturate every SM sub-partition) and times them with CUDA events.
#include <cuda_runtime.h>

#include <algorithm>

#include "bv_pairhmm.h"

namespace {

__global__ void __launch_bounds__(256) k_ffma(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-7f, x2 = x0 + 2e-7f, x3 = x0 + 3e-7f;
  float x4 = x0 + 4e-7f, x5 = x0 + 5e-7f, x6 = x0 + 6e-7f, x7 = x0 + 7e-7f;
  for (int k = 0; k < iters; ++k) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = __fmaf_rn(x0, a, b); x1 = __fmaf_rn(x1, a, b); x2 = __fmaf_rn(x2, a, b); x3 = __fmaf_rn(x3, a, b);
      x4 = __fmaf_rn(x4, a, b); x5 = __fmaf_rn(x5, a, b); x6 = __fmaf_rn(x6, a, b); x7 = __fmaf_rn(x7, a, b);
    }
  }
  const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 1.2345f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" int bv_phmm_measure_fp32_peak(int device, double* tflops) {
  if (!tflops) return BV_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return BV_ERR_NO_DEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  float* out = nullptr;
  const int threads = 256, blocks = sms * 8;
  if (cudaMalloc(&out, sizeof(float) * threads * blocks) != cudaSuccess) return BV_ERR_OOM;
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int iters = 4096;
  k_ffma<<<blocks, threads, 0, st>>>(out, 256, 0.999f, 1e-3f);  // warm-up
  double best = 0;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0, st);
    k_ffma<<<blocks, threads, 0, st>>>(out, iters, 0.999f, 1e-3f);
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
