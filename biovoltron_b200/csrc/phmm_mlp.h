// phmm_mlp.h -- band MLP training interface (kernels in phmm_mlp_train.cu,
// label kernel in phmm_labels.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "phmm_band.h"
#include "phmm_common.h"

namespace bvphmm {

// Flattened FP32 parameters: W1 [kHid][kFeat], b1 [kHid], W2 [kHid][kHid],
// b2 [kHid], W3 [kOut][kHid], b3 [kOut] (weights as [out][in]).
constexpr int kMlpParamCount = kHid * kFeat + kHid + kHid * kHid + kHid + kOut * kHid + kOut;

struct MlpTrainBuffers {
  float* w;      // master weights
  float* wq;     // BF16-rounded copy used by forward and backward
  float* g;      // gradient
  float* m;      // Adam moments
  float* v;
  float* X;      // [cap][kFeat] minibatch inputs
  float* T;      // [cap][2] targets
  float* mask;   // [cap]
  float* Z1; float* H1; float* Z2; float* H2; float* O;
  float* dO; float* dH; float* dH2;
  float* loss;   // scalar
  float* part;             // split-K partial products of the weight gradients, ceil(cap / 128) x 128 x 128
  unsigned int* tc_fail;   // set when a tensor-core GEMM's completion wait gave up
  int cap;
};

cudaError_t mlp_forward_backward(const MlpTrainBuffers& b, int n, float alpha, bool backward, cudaStream_t st);
cudaError_t mlp_adam(const MlpTrainBuffers& b, int step, float lr, cudaStream_t st);
cudaError_t mlp_gather(const __nv_bfloat16* feat, const float* targets, const float* mask, const int32_t* idx, int n,
                       const MlpTrainBuffers& b, cudaStream_t st);
cudaError_t mlp_export(const float* w, MlpParams* out, cudaStream_t st);

// Label kernel (one warp per pair; each warp keeps its forward rows in
// fbuf + warp * fbuf_stride, so fbuf holds blocks * label_warps_per_block()
// strides of floats).
int label_smem_bytes();
int label_warps_per_block();
cudaError_t launch_posterior_spread(const DeviceBatch& b, const Tables* tb, const int32_t* pair_read,
                                    const int32_t* pair_hap, long long n_pairs, float tau, float* fbuf,
                                    long long fbuf_stride, int32_t* lo, int32_t* hi, int blocks, cudaStream_t st);

}  // namespace bvphmm
