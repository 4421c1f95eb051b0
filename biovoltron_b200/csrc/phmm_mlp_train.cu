// phmm_mlp_train.cu -- training kernels of the band MLP (80-128-128-2, ReLU).
//
// Master weights are FP32; every step rounds them to BF16 (the precision the
// tensor-core inference kernel uses) and runs forward and backward in FP32 on
// those rounded values, so the gradient is that of the deployed network
// (straight-through rounding).  The loss is an asymmetric squared error on
// the band's lower and upper edge (diagonals relative to the seed diagonal):
//   L = mean( w_lo (o_lo - t_lo)^2 + w_hi (o_hi - t_hi)^2 ),
//   w_lo = alpha if o_lo > t_lo (band too narrow below) else 1,
//   w_hi = alpha if o_hi < t_hi (band too narrow above) else 1,
// so under-covering the posterior spread costs alpha times more than
// over-covering it.  Optimiser: Adam.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "phmm_band.h"
#include "phmm_mlp.h"

namespace bvphmm {
namespace {

constexpr int TS = 16;

// C[M x N] = op(A) op(B) (+ C if accumulate); A is M x K (or K x M when ta),
// B is K x N (or N x K when tb); all row-major FP32.
__global__ void k_gemm(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ Cm, int M, int N,
                       int K, int ta, int tb, int accumulate) {
  __shared__ float sa[TS][TS + 1], sb[TS][TS + 1];
  const int row = blockIdx.y * TS + threadIdx.y, col = blockIdx.x * TS + threadIdx.x;
  float acc = 0.f;
  for (int k0 = 0; k0 < K; k0 += TS) {
    const int ka = k0 + threadIdx.x, kb = k0 + threadIdx.y;
    float va = 0.f, vb = 0.f;
    if (row < M && ka < K) va = ta ? A[(size_t)ka * M + row] : A[(size_t)row * K + ka];
    if (col < N && kb < K) vb = tb ? B[(size_t)col * K + kb] : B[(size_t)kb * N + col];
    sa[threadIdx.y][threadIdx.x] = va;
    sb[threadIdx.y][threadIdx.x] = vb;
    __syncthreads();
#pragma unroll
    for (int t = 0; t < TS; ++t) acc = fmaf(sa[threadIdx.y][t], sb[t][threadIdx.x], acc);
    __syncthreads();
  }
  if (row < M && col < N) {
    float* c = Cm + (size_t)row * N + col;
    *c = accumulate ? *c + acc : acc;
  }
}

// weight matrices to BF16, biases unchanged (the inference kernel keeps FP32 biases)
__global__ void k_round_bf16(const float* __restrict__ w, float* __restrict__ wq, int n) {
  const int n1 = kHid * kFeat, n2 = kHid * kHid;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    const bool bias = (x >= n1 && x < n1 + kHid) || (x >= n1 + kHid + n2 && x < n1 + 2 * kHid + n2) ||
                      x >= n1 + 2 * kHid + n2 + kOut * kHid;
    wq[x] = bias ? w[x] : __bfloat162float(__float2bfloat16(w[x]));
  }
}

// Z[r][c] += bias[c]; H = relu(Z) rounded to BF16, as the inference kernel
// stores its hidden activations (the gradient passes the rounding straight)
__global__ void k_bias_relu(float* __restrict__ Z, const float* __restrict__ bias, float* __restrict__ Hout, int rows,
                            int cols, int relu) {
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < (long long)rows * cols;
       x += (long long)gridDim.x * blockDim.x) {
    const float z = Z[x] + bias[x % cols];
    Z[x] = z;
    if (Hout) Hout[x] = relu ? __bfloat162float(__float2bfloat16(fmaxf(z, 0.f))) : z;
  }
}

__global__ void k_relu_bwd(float* __restrict__ dH, const float* __restrict__ Z, long long n) {
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x)
    if (!(Z[x] > 0.f)) dH[x] = 0.f;
}

// db[c] = sum_r dZ[r][c]
__global__ void k_colsum(const float* __restrict__ dZ, float* __restrict__ db, int rows, int cols) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += dZ[(size_t)r * cols + c];
  db[c] = s;
}

__global__ void k_loss(const float* __restrict__ O, const float* __restrict__ T, const float* __restrict__ mask,
                       float* __restrict__ dO, float* __restrict__ loss, int rows, float alpha, float inv_n) {
  float l = 0.f;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const float m = mask ? mask[r] : 1.f;
    const float e0 = O[2 * r] - T[2 * r], e1 = O[2 * r + 1] - T[2 * r + 1];
    const float w0 = e0 > 0.f ? alpha : 1.f, w1 = e1 < 0.f ? alpha : 1.f;
    dO[2 * r] = m * 2.f * w0 * e0 * inv_n;
    dO[2 * r + 1] = m * 2.f * w1 * e1 * inv_n;
    l += m * (w0 * e0 * e0 + w1 * e1 * e1);
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l * inv_n);
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    const float gg = g[x];
    const float mm = b1 * m[x] + (1.f - b1) * gg;
    const float vv = b2 * v[x] + (1.f - b2) * gg * gg;
    m[x] = mm;
    v[x] = vv;
    w[x] -= lr * (mm * c1) / (sqrtf(vv * c2) + eps);
  }
}

__global__ void k_gather_rows(const __nv_bfloat16* __restrict__ feat, const float* __restrict__ targets,
                              const float* __restrict__ mask, const int32_t* __restrict__ idx, int n, float* __restrict__ X,
                              float* __restrict__ T, float* __restrict__ Mk) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n * kFeat; x += gridDim.x * blockDim.x) {
    const int r = x / kFeat, c = x % kFeat;
    const long long src = idx ? idx[r] : r;
    X[x] = __bfloat162float(feat[src * kFeat + c]);
    if (c < 2) T[2 * r + c] = targets[2 * src + c];
    if (c == 0) Mk[r] = mask ? mask[src] : 1.f;
  }
}

__global__ void k_export_params(const float* __restrict__ w, MlpParams* __restrict__ out) {
  const int n1 = kHid * kFeat, n2 = kHid * kHid, n3 = kOut * kHid;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < kMlpParamCount; x += gridDim.x * blockDim.x) {
    const float v = w[x];
    if (x < n1) out->w1[x] = __float2bfloat16(v);
    else if (x < n1 + kHid) out->b1[x - n1] = v;
    else if (x < n1 + kHid + n2) out->w2[x - n1 - kHid] = __float2bfloat16(v);
    else if (x < n1 + 2 * kHid + n2) out->b2[x - n1 - kHid - n2] = v;
    else if (x < n1 + 2 * kHid + n2 + n3) out->w3[x - n1 - 2 * kHid - n2] = __float2bfloat16(v);
    else out->b3[x - n1 - 2 * kHid - n2 - n3] = v;
  }
}

inline dim3 grid2(int M, int N) { return dim3((N + TS - 1) / TS, (M + TS - 1) / TS); }

}  // namespace

cudaError_t mlp_forward_backward(const MlpTrainBuffers& b, int n, float alpha, bool backward, cudaStream_t st) {
  const dim3 blk(TS, TS);
  const int o1 = 0, ob1 = kHid * kFeat, o2 = ob1 + kHid, ob2 = o2 + kHid * kHid, o3 = ob2 + kHid, ob3 = o3 + kOut * kHid;
  k_round_bf16<<<64, 256, 0, st>>>(b.w, b.wq, kMlpParamCount);
  // forward
  k_gemm<<<grid2(n, kHid), blk, 0, st>>>(b.X, b.wq + o1, b.Z1, n, kHid, kFeat, 0, 1, 0);
  k_bias_relu<<<256, 256, 0, st>>>(b.Z1, b.wq + ob1, b.H1, n, kHid, 1);
  k_gemm<<<grid2(n, kHid), blk, 0, st>>>(b.H1, b.wq + o2, b.Z2, n, kHid, kHid, 0, 1, 0);
  k_bias_relu<<<256, 256, 0, st>>>(b.Z2, b.wq + ob2, b.H2, n, kHid, 1);
  k_gemm<<<grid2(n, kOut), blk, 0, st>>>(b.H2, b.wq + o3, b.O, n, kOut, kHid, 0, 1, 0);
  k_bias_relu<<<256, 256, 0, st>>>(b.O, b.wq + ob3, nullptr, n, kOut, 0);
  cudaMemsetAsync(b.loss, 0, sizeof(float), st);
  k_loss<<<64, 256, 0, st>>>(b.O, b.T, b.mask, b.dO, b.loss, n, alpha, 1.f / (float)n);
  if (!backward) return cudaGetLastError();
  // backward: dW = dZ^T H, db = colsum(dZ), dH_prev = dZ W
  k_gemm<<<grid2(kOut, kHid), blk, 0, st>>>(b.dO, b.H2, b.g + o3, kOut, kHid, n, 1, 0, 0);
  k_colsum<<<1, 32, 0, st>>>(b.dO, b.g + ob3, n, kOut);
  k_gemm<<<grid2(n, kHid), blk, 0, st>>>(b.dO, b.wq + o3, b.dH, n, kHid, kOut, 0, 0, 0);
  k_relu_bwd<<<256, 256, 0, st>>>(b.dH, b.Z2, (long long)n * kHid);
  k_gemm<<<grid2(kHid, kHid), blk, 0, st>>>(b.dH, b.H1, b.g + o2, kHid, kHid, n, 1, 0, 0);
  k_colsum<<<(kHid + 127) / 128, 128, 0, st>>>(b.dH, b.g + ob2, n, kHid);
  k_gemm<<<grid2(n, kHid), blk, 0, st>>>(b.dH, b.wq + o2, b.dH2, n, kHid, kHid, 0, 0, 0);
  k_relu_bwd<<<256, 256, 0, st>>>(b.dH2, b.Z1, (long long)n * kHid);
  k_gemm<<<grid2(kHid, kFeat), blk, 0, st>>>(b.dH2, b.X, b.g + o1, kHid, kFeat, n, 1, 0, 0);
  k_colsum<<<(kHid + 127) / 128, 128, 0, st>>>(b.dH2, b.g + ob1, n, kHid);
  return cudaGetLastError();
}

cudaError_t mlp_adam(const MlpTrainBuffers& b, int step, float lr, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f / (1.f - powf(b1, (float)step)), c2 = 1.f / (1.f - powf(b2, (float)step));
  k_adam<<<64, 256, 0, st>>>(b.w, b.g, b.m, b.v, kMlpParamCount, lr, b1, b2, 1e-8f, c1, c2);
  return cudaGetLastError();
}

cudaError_t mlp_gather(const __nv_bfloat16* feat, const float* targets, const float* mask, const int32_t* idx, int n,
                       const MlpTrainBuffers& b, cudaStream_t st) {
  k_gather_rows<<<256, 256, 0, st>>>(feat, targets, mask, idx, n, b.X, b.T, b.mask);
  return cudaGetLastError();
}

cudaError_t mlp_export(const float* w, MlpParams* out, cudaStream_t st) {
  k_export_params<<<64, 256, 0, st>>>(w, out);
  return cudaGetLastError();
}

}  // namespace bvphmm
