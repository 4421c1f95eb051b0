// phmm_mlp_train.cu -- training kernels of the band MLP (80-128-128-2, ReLU).
//
// Master weights are FP32; every step rounds them to BF16 (the precision the
// tensor-core inference kernel uses) and runs forward and backward in FP32 on
// those rounded values, so the gradient is that of the deployed network
// (straight-through rounding).  The GEMMs with 80 or 128 rows on every side
// run on the tensor cores (tcgen05.mma kind::f16: BF16 operands, FP32
// accumulation in tensor memory) -- the two hidden layers' forward products
// (inputs, weights and hidden activations are BF16 values already), the
// hidden layers' weight gradients and the back-propagated hidden gradient
// (the FP32 gradient operands rounded to BF16, as mixed-precision training
// does); the products with the 2-wide output layer stay FP32 SIMT.  The loss
// is an asymmetric squared error on
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
#include "phmm_tc.cuh"

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

// ---- tensor-core GEMM ---------------------------------------------------------
// C = A . B^T over K with FP32 operands read through strides and rounded to
// BF16 while they are staged: A(r, k) = A[r sar + k sak] for r < m_valid and
// k < k_valid (else 0), B(n, k) = B[n sbn + k sbk] for k < k_valid; C FP32
// row-major (ldc = N), rows past m_valid not written.  N a multiple of 16, at
// most 128.  Block (x, y) takes rows 128 x .. 128 x + 127 and the K range
// y kspan .. (y + 1) kspan (kspan a multiple of 16) and writes its product to
// C + y c_split (split K: the partial products are summed in a fixed order by
// k_sum_splits).  Four warps: K in chunks of up to 64 staged into shared
// memory in the canonical K-major layout without swizzling, one thread issues
// the chunk's MMAs (K = 16 each) into the FP32 accumulator in tensor memory
// and commits them to an mbarrier, every thread waits (bounded: a wait that
// gives up sets *fail and the block skips its epilogue), and the warps drain
// the accumulator with tcgen05.ld (warp w: rows 32 w .. 32 w + 31).
constexpr int kTcKc = 64;
struct GemmTcSmem {
  __nv_bfloat16 a[128 * kTcKc];
  __nv_bfloat16 b[128 * kTcKc];
  uint64_t mbar;
  uint32_t tmem_base;
  int fail;
};
struct GemmTcArgs {
  const float* A;
  long long sar, sak;
  const float* B;
  long long sbn, sbk;
  float* C;
  long long c_split;
  int m_valid, N, k_valid, kspan;
};

// eight consecutive k of one row, rounded to BF16 (nearest even), zero where invalid
__device__ __forceinline__ uint4 stage8(const float* base, long long sk, bool row_ok, int k, int k_valid) {
  uint32_t w[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int k0 = k + 2 * t, k1 = k0 + 1;
    const float v0 = row_ok && k0 < k_valid ? base[(long long)k0 * sk] : 0.f;
    const float v1 = row_ok && k1 < k_valid ? base[(long long)k1 * sk] : 0.f;
    const __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
    w[t] = *reinterpret_cast<const uint32_t*>(&h);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

__global__ void __launch_bounds__(128, 1) k_gemm_tc(GemmTcArgs g, unsigned int* fail) {
  using namespace tc;
  __shared__ __align__(1024) GemmTcSmem s;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int row0 = blockIdx.x * 128;
  const int kb = blockIdx.y * g.kspan, ke = min(kb + g.kspan, g.k_valid);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem_base)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mbar)) : "memory");
    s.fail = 0;
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = s.tmem_base;
  const uint32_t idesc = instr_desc(128, g.N);
  unsigned char* sa = reinterpret_cast<unsigned char*>(s.a);
  unsigned char* sb = reinterpret_cast<unsigned char*>(s.b);
  unsigned phase = 0;
  bool any = false;  // the accumulator holds a product
  for (int k0 = kb; k0 < kb + g.kspan; k0 += kTcKc) {
    const int kc = min(kTcKc, kb + g.kspan - k0);  // a multiple of 16
    const int pieces = kc / 8;                     // 16-byte row pieces per row
    for (int x = tid; x < 128 * pieces; x += 128) {
      const int r = x / pieces, c = 8 * (x % pieces);
      const int gr = row0 + r;
      *reinterpret_cast<uint4*>(sa + core_offset(r, c, kc)) =
          stage8(g.A + (long long)gr * g.sar, g.sak, gr < g.m_valid, k0 + c, ke);
    }
    for (int x = tid; x < g.N * pieces; x += 128) {
      const int r = x / pieces, c = 8 * (x % pieces);
      *reinterpret_cast<uint4*>(sb + core_offset(r, c, kc)) = stage8(g.B + (long long)r * g.sbn, g.sbk, true, k0 + c, ke);
    }
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      const uint32_t sbo = sbo_for(kc);
      for (int k = 0; k < kc / 16; ++k)
        mma_f16(tmem, mat_desc(sa + k * 2 * kLbo, kLbo, sbo), mat_desc(sb + k * 2 * kLbo, kLbo, sbo), idesc,
                any || k > 0);
      mma_commit(&s.mbar);
    }
    any = true;
    if (!mbar_wait_parity(&s.mbar, phase)) {
      s.fail = 1;
      mbar_wait_parity(&s.mbar, phase);  // again bounded: the MMAs still reading this chunk
    }
    phase ^= 1u;
    fence_after_sync();
    __syncthreads();  // the chunk's shared memory is free for the next one
    if (*reinterpret_cast<volatile int*>(&s.fail)) break;
  }
  if (!*reinterpret_cast<volatile int*>(&s.fail)) {
    const int r = row0 + tid;
    float* C = g.C + blockIdx.y * g.c_split;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < g.N; c0 += 32) {
      float v[32];
      if (any) {
        tmem_ld32(trow + (uint32_t)c0, v);
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = 0.f;
      }
      if (r < g.m_valid) {
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (c0 + j < g.N) C[(size_t)r * g.N + c0 + j] = v[j];
      }
    }
  } else if (tid == 0) {
    atomicOr(fail, 1u);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem_base), "r"(128) : "memory");
  }
}

// out[x] = sum over s of part[s * n + x], s = 0, 1, .. in order
__global__ void k_sum_splits(const float* __restrict__ part, int splits, int n, float* __restrict__ out) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int sp = 0; sp < splits; ++sp) acc += part[(size_t)sp * n + x];
    out[x] = acc;
  }
}

// C[m x N] = A . B^T on the tensor cores (one K range)
inline void gemm_tc(GemmTcArgs g, unsigned int* fail, cudaStream_t st) {
  if (g.m_valid <= 0 || g.k_valid <= 0) return;
  g.c_split = 0;
  g.kspan = (g.k_valid + 15) / 16 * 16;
  k_gemm_tc<<<dim3((g.m_valid + 127) / 128, 1), 128, 0, st>>>(g, fail);
}
// C[128 x N] = A . B^T with K = the batch split into ranges of 128 (partials in `part`, summed in order)
inline void gemm_tc_splitk(GemmTcArgs g, float* part, unsigned int* fail, cudaStream_t st) {
  if (g.m_valid <= 0 || g.k_valid <= 0) return;
  float* C = g.C;
  const int splits = (g.k_valid + 127) / 128;
  g.C = part;
  g.c_split = (long long)g.m_valid * g.N;
  g.kspan = 128;
  k_gemm_tc<<<dim3((g.m_valid + 127) / 128, splits), 128, 0, st>>>(g, fail);
  k_sum_splits<<<64, 256, 0, st>>>(part, splits, g.m_valid * g.N, C);
}

}  // namespace

cudaError_t mlp_forward_backward(const MlpTrainBuffers& b, int n, float alpha, bool backward, cudaStream_t st) {
  const dim3 blk(TS, TS);
  const int o1 = 0, ob1 = kHid * kFeat, o2 = ob1 + kHid, ob2 = o2 + kHid * kHid, o3 = ob2 + kHid, ob3 = o3 + kOut * kHid;
  k_round_bf16<<<64, 256, 0, st>>>(b.w, b.wq, kMlpParamCount);
  // forward: the hidden layers on the tensor cores (X and the rounded weights are BF16 values)
  gemm_tc({b.X, kFeat, 1, b.wq + o1, kFeat, 1, b.Z1, 0, n, kHid, kFeat, 0}, b.tc_fail, st);
  k_bias_relu<<<256, 256, 0, st>>>(b.Z1, b.wq + ob1, b.H1, n, kHid, 1);
  gemm_tc({b.H1, kHid, 1, b.wq + o2, kHid, 1, b.Z2, 0, n, kHid, kHid, 0}, b.tc_fail, st);
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
  // dW2 = dZ2^T H1 (K = the batch, split in ranges of 128)
  gemm_tc_splitk({b.dH, 1, kHid, b.H1, 1, kHid, b.g + o2, 0, kHid, kHid, n, 0}, b.part, b.tc_fail, st);
  k_colsum<<<(kHid + 127) / 128, 128, 0, st>>>(b.dH, b.g + ob2, n, kHid);
  // dH1 = dZ2 W2 (B(i, o) = W2[o][i])
  gemm_tc({b.dH, kHid, 1, b.wq + o2, 1, kHid, b.dH2, 0, n, kHid, kHid, 0}, b.tc_fail, st);
  k_relu_bwd<<<256, 256, 0, st>>>(b.dH2, b.Z1, (long long)n * kHid);
  // dW1 = dZ1^T X
  gemm_tc_splitk({b.dH2, 1, kHid, b.X, 1, kFeat, b.g + o1, 0, kHid, kFeat, n, 0}, b.part, b.tc_fail, st);
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
