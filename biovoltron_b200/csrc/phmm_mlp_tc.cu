// phmm_mlp_tc.cu -- band MLP inference on the 5th-generation tensor cores.
//
// The network (80 -> 128 ReLU -> 128 ReLU -> 2, BF16 weights and hidden
// activations, FP32 accumulation and biases) scores 128 pairs per tile with
// tcgen05.mma (kind::f16, BF16 operands, M = 128): the A operand (features,
// then hidden activations) and the B operand (weights) sit in shared memory
// in the canonical K-major layout without swizzling, the accumulator in
// tensor memory (TMEM).  A block holds kMlpGroups groups of four warps; each
// group owns a tile, 128 TMEM columns and an mbarrier, its first thread
// issues the group's MMAs, and the four warps drain the accumulator with
// tcgen05.ld (warp w reads TMEM lanes 32w..32w+31, i.e. the tile's rows),
// add the bias, apply ReLU, round to BF16 and write the next layer's A
// operand.  The groups interleave, so one group's epilogue overlaps another
// group's MMAs.  The weights are staged once per block.  Every wait on an
// MMA completion is bounded; a wait that gives up sets status bit 16 and the
// block stops after releasing its TMEM.  Single-GPU kernel: every operand is
// this GPU's own memory, and no TMA or multicast copy is used.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "phmm_band.h"
#include "phmm_common.h"
#include "phmm_kernels.h"
#include "phmm_tc.cuh"

namespace bvphmm {
namespace {

constexpr int kMlpGroups = 4;                 // tiles in flight per block
constexpr int kMlpTile = 128;                 // pairs per tile (the MMA's M)
constexpr int kMlpThreads = kMlpGroups * 128;
constexpr int kOutPad = 16;                   // layer 3's N (two used columns)

using namespace tc;

struct MlpTcSmem {
  __nv_bfloat16 w1[kHid * kFeat];      // B of layer 1: [128][80]
  __nv_bfloat16 w2[kHid * kHid];       // B of layer 2: [128][128]
  __nv_bfloat16 w3[kOutPad * kHid];    // B of layer 3: [16][128], rows 2.. zero
  __nv_bfloat16 act[kMlpGroups][kMlpTile * kHid];  // per group: A of the current layer
  float b1[kHid], b2[kHid], b3[kOut];
  uint64_t mbar[kMlpGroups];
  uint32_t tmem_base;
  int fail;
};

// This thread's accumulator row, columns [0, 128): bias, ReLU, BF16, written
// as row `row` of the next layer's A operand (K = 128).  Same rounding as the
// training kernels: fmaxf(acc + bias, 0) to the nearest BF16.
__device__ __forceinline__ void hidden_epilogue(uint32_t trow, const float* bias, unsigned char* act, int row) {
#pragma unroll 1
  for (int c0 = 0; c0 < kHid; c0 += 32) {
    float v[32];
    tmem_ld32(trow + (uint32_t)c0, v);
#pragma unroll
    for (int j8 = 0; j8 < 4; ++j8) {
      uint32_t w[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int j = 8 * j8 + 2 * t;
        const __nv_bfloat162 b2 =
            __floats2bfloat162_rn(fmaxf(v[j] + bias[c0 + j], 0.f), fmaxf(v[j + 1] + bias[c0 + j + 1], 0.f));
        w[t] = *reinterpret_cast<const uint32_t*>(&b2);
      }
      *reinterpret_cast<uint4*>(act + core_offset(row, c0 + 8 * j8, kHid)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// One layer's MMAs over K (16 per instruction): D[tmem] (+)= A x B^T.
template <int K, int N>
__device__ __forceinline__ void layer_mma(uint32_t d_tmem, const unsigned char* a, const unsigned char* b) {
  constexpr uint32_t kSbo = sbo_for(K);
  constexpr uint32_t kIdesc = instr_desc(kMlpTile, N);
#pragma unroll
  for (int k = 0; k < K / 16; ++k)
    mma_f16(d_tmem, mat_desc(a + k * 2 * kLbo, kLbo, kSbo), mat_desc(b + k * 2 * kLbo, kLbo, kSbo), kIdesc, k > 0);
}

// Waits for the group's MMAs; a wait that gives up sets status bit 16 and the
// shared fail flag (every group then leaves its loop at its next check), and
// waits once more, again bounded, for the MMAs still in flight.
__device__ __forceinline__ bool group_wait(MlpTcSmem& s, const BandParams& p, int g, unsigned& phase) {
  bool ok = mbar_wait_parity(&s.mbar[g], phase);
  if (!ok) {
    atomicOr(&p.ctr->status, 16ull);
    s.fail = 1;
    mbar_wait_parity(&s.mbar[g], phase);
  }
  phase ^= 1u;
  fence_after_sync();
  group_sync(g);
  return !*reinterpret_cast<volatile int*>(&s.fail);
}

__global__ void __launch_bounds__(kMlpThreads, 1) k_mlp_forward_tc(BandParams p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  MlpTcSmem& s = *reinterpret_cast<MlpTcSmem*>(smem_raw);
  const int tid = threadIdx.x, g = tid >> 7, gt = tid & 127, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem_base)),
                 "r"(kMlpGroups * 128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid < kMlpGroups)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mbar[tid])) : "memory");
  if (tid == 0) s.fail = 0;
  // weights into the canonical layout, one 16-byte row chunk per thread and step
  const MlpParams* W = p.mlp;
  unsigned char* w1 = reinterpret_cast<unsigned char*>(s.w1);
  unsigned char* w2 = reinterpret_cast<unsigned char*>(s.w2);
  unsigned char* w3 = reinterpret_cast<unsigned char*>(s.w3);
  for (int x = tid; x < kHid * kFeat / 8; x += kMlpThreads) {
    const int r = x / (kFeat / 8), c = 8 * (x % (kFeat / 8));
    *reinterpret_cast<uint4*>(w1 + core_offset(r, c, kFeat)) = *reinterpret_cast<const uint4*>(W->w1 + r * kFeat + c);
  }
  for (int x = tid; x < kHid * kHid / 8; x += kMlpThreads) {
    const int r = x / (kHid / 8), c = 8 * (x % (kHid / 8));
    *reinterpret_cast<uint4*>(w2 + core_offset(r, c, kHid)) = *reinterpret_cast<const uint4*>(W->w2 + r * kHid + c);
  }
  for (int x = tid; x < kOutPad * kHid / 8; x += kMlpThreads) {
    const int r = x / (kHid / 8), c = 8 * (x % (kHid / 8));
    *reinterpret_cast<uint4*>(w3 + core_offset(r, c, kHid)) =
        r < kOut ? *reinterpret_cast<const uint4*>(W->w3 + r * kHid + c) : make_uint4(0, 0, 0, 0);
  }
  for (int x = tid; x < kHid; x += kMlpThreads) {
    s.b1[x] = W->b1[x];
    s.b2[x] = W->b2[x];
  }
  if (tid < kOut) s.b3[tid] = W->b3[tid];
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tcol = s.tmem_base + (uint32_t)(g * 128);           // the group's 128 columns
  const uint32_t trow = tcol + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's 32 lanes
  unsigned char* act = reinterpret_cast<unsigned char*>(s.act[g]);
  unsigned phase = 0;
  const long long ntiles = (p.n_pairs + kMlpTile - 1) / kMlpTile;
  for (long long tile = (long long)blockIdx.x * kMlpGroups + g; tile < ntiles;
       tile += (long long)gridDim.x * kMlpGroups) {
    const long long row = tile * kMlpTile + gt;
    // layer 1: the tile's features (rows past the end zero)
    const uint4* src = reinterpret_cast<const uint4*>(p.feat + row * kFeat);
#pragma unroll
    for (int c = 0; c < kFeat / 8; ++c)
      *reinterpret_cast<uint4*>(act + core_offset(gt, 8 * c, kFeat)) =
          row < p.n_pairs ? __ldg(src + c) : make_uint4(0, 0, 0, 0);
    fence_async_smem();
    fence_before_sync();
    group_sync(g);
    if (gt == 0) {
      fence_after_sync();
      layer_mma<kFeat, kHid>(tcol, act, w1);
      mma_commit(&s.mbar[g]);
    }
    if (!group_wait(s, p, g, phase)) break;
    hidden_epilogue(trow, s.b1, act, gt);
    fence_async_smem();
    fence_before_sync();
    group_sync(g);
    if (gt == 0) {
      fence_after_sync();
      layer_mma<kHid, kHid>(tcol, act, w2);
      mma_commit(&s.mbar[g]);
    }
    if (!group_wait(s, p, g, phase)) break;
    hidden_epilogue(trow, s.b2, act, gt);
    fence_async_smem();
    fence_before_sync();
    group_sync(g);
    if (gt == 0) {
      fence_after_sync();
      layer_mma<kHid, kOutPad>(tcol, act, w3);
      mma_commit(&s.mbar[g]);
    }
    if (!group_wait(s, p, g, phase)) break;
    float o[2];
    tmem_ld2(trow, o);
    if (row < p.n_pairs) {
      p.mlp_out[row * kOut + 0] = o[0] + s.b3[0];
      p.mlp_out[row * kOut + 1] = o[1] + s.b3[1];
    }
    // the next tile's MMAs overwrite these columns and this group's A tile
    fence_before_sync();
    group_sync(g);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem_base), "r"(kMlpGroups * 128)
                 : "memory");
  }
}

}  // namespace

cudaError_t prepare_mlp_tc() {
  return raise_dynamic_smem(reinterpret_cast<const void*>(&k_mlp_forward_tc), (int)sizeof(MlpTcSmem));
}

cudaError_t launch_mlp_forward_tc(const BandParams& p, int sms, cudaStream_t st) {
  if (p.n_pairs <= 0) return cudaSuccess;
  const cudaError_t e = prepare_mlp_tc();  // sets the attribute once per device
  if (e != cudaSuccess) return e;
  const long long tiles = (p.n_pairs + kMlpTile - 1) / kMlpTile;
  const long long blocks = std::min<long long>((tiles + kMlpGroups - 1) / kMlpGroups, (long long)sms);
  k_mlp_forward_tc<<<(int)blocks, kMlpThreads, (int)sizeof(MlpTcSmem), st>>>(p);
  return cudaGetLastError();
}

}  // namespace bvphmm
