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

namespace bvphmm {
namespace {

constexpr int kMlpGroups = 4;                 // tiles in flight per block
constexpr int kMlpTile = 128;                 // pairs per tile (the MMA's M)
constexpr int kMlpThreads = kMlpGroups * 128;
constexpr int kOutPad = 16;                   // layer 3's N (two used columns)
constexpr unsigned kMmaWaitLimit = 1u << 24;  // polls before a completion wait gives up

// Canonical K-major layout without swizzling: 8 x 8 BF16 core matrices of
// 128 contiguous bytes (row r of the core matrix at +16 r); the core matrix
// holding rows 8i.. and columns 8j.. starts at i * SBO + j * LBO, LBO = 128.
constexpr uint32_t kLbo = 128;
constexpr uint32_t sbo_for(int k) { return (uint32_t)(k / 8) * 128u; }
__device__ __forceinline__ int core_offset(int row, int col, int k) {  // bytes
  return (row >> 3) * (int)sbo_for(k) + (col >> 3) * (int)kLbo + (row & 7) * 16 + (col & 7) * 2;
}

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

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// tcgen05 shared-memory matrix descriptor: start address, leading and stride
// byte offsets (all >> 4), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t mat_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((smem_u32(p) >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t instr_desc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate ? 1u : 0u)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// named barrier of one group's four warps
__device__ __forceinline__ void group_sync(int g) { asm volatile("bar.sync %0, 128;" ::"r"(g + 1) : "memory"); }

__device__ __forceinline__ bool mbar_wait_parity(uint64_t* mb, unsigned phase) {
  for (unsigned it = 0; it < kMmaWaitLimit; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(mb)), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}
__device__ __forceinline__ void tmem_ld2(uint32_t taddr, float* v) {
  uint32_t r0, r1;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  v[0] = __uint_as_float(r0);
  v[1] = __uint_as_float(r1);
}

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
