// phmm_forward.cu -- PairHMM forward pass on sm_100a.
//
// Computes, for each (read, haplotype) pair, the quantity that
// compute_full_prob_avx{s,d} returns (lib/intel_native/pairhmm/
// avx-pairhmm-template.h:210-346): the sum over the last read row of M + X of
// the Match/Insert/Delete forward DP, scaled by INITIAL_CONSTANT, with the
// per-row transition probabilities of initializeVectors (:83-128) and the
// emission select of computeDistVec (:70-75).  The recurrence (computeMXY,
// :183-198) is
//
//   M(r,c) = e(r,c) * (pMM(r) M(r-1,c-1) + pGAPM(r) (X(r-1,c-1) + Y(r-1,c-1)))
//   X(r,c) = pMX(r) M(r-1,c) + pXX(r) X(r-1,c)
//   Y(r,c) = pMY(r) M(r,c-1) + pYY(r) Y(r,c-1)
//
// with Y(0,c) = INITIAL_CONSTANT / haplen on row 0.
//
// GPU formulation
// ---------------
// * One warp per pair.  Lane k owns RT consecutive rows of a strip of 32*RT
//   rows and sweeps the haplotype columns; lane k works on column s-k+1 at
//   step s (an anti-diagonal wavefront), so the row above a lane's top row was
//   produced by lane k-1 one step earlier and arrives by __shfl_up_sync.  A
//   read longer than one strip runs strip after strip; the bottom row of a
//   strip goes through a per-warp global buffer, streamed through shared
//   memory in 32-column chunks with cp.async.
// * Rows are padded at the TOP of the first strip with rows whose transition
//   coefficients are zero, so the read's last row always sits in lane 31's
//   bottom register and row 0 (the initial row) is an ordinary row with
//   Y = INITIAL/haplen carried unchanged.
// * X and Y are kept divided by their row's pMX / pMY:
//       Xh(r,c) = X(r,c)/pMX(r) = Xh(r-1,c) * pXX(r) pMX(r-1)/pMX(r) + M(r-1,c)
//       Yh(r,c) = Y(r,c)/pMY(r) = Yh(r,c-1) * pYY(r) + M(r,c-1)
//   so each costs one FMA, and M costs FMUL + 2 FMA + FMUL: six FP32
//   instructions per cell instead of the reference's twelve flops.
// * Folded form (the default): pMM(r) is folded into row r's emission table
//   and cx, cy carry 1/pMM, so M costs 2 FMA + FMUL: five instructions per
//   cell.  A strip with a row whose pMM is below kFoldMin keeps the six-
//   instruction form (phmm_device.cuh, setup_rows).
// * Constant transitions (the scalar PairHMM model) take the seven
//   probabilities from the table instead of the quality bytes.
// * The emission e(r,c) is read from a per-lane shared-memory table indexed by
//   the haplotype code of the column: one 16-byte load yields four rows' e.
//   Columns outside the haplotype have code 5 and e = 0, which makes the
//   wavefront's ramp-up and ramp-down reproduce the DP boundary exactly.
// * Pairs whose FP32 result is below MIN_ACCEPTED (1e-28, pairhmm_common.h:16)
//   or not finite are appended to a list that the FP64 kernel recomputes, as
//   AvxPairHMM::computeLikelihoodsNative does (pairhmm_avx.hpp:140-149).  The
//   FP64 kernel renormalises the strip boundary row by an exact power of two
//   so reads of many kilobases stay finite.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>
#include <cstdint>
#include <cmath>

#include "phmm_common.h"
#include "phmm_device.cuh"
#include "phmm_kernels.h"

namespace bvphmm {

// A kernel's dynamic shared-memory limit is one value per function and
// device, shared by every context of the process.  Contexts that plan
// different haplotype lengths (several on one GPU, from different host
// threads) would otherwise lower it under each other's launches, so the
// limit only ever rises: a process-wide record of each (device, kernel)'s
// current limit, under a lock.
cudaError_t raise_dynamic_smem(const void* func, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> limit;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  int& cur = limit[{dev, func}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

template <typename T, int RT, bool MULTI, bool PAIR>
__global__ void __launch_bounds__(kThreadsPerBlock) k_forward(KernelParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & (kWarp - 1);
  const int wib = threadIdx.x >> 5;
  const int warp_global = blockIdx.x * p.warps_per_block + wib;
  unsigned char* wsm = smem + (size_t)wib * p.warp_smem_bytes;
  T* bnd = MULTI ? reinterpret_cast<T*>(p.bnd) + (size_t)warp_global * p.bnd_cols * 4 : nullptr;
  // only the FP64 variants drain the FP64 list
  constexpr bool kList = sizeof(T) == 8;
  const bool from_list = kList && p.from_rescue;
  const unsigned long long n = from_list ? p.ctr->rescue_count
                               : p.n_units_dev ? *p.n_units_dev : (unsigned long long)p.n_units;
  const unsigned long long n_short = from_list && n > (unsigned long long)p.rescue_cap ? p.rescue_cap : n;
  // FP64 pass: after the short list, the long list's entries the long-read
  // kernel handed back (read index complemented)
  const unsigned long long n_long =
      from_list && p.long_rows > 0 ? min(p.ctr->rescue_long_count, (unsigned long long)p.rescue_cap) : 0ull;
  const unsigned long long n_eff = n_short + n_long;
  unsigned long long* next = from_list ? &p.ctr->rescue_next : &p.ctr->unit_next[p.slot];
  for (;;) {
    unsigned long long w = 0;
    if (lane == 0) w = atomicAdd(next, 1ull);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= n_eff) break;
    Item it;
    long long handed_back = -1;  // list slot of an entry the long-read kernel handed back
    if (kList && from_list) {
      PairRef pr;
      if (w < n_short) {
        pr = p.rescue[w];
      } else {
        handed_back = p.rescue_cap - 1 - (long long)(w - n_short);
        pr = p.rescue[handed_back];
        if (pr.read >= 0) continue;  // scored by the long-read kernel
        pr.read = ~pr.read;
      }
      it.read = pr.read; it.hap0 = pr.hap; it.nh = 1; it.out0 = pr.out;
    } else {
      const Unit u = p.units[p.unit_base + w];
      it.read = u.read; it.hap0 = u.hap0; it.nh = u.nh; it.out0 = u.out0;
    }
    process_item<T, RT, MULTI, PAIR>(p, it, wsm, lane, bnd);
    // the mark is cleared: a replayed batch finds the list as it was staged
    if (kList && handed_back >= 0 && lane == 0) p.rescue[handed_back].read = it.read;
  }
}

// Packs the four quality arrays into one uchar4 per read position.
__global__ void k_pack_quals(const uint8_t* __restrict__ q, const uint8_t* __restrict__ i,
                             const uint8_t* __restrict__ d, const uint8_t* __restrict__ c,
                             uchar4* __restrict__ out, long long n) {
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x)
    out[x] = make_uchar4(q[x], i[x], d[x], c[x]);
}

__global__ void k_pack_quals_uniform(const uint8_t* __restrict__ q, uint8_t gi, uint8_t gd, uint8_t gc,
                                     uchar4* __restrict__ out, long long n) {
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x)
    out[x] = make_uchar4(q[x], gi, gd, gc);
}

__global__ void k_set_u64(unsigned long long* dst, unsigned long long v) { *dst = v; }

cudaError_t launch_set_u64(unsigned long long* dst, unsigned long long v, cudaStream_t st) {
  k_set_u64<<<1, 1, 0, st>>>(dst, v);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Host-side launch table
// ---------------------------------------------------------------------------
template <typename T, int RT, bool MULTI, bool PAIR>
int warp_smem_bytes_for(int hap_bytes) {
  using S = WarpSmem<T, RT>;
  return hap_bytes + S::kEtabBytes + (MULTI ? S::kRingBytes : 0);
}

template <typename T, int RT, bool MULTI, bool PAIR>
static cudaError_t launch_one(const KernelParams& p, int grid, cudaStream_t st) {
  const int smem = p.warps_per_block * p.warp_smem_bytes;
  k_forward<T, RT, MULTI, PAIR><<<grid, p.warps_per_block * kWarp, smem, st>>>(p);
  return cudaGetLastError();
}

template <typename T, int RT, bool MULTI, bool PAIR>
static cudaError_t prepare_one(int smem_per_block) {
  return raise_dynamic_smem(reinterpret_cast<const void*>(&k_forward<T, RT, MULTI, PAIR>), smem_per_block);
}

template <typename T, int RT, bool MULTI, bool PAIR>
static int occupancy_one(int smem_per_block, int threads) {
  int nb = 0;
  auto k = &k_forward<T, RT, MULTI, PAIR>;
  if (raise_dynamic_smem(reinterpret_cast<const void*>(k), smem_per_block) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, threads, smem_per_block) != cudaSuccess) return 0;
  return nb;
}

// Variant order: indices 0..7 are FP32 single strip with 1..8 rows per lane
// and 8 the FP32 multi-strip variant (the band path's fallback buckets use
// these numbers); then the FP64 variants and the paired FP32 variants.
#define BV_VARIANTS(X)              \
  X(float, 1, false, false) X(float, 2, false, false) X(float, 3, false, false) X(float, 4, false, false) \
  X(float, 5, false, false) X(float, 6, false, false) X(float, 7, false, false) X(float, 8, false, false) \
  X(float, 8, true, false) X(double, 4, true, false) X(double, 2, true, false)                           \
  X(float, 1, false, true) X(float, 2, false, true) X(float, 3, false, true) X(float, 4, false, true)     \
  X(float, 5, false, true) X(float, 6, false, true) X(float, 7, false, true) X(float, 8, false, true)

int variant_index(bool f64, int rt, bool multi, bool paired) {
  int idx = 0;
#define BV_IDX(T, RT, MULTI, PAIR)                                                                 \
  if ((sizeof(T) == 8) == f64 && RT == rt && MULTI == multi && PAIR == paired) return idx; \
  ++idx;
  BV_VARIANTS(BV_IDX)
#undef BV_IDX
  return -1;
}

bool variant_paired(int variant) {
  int idx = 0;
#define BV_PAIRED(T, RT, MULTI, PAIR) \
  if (idx++ == variant) return PAIR;
  BV_VARIANTS(BV_PAIRED)
#undef BV_PAIRED
  return false;
}

int warp_smem_bytes(int variant, int hap_bytes) {
  int idx = 0;
#define BV_SM(T, RT, MULTI, PAIR) \
  if (idx++ == variant) return warp_smem_bytes_for<T, RT, MULTI, PAIR>(hap_bytes);
  BV_VARIANTS(BV_SM)
#undef BV_SM
  return -1;
}

cudaError_t prepare_variant(int variant, int smem_per_block) {
  int idx = 0;
#define BV_PREP(T, RT, MULTI, PAIR) \
  if (idx++ == variant) return prepare_one<T, RT, MULTI, PAIR>(smem_per_block);
  BV_VARIANTS(BV_PREP)
#undef BV_PREP
  return cudaErrorInvalidValue;
}

cudaError_t launch_forward(int variant, const KernelParams& p, int grid, cudaStream_t st) {
  int idx = 0;
#define BV_LAUNCH(T, RT, MULTI, PAIR) \
  if (idx++ == variant) return launch_one<T, RT, MULTI, PAIR>(p, grid, st);
  BV_VARIANTS(BV_LAUNCH)
#undef BV_LAUNCH
  return cudaErrorInvalidValue;
}

int blocks_per_sm(int variant, int smem_per_block, int threads) {
  int idx = 0;
#define BV_OCC(T, RT, MULTI, PAIR) \
  if (idx++ == variant) return occupancy_one<T, RT, MULTI, PAIR>(smem_per_block, threads);
  BV_VARIANTS(BV_OCC)
#undef BV_OCC
  return 0;
}

cudaError_t launch_pack_quals(const uint8_t* q, const uint8_t* i, const uint8_t* d, const uint8_t* c, uchar4* out,
                              long long n, int sms, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  long long blocks = (n + 255) / 256;
  if (blocks > (long long)sms * 8) blocks = (long long)sms * 8;
  k_pack_quals<<<(int)blocks, 256, 0, st>>>(q, i, d, c, out, n);
  return cudaGetLastError();
}

cudaError_t launch_pack_quals_uniform(const uint8_t* q, uint8_t gi, uint8_t gd, uint8_t gc, uchar4* out, long long n,
                                      int sms, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  long long blocks = (n + 255) / 256;
  if (blocks > (long long)sms * 8) blocks = (long long)sms * 8;
  k_pack_quals_uniform<<<(int)blocks, 256, 0, st>>>(q, gi, gd, gc, out, n);
  return cudaGetLastError();
}

}  // namespace bvphmm
