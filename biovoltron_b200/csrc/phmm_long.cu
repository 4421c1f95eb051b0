// phmm_long.cu -- FP64 forward pass of long reads, several warps per pair.
//
// The FP64 pass (the rescue of pairs whose FP32 result falls below 1e-28, or
// every pair in FP64 mode) runs a long read strip after strip: strip s holds
// read rows [128 s, 128 s + 128) (4 rows per lane).  With one warp per pair
// the strips run one after the other and the longest pair sets the launch
// time; here a block of kLongWarps warps takes one pair and warp w runs
// strips w, w + K, w + 2K, ... as a pipelined wavefront: strip s + 1 starts a
// 32-column chunk as soon as strip s has finished the next one.
//
// Strip boundaries.  Inside a group of K consecutive strips (one per warp) a
// strip's bottom row goes to the next warp through a shared-memory channel of
// kLongSlots chunk slots; a slot's mbarriers say "full" (the producer's lane
// 31 arrives after writing the chunk) and "empty" (the consumer's lane 0
// arrives after reading it).  Between groups the bottom row goes through the
// block's global boundary buffer, read back by the next group's first strip
// with bulk (TMA) copies as in the one-warp kernel, and renormalised: the
// row's maximum is scaled to 2^target by an exact power of two, the exponent
// carried to the result.  So the values of a group share one scale and may
// shrink over its 128 K rows before the next renormalisation (the one-warp
// kernel renormalises every 128 rows).
//
// A pair whose group-end row maximum falls below 2^kLongMinExp, or whose
// result is not a positive finite number, is handed back to the one-warp FP64
// kernel (its list entry marked), which runs after this one.
//
// The haplotype codes are staged once per pair for all warps.  Every wait is
// bounded (status bit 8 when one gives up); after the first wait of a block
// that gives up the others are skipped, so a broken hand-over ends after one
// time-out.  Single-GPU kernel: the bulk copies read this GPU's own memory,
// without multicast.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "phmm_device.cuh"
#include "phmm_kernels.h"

namespace bvphmm {
namespace {

constexpr int kLongRT = 4;     // rows per lane (FP64)
// a group whose last row's maximum is below 2^kLongMinExp (relative to the
// 2^1000 its first row started from, more than 1,600 binary orders) hands the
// pair back: the one-warp kernel renormalises every 128 rows instead of 512
constexpr int kLongMinExp = -600;
constexpr int kLongSlots = 4;  // chunk slots per channel
using LS = WarpSmem<double, kLongRT>;
constexpr int kColB = LS::kColBytes;  // bytes per boundary column (M, X, Y, unused)
constexpr int kChunkB = 32 * kColB;   // one 32-column chunk

// Dynamic shared memory of a block of K warps, after the staged haplotype
// codes (hap_bytes, a multiple of 16):
//   per warp: emission table, 32-column output staging (global output)
//   warp 0:   64-column input ring (global input)
//   channels 0 .. K-2: kLongSlots chunks each
//   barriers: full / empty per channel slot, the group-done barrier, the two
//   input-ring halves; then the shared scalars.
template <int K>
struct LongLayout {
  static constexpr int kWarpBytes = LS::kEtabBytes + kChunkB;
  static constexpr int kRingIn = K * kWarpBytes;
  static constexpr int kChan = kRingIn + 2 * kChunkB;
  static constexpr int kBars = kChan + (K - 1) * kLongSlots * kChunkB;
  static constexpr int kNumBars = 2 * (K - 1) * kLongSlots + 3;
  static constexpr int kScalars = kBars + 8 * kNumBars;
  static constexpr int kBytes = kScalars + 64;
};

struct LongShared {  // at LongLayout::kScalars
  double grp_max;    // the last group-end row's maximum (in its own scale)
  long long kexp;    // current group's exponent: stored values are true values * 2^-kexp
  long long item;
  int fail;
  int redo;          // the pair goes back to the one-warp FP64 kernel
};

struct LongIO {
  int in_mode, out_mode;  // warp-uniform
  const double* chin;
  uint64_t* in_full;
  uint64_t* in_empty;
  double* chout;
  uint64_t* out_full;
  uint64_t* out_empty;
  double* bnd;
  double* ring_in;
  uint64_t* ring_mb;
  double* ring_out;
  double in_scale, in_scale2;  // the group-start renormalisation, as two exact power-of-two factors
};
constexpr int kInZero = 0, kInChan = 1, kInGlobal = 2;
constexpr int kOutNone = 0, kOutChan = 1, kOutGlobal = 2;

__device__ __forceinline__ void mbar_arrive(uint64_t* mb) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(mb)) : "memory");
}
// Waits for the barrier's phase of parity ((bits >> i) & 1) and flips that
// bit.  Once any wait of the block has given up (*fail), waits are skipped.
__device__ __forceinline__ bool wait_flip(uint64_t* mb, unsigned& bits, int i, volatile int* fail) {
  bool ok = true;
  if (!*fail) {
    ok = mbar_wait(mb, (bits >> i) & 1u);
    if (!ok) *fail = 1;
  }
  bits ^= 1u << i;
  return ok;
}

// One FP64 strip of a long pair (the one-warp kernel's run_strip with the
// boundary row taken from, and given to, the modes of `io`).  Column c of a
// boundary row is row c + 31 of the boundary space: chunk j of a producer
// (steps 32j .. 32j+31 of lane 31) holds rows 32j+1 .. 32j+32 (slot entry u:
// step 32j+u); at step s lane 0 reads row s + 32, its diagonal starts at row
// 31.  fph (lane 0) and eph (lane 31) are the parities of the channel
// barriers' next phases; ok turns false when a wait gives up.
template <int RT>
__device__ __forceinline__ void run_strip_long(const Rows<double, RT>& rw, const ELane el,
                                               const unsigned char* __restrict__ hc_lane, int nsteps, int lane,
                                               const LongIO& io, unsigned& fph, unsigned& eph, double& sumM,
                                               double& sumX, double& bmax, bool& ok, volatile int* fail) {
  using T = double;
  T M[RT], X[RT], Y[RT];
#pragma unroll
  for (int j = 0; j < RT; ++j) { M[j] = T(0); X[j] = T(0); Y[j] = rw.y0[j]; }
  sumM = T(0); sumX = T(0); bmax = T(0);
  T upM = __shfl_up_sync(0xffffffffu, M[RT - 1], 1);
  T upX = __shfl_up_sync(0xffffffffu, X[RT - 1], 1);
  T upY = __shfl_up_sync(0xffffffffu, Y[RT - 1], 1);
  T dM = upM, dX = upX, dY = upY;
  const int nch = nsteps / 32;
  unsigned rphase = 0;  // lane 0, global input: parity bits of the two ring halves
  if (lane == 0) {
    if (io.in_mode == kInZero) {
      dM = dX = dY = T(0);
    } else if (io.in_mode == kInChan) {
      ok &= wait_flip(io.in_full, fph, 0, fail);
      if (nch > 1) ok &= wait_flip(io.in_full + 1, fph, 1, fail);
      const T* r31 = io.chin + 30 * 4;  // row 31 = chunk 0, entry 30
      dM = r31[0]; dX = r31[1]; dY = r31[2];
    }
  }
  if (io.in_mode == kInGlobal) {
    fence_for_bulk();
    __syncwarp();
    if (lane == 0) {
      mbar_init(io.ring_mb, 1);
      mbar_init(io.ring_mb + 1, 1);
      fence_for_bulk();
      bulk_g2s(io.ring_in, io.bnd + (size_t)32 * 4, kChunkB, io.ring_mb);
      dM = io.bnd[31 * 4 + 0] * io.in_scale * io.in_scale2;
      dX = io.bnd[31 * 4 + 1] * io.in_scale * io.in_scale2;
      dY = io.bnd[31 * 4 + 2] * io.in_scale * io.in_scale2;
      if (!*fail && !mbar_wait(io.ring_mb, 0)) { ok = false; *fail = 1; }
      rphase ^= 1u;
    }
    __syncwarp();
  }
  for (int k = 0; k < nch; ++k) {
    const int s0 = 32 * k;
    if (lane == 0) {
      if (io.in_mode == kInChan && k >= 1 && k + 1 < nch)
        ok &= wait_flip(io.in_full + (k + 1) % kLongSlots, fph, (k + 1) % kLongSlots, fail);
      if (io.in_mode == kInGlobal)
        bulk_g2s(io.ring_in + ((k + 1) & 1) * 32 * 4, io.bnd + (size_t)(32 * (k + 1) + 32) * 4, kChunkB,
                 io.ring_mb + ((k + 1) & 1));
    }
    if (lane == kWarp - 1 && io.out_mode == kOutChan)
      ok &= wait_flip(io.out_empty + k % kLongSlots, eph, k % kLongSlots, fail);
    const T* cur = io.chin + (k % kLongSlots) * 32 * 4;
    const T* nxt = io.chin + ((k + 1) % kLongSlots) * 32 * 4;
    T* out_slot = io.chout + (k % kLongSlots) * 32 * 4;
#pragma unroll 8  // a fully unrolled chunk (32 steps, five I/O modes) overflows the instruction cache
    for (int u = 0; u < 32; ++u) {
      if (lane == 0) {
        if (io.in_mode == kInChan) {
          if (u == 0) { upM = cur[31 * 4]; upX = cur[31 * 4 + 1]; upY = cur[31 * 4 + 2]; }
          else if (k + 1 < nch) { upM = nxt[(u - 1) * 4]; upX = nxt[(u - 1) * 4 + 1]; upY = nxt[(u - 1) * 4 + 2]; }
          else { upM = T(0); upX = T(0); upY = T(0); }
        } else if (io.in_mode == kInGlobal) {
          const T* rin = io.ring_in + ((k & 1) * 32 + u) * 4;
          upM = rin[0] * io.in_scale * io.in_scale2;
          upX = rin[1] * io.in_scale * io.in_scale2;
          upY = rin[2] * io.in_scale * io.in_scale2;
        } else {
          upM = T(0); upX = T(0); upY = T(0);
        }
      }
      T e[RT];
      load_emissions<T, RT>(el, (unsigned)hc_lane[s0 + u] * LS::kCodeStride, e);
      T um = upM, ux = upX;
      T dm = dM, dx = dX, dy = dY;
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        const T mn = e[j] * fma_(rw.mm[j], dm, fma_(rw.cx[j], dx, rw.cy[j] * dy));
        const T xn = fma_(rw.gx[j], ux, rw.kap[j] * um);
        const T yn = fma_(rw.g[j], Y[j], rw.my[j] * M[j]);
        dm = M[j]; dx = X[j]; dy = Y[j];
        um = mn; ux = xn;
        M[j] = mn; X[j] = xn; Y[j] = yn;
      }
      sumM += M[RT - 1];
      sumX += X[RT - 1];
      const T nM = __shfl_up_sync(0xffffffffu, M[RT - 1], 1);
      const T nX = __shfl_up_sync(0xffffffffu, X[RT - 1], 1);
      const T nY = __shfl_up_sync(0xffffffffu, Y[RT - 1], 1);
      if (lane == kWarp - 1) {
        if (io.out_mode == kOutChan) {
          T* o = out_slot + u * 4;
          o[0] = M[RT - 1]; o[1] = X[RT - 1]; o[2] = Y[RT - 1];
        } else if (io.out_mode == kOutGlobal) {
          T* o = io.ring_out + u * 4;
          o[0] = M[RT - 1]; o[1] = X[RT - 1]; o[2] = Y[RT - 1];
          bmax = fmax(bmax, fmax(M[RT - 1], fmax(X[RT - 1], Y[RT - 1])));
        }
      }
      dM = upM; dX = upX; dY = upY;
      upM = nM; upX = nX; upY = nY;
    }
    // end of chunk k
    if (lane == kWarp - 1 && io.out_mode == kOutChan) mbar_arrive(io.out_full + k % kLongSlots);
    if (lane == 0 && io.in_mode == kInChan) mbar_arrive(io.in_empty + k % kLongSlots);
    if (io.out_mode == kOutGlobal) {
      __syncwarp();
      T* dstb = io.bnd + (size_t)(s0 + 1 + lane) * 4;
      const T* srco = io.ring_out + lane * 4;
      reinterpret_cast<double2*>(dstb)[0] = reinterpret_cast<const double2*>(srco)[0];
      reinterpret_cast<double2*>(dstb)[1] = reinterpret_cast<const double2*>(srco)[1];
      __syncwarp();
    }
    if (io.in_mode == kInGlobal) {
      if (lane == 0) {
        const int h = (k + 1) & 1;
        if (!*fail && !mbar_wait(io.ring_mb + h, (rphase >> h) & 1u)) { ok = false; *fail = 1; }
        rphase ^= 1u << h;
      }
      __syncwarp();
    }
  }
  if (io.in_mode == kInGlobal && lane == 0 && ok) {
    mbar_inval(io.ring_mb);
    mbar_inval(io.ring_mb + 1);
  }
  __syncwarp();
}

// One block of K warps per long pair (the FP64 list's long part, read from
// the list's far end).
template <int K>
__global__ void __launch_bounds__(K * kWarp) k_forward_long(KernelParams p) {
  using L = LongLayout<K>;
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & (kWarp - 1), w = threadIdx.x >> 5;
  unsigned char* hc = smem;
  unsigned char* base = smem + p.hap_bytes;
  unsigned char* etab = base + w * L::kWarpBytes;
  const ELane el = elane<double, kLongRT>(etab, lane);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + L::kBars);
  uint64_t* full = bars;                                 // [(K-1) * slots]
  uint64_t* empty = bars + (K - 1) * kLongSlots;         // [(K-1) * slots]
  uint64_t* grp_done = bars + 2 * (K - 1) * kLongSlots;  // group-end row written
  LongShared& sh = *reinterpret_cast<LongShared*>(base + L::kScalars);
  double* bnd = reinterpret_cast<double*>(p.bnd) + (size_t)blockIdx.x * p.bnd_cols * 4;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2 * (K - 1) * kLongSlots + 1; ++i) mbar_init(bars + i, 1);
    sh.fail = 0;
  }
  fence_for_bulk();
  __syncthreads();
  LongIO io{};
  io.chin = w >= 1 ? reinterpret_cast<const double*>(base + L::kChan + (w - 1) * kLongSlots * kChunkB) : nullptr;
  io.in_full = w >= 1 ? full + (w - 1) * kLongSlots : nullptr;
  io.in_empty = w >= 1 ? empty + (w - 1) * kLongSlots : nullptr;
  io.chout = w + 1 < K ? reinterpret_cast<double*>(base + L::kChan + w * kLongSlots * kChunkB) : nullptr;
  io.out_full = w + 1 < K ? full + w * kLongSlots : nullptr;
  io.out_empty = w + 1 < K ? empty + w * kLongSlots : nullptr;
  io.bnd = bnd;
  io.ring_in = reinterpret_cast<double*>(base + L::kRingIn);
  io.ring_mb = grp_done + 1;
  io.ring_out = reinterpret_cast<double*>(etab + LS::kEtabBytes);
  unsigned fph = 0;                        // lane 0: input channel slots' next full phases
  unsigned eph = (1u << kLongSlots) - 1u;  // lane 31: output slots; their first wait passes at once
  unsigned gph = 0;                        // warp 0, lane 0: group-done barrier
  bool ok = true;
  volatile int* fail = &sh.fail;
  const DeviceBatch& b = p.batch;
  const unsigned long long n_long = min(p.ctr->rescue_long_count, (unsigned long long)p.rescue_cap);
  for (;;) {
    if (threadIdx.x == 0) sh.item = (long long)atomicAdd(&p.ctr->rescue_long_next, 1ull);
    __syncthreads();
    const long long wi = sh.item;
    if (wi >= (long long)n_long || *fail) break;
    const PairRef pr = p.rescue[p.rescue_cap - 1 - wi];
    const int64_t ro = b.read_off[pr.read], ho = b.hap_off[pr.hap];
    const int R = (int)(b.read_off[pr.read + 1] - ro), H = (int)(b.hap_off[pr.hap + 1] - ho);
    const uchar4* quals = b.read_quals + ro;
    const uint8_t* bases = b.read_bases + ro;
    if (H == 0 || R == 0) {
      if (threadIdx.x == 0) p.out[pr.out] = -INFINITY;
      __syncthreads();
      continue;
    }
    const double init_y = p.tables->init_d / (double)H;
    const int nsteps = (H + kWarp - 1 + 31) / 32 * 32;
    const int rows = R + 1;
    const int nstrips = (rows + 32 * kLongRT - 1) / (32 * kLongRT);
    const int pad = nstrips * 32 * kLongRT - rows;
    stage_hap_block(b.hap_bases + ho, H, hc, nsteps + kHapLead);
    // boundary rows past the last column, read as zeros by a group's first strip
    for (int x = threadIdx.x; x < 96; x += blockDim.x) {
      double* r = bnd + (size_t)(nsteps + 1 + x) * 4;
      r[0] = 0.0; r[1] = 0.0; r[2] = 0.0;
    }
    fence_for_bulk();  // those rows are read by bulk copies
    if (threadIdx.x == 0) {
      sh.kexp = 0;
      sh.redo = 0;
    }
    __syncthreads();
    for (int s = w; s < nstrips; s += K) {
      Rows<double, kLongRT> rw;
      setup_rows<double, kLongRT>(p.tables, quals, bases, R, s * 32 * kLongRT + lane * kLongRT - pad, init_y, rw,
                                  etab, lane);
      __syncwarp();
      io.in_mode = s == 0 ? kInZero : (s % K == 0 ? kInGlobal : kInChan);
      io.out_mode = s == nstrips - 1 ? kOutNone : (s % K == K - 1 ? kOutGlobal : kOutChan);
      io.in_scale = 1.0;
      io.in_scale2 = 1.0;
      if (io.in_mode == kInGlobal) {
        // renormalise: the previous group's last row, maximum scaled to 2^target
        // (a factor up to 2^2074 does not fit one double: two factors, each exact)
        double m = 0.0;
        if (lane == 0) {
          ok &= wait_flip(grp_done, gph, 0, fail);
          m = sh.grp_max;
        }
        m = __shfl_sync(0xffffffffu, m, 0);
        if (m > 0.0) {
          int e2;
          frexp(m, &e2);
          const int shift = e2 - p.rescale_target;
          const int a = min(-shift, 1023), b2 = min(-shift - a, 1023);
          io.in_scale = ldexp(1.0, a);
          io.in_scale2 = ldexp(1.0, b2);
          if (lane == 0) sh.kexp += shift;
          // the group fell far below the one-warp kernel's per-strip range: that kernel redoes the pair
          if (lane == 0 && e2 < kLongMinExp) sh.redo = 1;
        } else if (lane == 0) {
          sh.redo = 1;
        }
        __syncwarp();
      }
      double sumM, sumX, bmax;
      run_strip_long<kLongRT>(rw, el, hc + kHapLead - lane, nsteps, lane, io, fph, eph, sumM, sumX, bmax, ok, fail);
      if (io.out_mode == kOutGlobal) {
        fence_for_bulk();  // the rows just written are read by bulk copies
        __syncwarp();
        if (lane == kWarp - 1) sh.grp_max = bmax;
        __syncwarp();
        if (lane == 0) mbar_arrive(grp_done);
      }
      if (s == nstrips - 1 && lane == kWarp - 1) {
        const double res = sumM + sumX;
        if (sh.redo || !(res > 0.0 && isfinite(res))) {
          sh.redo = 1;
        } else {
          write_result<double>(p, pr.read, pr.hap, pr.out, res, sh.kexp);
          if (p.cells_ctr) atomicAdd(p.cells_ctr, (unsigned long long)R * (unsigned long long)H);
        }
      }
    }
    __syncthreads();
    // handed back: the entry is marked (read index complemented) for the one-warp FP64 kernel
    if (threadIdx.x == 0 && sh.redo) p.rescue[p.rescue_cap - 1 - wi].read = ~pr.read;
  }
  if (!ok) atomicOr(&p.ctr->status, 8ull);
}

}  // namespace

// The kernel for `warps` warps per pair (2, 4 or 8; long_warps_valid).
namespace {
template <int K>
int smem_for(int hap_bytes) { return hap_bytes + LongLayout<K>::kBytes; }
template <int K>
int blocks_for(int smem) {
  int nb = 0;
  if (raise_dynamic_smem(reinterpret_cast<const void*>(&k_forward_long<K>), smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_forward_long<K>, K * kWarp, smem) != cudaSuccess) return 0;
  return nb;
}
}  // namespace

bool long_warps_valid(int warps) { return warps == 2 || warps == 4 || warps == 8; }

int long_smem_bytes(int hap_bytes, int warps) {
  return warps == 2 ? smem_for<2>(hap_bytes) : warps == 8 ? smem_for<8>(hap_bytes) : smem_for<4>(hap_bytes);
}

cudaError_t prepare_long(int smem, int warps) {
  const void* f = warps == 2   ? reinterpret_cast<const void*>(&k_forward_long<2>)
                  : warps == 8 ? reinterpret_cast<const void*>(&k_forward_long<8>)
                               : reinterpret_cast<const void*>(&k_forward_long<4>);
  return raise_dynamic_smem(f, smem);
}

int long_blocks_per_sm(int smem, int warps) {
  return warps == 2 ? blocks_for<2>(smem) : warps == 8 ? blocks_for<8>(smem) : blocks_for<4>(smem);
}

cudaError_t launch_forward_long(const KernelParams& p, int grid, int smem, int warps, cudaStream_t st) {
  if (warps == 2) k_forward_long<2><<<grid, 2 * kWarp, smem, st>>>(p);
  else if (warps == 8) k_forward_long<8><<<grid, 8 * kWarp, smem, st>>>(p);
  else k_forward_long<4><<<grid, 4 * kWarp, smem, st>>>(p);
  return cudaGetLastError();
}

}  // namespace bvphmm
