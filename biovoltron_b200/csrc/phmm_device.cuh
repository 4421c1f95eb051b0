// phmm_device.cuh -- device-side building blocks of the PairHMM forward
// kernels (row set-up, emission table, haplotype staging, the wavefront strip
// and the per-item driver).  The formulation is described at the top of
// phmm_forward.cu, which instantiates the kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>
#include <type_traits>

#include "phmm_common.h"
#include "phmm_kernels.h"
#include "phmm_rows.h"

namespace bvphmm {


// Shared-memory loads written in PTX (full vector width).
__device__ __forceinline__ float4 lds4f(const unsigned char* p) {
  float4 v;
  asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "r"((unsigned)__cvta_generic_to_shared(p)));
  return v;
}
__device__ __forceinline__ float2 lds2f(const unsigned char* p) {
  float2 v;
  asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"((unsigned)__cvta_generic_to_shared(p)));
  return v;
}
__device__ __forceinline__ double2 lds2d(const unsigned char* p) {
  double2 v;
  asm("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"((unsigned)__cvta_generic_to_shared(p)));
  return v;
}

// Emission table of one warp.  For each haplotype code, a block of
// 32 * RT values: every lane's RT rows, split into chunks of Wm = 16 /
// sizeof(T) rows (4 FP32, 2 FP64) and, for the remainder, one chunk of 2
// and/or one of 1 row.  Chunk region r of width w holds lane l's rows at
// region + l * w * sizeof(T), so one load per chunk covers 32 * w
// consecutive words: bank-conflict free, and a lookup of all RT rows moves
// exactly RT * 128 bytes (RT shared-memory wavefronts for FP32).
template <typename T, int RT>
struct ETab {
  static constexpr int Wm = 16 / (int)sizeof(T);
  static constexpr int NF = RT / Wm;                                   // full-width chunks
  static constexpr bool kHalf = Wm == 4 && (RT % Wm) >= 2;            // FP32 only: a 2-row chunk
  static constexpr bool kOne = (RT % 2) == 1;                          // a 1-row chunk
  static constexpr int kOffHalf = NF * kWarp * 16;
  static constexpr int kOffOne = kOffHalf + (kHalf ? kWarp * 2 * (int)sizeof(T) : 0);
  static constexpr int kCodeStride = kWarp * RT * (int)sizeof(T);
  static constexpr int kBytes = kCodes * kCodeStride;
  static_assert(NF * Wm + (kHalf ? 2 : 0) + (kOne ? 1 : 0) == RT, "chunking covers the rows");
};

// A lane's three chunk bases in the warp's table.
struct ELane {
  const unsigned char* full;
  const unsigned char* half;
  const unsigned char* one;
};

template <typename T, int RT>
__device__ __forceinline__ ELane elane(const unsigned char* etab, int lane) {
  using E = ETab<T, RT>;
  return ELane{etab + lane * 16, etab + E::kOffHalf + lane * 2 * (int)sizeof(T),
               etab + E::kOffOne + lane * (int)sizeof(T)};
}

// Loads the lane's RT emissions for the code whose block starts at `off`.
template <typename T, int RT>
__device__ __forceinline__ void load_emissions(const ELane& el, unsigned off, T* e) {
  using E = ETab<T, RT>;
#pragma unroll
  for (int ch = 0; ch < E::NF; ++ch) {
    if constexpr (sizeof(T) == 4) {
      const float4 v = lds4f(el.full + off + ch * kWarp * 16);
      e[4 * ch] = v.x; e[4 * ch + 1] = v.y; e[4 * ch + 2] = v.z; e[4 * ch + 3] = v.w;
    } else {
      const double2 v = lds2d(el.full + off + ch * kWarp * 16);
      e[2 * ch] = v.x; e[2 * ch + 1] = v.y;
    }
  }
  if constexpr (E::kHalf) {
    const float2 v = lds2f(el.half + off);
    e[E::NF * 4] = v.x; e[E::NF * 4 + 1] = v.y;
  }
  if constexpr (E::kOne) {
    e[RT - 1] = *reinterpret_cast<const T*>(el.one + off);
  }
}

// Stores the lane's RT emissions of one code (set-up).
template <typename T, int RT>
__device__ __forceinline__ void store_emissions(unsigned char* etab, int lane, int code, const T* v) {
  using E = ETab<T, RT>;
  unsigned char* blk = etab + code * E::kCodeStride;
#pragma unroll
  for (int ch = 0; ch < E::NF; ++ch) {
    if constexpr (sizeof(T) == 4) {
      *reinterpret_cast<float4*>(blk + ch * kWarp * 16 + lane * 16) =
          make_float4(v[4 * ch], v[4 * ch + 1], v[4 * ch + 2], v[4 * ch + 3]);
    } else {
      *reinterpret_cast<double2*>(blk + ch * kWarp * 16 + lane * 16) = make_double2(v[2 * ch], v[2 * ch + 1]);
    }
  }
  if constexpr (E::kHalf) {
    *reinterpret_cast<float2*>(blk + E::kOffHalf + lane * 8) = make_float2(v[E::NF * 4], v[E::NF * 4 + 1]);
  }
  if constexpr (E::kOne) {
    *reinterpret_cast<T*>(blk + E::kOffOne + lane * (int)sizeof(T)) = v[RT - 1];
  }
}

__device__ __forceinline__ float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T> __device__ __forceinline__ const T* ph2pr_tab(const Tables* t);
template <> __device__ __forceinline__ const float* ph2pr_tab<float>(const Tables* t) { return t->ph2pr_f; }
template <> __device__ __forceinline__ const double* ph2pr_tab<double>(const Tables* t) { return t->ph2pr_d; }
template <typename T> __device__ __forceinline__ const T* mm_tab(const Tables* t);
template <> __device__ __forceinline__ const float* mm_tab<float>(const Tables* t) { return t->mm_f; }
template <> __device__ __forceinline__ const double* mm_tab<double>(const Tables* t) { return t->mm_d; }

__device__ __forceinline__ uint32_t base_code(uint32_t b) {
  // ConvertChar (pairhmm_common.h:26-44): A0 C1 T2 G3 N4, anything else 0.
  return b == 'C' ? 1u : b == 'T' ? 2u : b == 'G' ? 3u : b == 'N' ? 4u : 0u;
}

__device__ __forceinline__ int mm_index(int ins, int del) {
  const int mx = ins > del ? ins : del;
  const int mn = ins > del ? del : ins;
  return ((mx * (mx + 1)) >> 1) + mn;
}

// Shared-memory layout of one warp's slice.
template <typename T, int RT>
struct WarpSmem {
  static constexpr int kCodeStride = ETab<T, RT>::kCodeStride;  // bytes per code
  static constexpr int kEtabBytes = ETab<T, RT>::kBytes;
  static constexpr int kRingInCols = 64;
  static constexpr int kRingOutCols = 32;
  static constexpr int kColBytes = 4 * (int)sizeof(T);     // M, Xh, Yh, unused
  // the two input-ring halves' transaction barriers follow the rings
  static constexpr int kRingBytes = (kRingInCols + kRingOutCols) * kColBytes + 16;
};

// Bulk (TMA) copies of the strip-boundary rows.  One lane moves a 32-row
// chunk of the boundary buffer (global memory written by this warp's previous
// strip) into a ring half in shared memory with cp.async.bulk, completing on
// that half's mbarrier; the reader waits on the barrier's phase.  Sources and
// destinations are 16-byte aligned and sizes multiples of 16 (rows of 16 or 32
// bytes, 32 rows); the source is this GPU's own memory and no multicast is
// used.  Every wait is bounded: after kBulkWaitLimit polls it sets status bit
// 8 (the host reports BV_ERR_INTERNAL) and goes on.
constexpr unsigned kBulkWaitLimit = 1u << 22;

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* mb, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mb)), "r"(count) : "memory");
}
// A live barrier may not be initialised again: each strip invalidates its
// barriers once their last phase has completed.
__device__ __forceinline__ void mbar_inval(uint64_t* mb) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(mb)) : "memory");
}
// Makes barrier initialisation and this thread's earlier generic writes to
// global memory visible to the async proxy (the bulk copies).
__device__ __forceinline__ void fence_for_bulk() {
  asm volatile("fence.mbarrier_init.release.cluster;\n\tfence.proxy.async.global;\n\tfence.proxy.async.shared::cta;" ::
                   : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* mb) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%2], %3;\n\t"
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %3, [%2];"
      ::"r"(smem_addr(dst)), "l"(src), "r"(smem_addr(mb)), "r"(bytes) : "memory");
}
// Waits until the barrier's current phase (parity `phase`) completes.
__device__ __forceinline__ bool mbar_wait(uint64_t* mb, unsigned phase) {
  for (unsigned it = 0; it < kBulkWaitLimit; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(smem_addr(mb)), "r"(phase) : "memory");
    if (done) return true;
  }
  return false;
}

// FP32 adds a summing row below the read's last row: with e = 1, pMM = 1,
// the X coefficient = pMX(R) (undoing the X/pMX scaling) and pYY = 1, its M is
// M(R,c-1) + X(R,c-1) and its Y accumulates those, so after the last column
// its Y + M is the reference's sum over the last row of M + X
// (avx-pairhmm-template.h:328-343) -- computed with the cell arithmetic
// instead of two extra adds per step.  The single-strip FP32 kernel also keeps
// at least one padding row on top: then lane 0's top row may read its own
// bottom row through the shuffle, because a padding row's outputs reach the
// rows below only through zero coefficients.
template <typename T> struct SumRow { static constexpr bool value = sizeof(T) == 4; };


// Per-lane row constants for one strip.
// FP32 keeps X and Y divided by pMX / pMY (one FMA each, see above).  FP64,
// the rescue path, uses the reference's unscaled form: X/pMX can exceed the
// exponent range when insertion qualities jump between rows, and the FP64
// boundary rows are renormalised close to the top of the range.
template <typename T> struct ScaledXY { static constexpr bool value = sizeof(T) == 4; };

// Per-lane row constants for one strip.  Scaled form: mm = pMM, cx = pGAPM *
// pMX(r-1), cy = pGAPM * pMY(r-1), kap = pXX pMX(r-1)/pMX(r), g = pYY.
// Unscaled form: mm = pMM, cx = pGAPM (X->M), cy = pGAPM (Y->M), kap = pMX,
// my = pMY, gx = pXX, g = pYY.  With constant transitions (Tables::const_mode,
// the scalar model) X->M / Y->M and X->X / Y->Y may differ; both forms take
// them from the table instead of the quality bytes.
//
// Folded form (FP32, every real row of the strip with pMM >= kFoldMin): pMM(r)
// moves into row r's emissions and out of the M coefficient, cx and cy are
// multiplied by 1/pMM (Tables::mm_inv_f), so
//   M(r,c) = [e(r,c) pMM(r)] (M(r-1,c-1) + cx/pMM Xh(r-1,c-1) + cy/pMM Yh(r-1,c-1))
// takes two FMAs and a multiply: five operations per cell instead of six.
// The states keep their meaning (M, X/pMX, Y/pMY), so strips of one read may
// differ in form.  Rows with a small pMM (indel qualities of a few units)
// would need large coefficients; a strip holding one keeps the plain form.
template <typename T, int RT>
struct Rows {
  T mm[RT], cx[RT], cy[RT], kap[RT], my[RT], g[RT], gx[RT], y0[RT];
};

template <typename T> __device__ __forceinline__ const T* const_tab(const Tables* t);
template <> __device__ __forceinline__ const float* const_tab<float>(const Tables* t) { return t->cf; }
template <> __device__ __forceinline__ const double* const_tab<double>(const Tables* t) { return t->cd; }

// Computes the lane's row constants for the rows [rbase, rbase+RT) (real row
// numbers, row 0 = initial row, negative = padding) and writes the lane's
// emission-table column.  initializeVectors (avx-pairhmm-template.h:108-127)
// and stripeINITIALIZATION (:150-158) give the per-row probabilities.
// Returns whether the strip uses the folded form (warp-uniform; FP32 only).
template <typename T, int RT>
__device__ __forceinline__ bool setup_rows(const Tables* __restrict__ tb, const uchar4* __restrict__ quals,
                                           const uint8_t* __restrict__ bases, int R, int rbase, T init_y,
                                           Rows<T, RT>& rw, unsigned char* etab, int lane) {
  const T* ph = ph2pr_tab<T>(tb);
  const T* mmt = mm_tab<T>(tb);
  T em[RT], ex[RT];
  float minv[RT];  // 1/pMM of the row (NaN: too small to fold)
  uint32_t rc[RT];
  bool valid[RT], sumrow[RT];
#pragma unroll
  for (int j = 0; j < RT; ++j) {
    em[j] = T(0); ex[j] = T(0); minv[j] = 1.f; rc[j] = 0; valid[j] = false; sumrow[j] = false;
  }
#pragma unroll
  for (int j = 0; j < RT; ++j) {
    const int r = rbase + j;
    if (SumRow<T>::value && r == R + 1 && R >= 1) {
      rw.mm[j] = T(1);
      // pMX(R): Xh(R) * pMX(R) = X(R)
      rw.cx[j] = tb->const_mode ? const_tab<T>(tb)[1] : ph[quals[R - 1].y & kQualMask];
      rw.cy[j] = T(0); rw.kap[j] = T(0); rw.my[j] = T(0);
      rw.g[j] = T(1); rw.gx[j] = T(1);
      rw.y0[j] = T(0);
      sumrow[j] = true;
    } else if (r >= 1 && r <= R) {
      const uchar4 qv = quals[r - 1];
      const int qq = qv.x & kQualMask;
      // transitions into row r: M->M, M->X, M->Y, X->M, X->X, Y->M, Y->Y
      T mmv, pmx, pmy, gpx, gx, gpy, gy;
      T ap = T(1), bp = T(1);  // scale of the row above: pMX/pMY, or 1 for row 0
      if (tb->const_mode) {
        const T* c = const_tab<T>(tb);
        mmv = c[0]; pmx = c[1]; pmy = c[2]; gpx = c[3]; gx = c[4]; gpy = c[5]; gy = c[6];
        minv[j] = tb->cf[7];
        if (ScaledXY<T>::value && r >= 2) { ap = pmx; bp = pmy; }
      } else {
        const int qi = qv.y & kQualMask, qd = qv.z & kQualMask, qc = qv.w & kQualMask;
        pmx = ph[qi]; pmy = ph[qd]; gx = ph[qc]; gy = gx;
        gpx = T(1) - gx; gpy = gpx;
        mmv = mmt[mm_index(qi, qd)];
        minv[j] = tb->mm_inv_f[mm_index(qi, qd)];
        if (ScaledXY<T>::value && r >= 2) {
          const uchar4 pv = quals[r - 2];
          ap = ph[pv.y & kQualMask];
          bp = ph[pv.z & kQualMask];
        }
      }
      rw.mm[j] = mmv;
      if constexpr (ScaledXY<T>::value) {
        rw.cx[j] = gpx * ap;
        rw.cy[j] = gpy * bp;
        rw.kap[j] = gx * ap / pmx;
        rw.my[j] = T(0);
      } else {
        rw.cx[j] = gpx;
        rw.cy[j] = gpy;
        rw.kap[j] = pmx;
        rw.my[j] = pmy;
      }
      rw.g[j] = gy;
      rw.gx[j] = gx;
      rw.y0[j] = T(0);
      const T eps = ph[qq];
      em[j] = T(1) - eps;
      ex[j] = eps / T(3);
      rc[j] = base_code(bases[r - 1]);
      valid[j] = true;
    } else {
      // padding rows and row 0: M = 0, X = 0, Y carried unchanged
      rw.mm[j] = T(0); rw.cx[j] = T(0); rw.cy[j] = T(0); rw.kap[j] = T(0); rw.my[j] = T(0);
      rw.g[j] = T(1); rw.gx[j] = T(0);
      rw.y0[j] = (r == 0) ? init_y : T(0);
    }
  }
  bool fold = false;
  if constexpr (ScaledXY<T>::value) {
    bool small = false;
#pragma unroll
    for (int j = 0; j < RT; ++j) small |= valid[j] && !(minv[j] > 0.f);
    fold = !__any_sync(0xffffffffu, small);
    if (fold) {
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        if (valid[j]) {
          rw.cx[j] = rw.cx[j] * minv[j];
          rw.cy[j] = rw.cy[j] * minv[j];
          em[j] = em[j] * rw.mm[j];
          ex[j] = ex[j] * rw.mm[j];
        }
      }
    }
  }
  // Emission table: for haplotype code h, row j: 1-eps on a match, eps/3 on a
  // mismatch (a read or haplotype N matches everything), 0 for padding; times
  // pMM in the folded form.
#pragma unroll
  for (int h = 0; h < kCodes; ++h) {
    T v[RT];
#pragma unroll
    for (int j = 0; j < RT; ++j) {
      const bool match = (rc[j] == (uint32_t)h) || rc[j] == 4u || h == 4;
      v[j] = sumrow[j] ? T(1) : (valid[j] && h != kPadCode) ? (match ? em[j] : ex[j]) : T(0);
    }
    store_emissions<T, RT>(etab, lane, h, v);
  }
  return fold;
}

// Stages a haplotype as column codes: code[kHapLead + c - 1] for c = 1..H,
// kPadCode everywhere else in [0, n_total).
__device__ __forceinline__ void stage_hap(const uint8_t* __restrict__ hap, int H, unsigned char* hc, int n_total,
                                          int lane) {
  for (int x = lane; x < n_total; x += kWarp) {
    const int c = x - kHapLead + 1;
    hc[x] = (c >= 1 && c <= H) ? (unsigned char)base_code(hap[c - 1]) : (unsigned char)kPadCode;
  }
}

// The same for all threads of a block (the long-read kernel's shared codes).
__device__ __forceinline__ void stage_hap_block(const uint8_t* __restrict__ hap, int H, unsigned char* hc,
                                                int n_total) {
  for (int x = threadIdx.x; x < n_total; x += blockDim.x) {
    const int c = x - kHapLead + 1;
    hc[x] = (c >= 1 && c <= H) ? (unsigned char)base_code(hap[c - 1]) : (unsigned char)kPadCode;
  }
}

// Stages two haplotypes for a paired warp: entry x holds the emission-table
// offsets of both haplotypes' codes at column kHapLead + c - 1 (first in the
// low 16 bits), so one 32-bit shared load per step serves both.
template <int STRIDE>
__device__ __forceinline__ void stage_hap_pair(const uint8_t* __restrict__ ha, int HA, const uint8_t* __restrict__ hb,
                                               int HB, uint32_t* hcp, int n_total, int lane) {
  static_assert(kCodes * STRIDE <= 65536, "offsets fit 16 bits");
  for (int x = lane; x < n_total; x += kWarp) {
    const int c = x - kHapLead + 1;
    const uint32_t ca = (c >= 1 && c <= HA) ? base_code(ha[c - 1]) : (uint32_t)kPadCode;
    const uint32_t cb = (c >= 1 && c <= HB) ? base_code(hb[c - 1]) : (uint32_t)kPadCode;
    hcp[x] = ca * STRIDE | (cb * STRIDE) << 16;
  }
}

// One strip of the wavefront.  MULTI: lane 0 reads the row above the strip
// from `bnd` (the previous strip's bottom row, or zeros for the first strip)
// and lane 31 writes this strip's bottom row back to `bnd`, both through
// shared-memory rings.  Column c of the boundary row is buffer row c + 31.
// On return, lane 31 holds its bottom row's final M and Y (the summing row's
// result for FP32), the per-step sums of M and X over the bottom row (FP64,
// which has no summing row) and the largest bottom-row value (FP64, for
// renormalisation between strips).
template <typename T, int RT, bool MULTI, int CH, bool FOLD = false>
__device__ __forceinline__ void run_strip(const Rows<T, RT>& rw, const ELane el,
                                          const unsigned char* __restrict__ hc_lane, int nsteps, int lane,
                                          T* __restrict__ bnd, unsigned char* ring, T in_scale, T& lastM,
                                          T& lastY, T& sumM, T& sumX, T& bmax,
                                          unsigned long long* status = nullptr) {
  using S = WarpSmem<T, RT>;
  constexpr bool kScale = sizeof(T) == 8;  // only the FP64 path renormalises
  constexpr bool kSums = !SumRow<T>::value;
  T M[RT], X[RT], Y[RT];
#pragma unroll
  for (int j = 0; j < RT; ++j) { M[j] = T(0); X[j] = T(0); Y[j] = rw.y0[j]; }
  sumM = T(0); sumX = T(0); bmax = T(0);
  // Values the lane above publishes before step 0: its bottom row at
  // "column <= 0", i.e. the column-0 boundary state.
  T upM = __shfl_up_sync(0xffffffffu, M[RT - 1], 1);
  T upX = __shfl_up_sync(0xffffffffu, X[RT - 1], 1);
  T upY = __shfl_up_sync(0xffffffffu, Y[RT - 1], 1);
  T dM = upM, dX = upX, dY = upY;
  T* ring_in = reinterpret_cast<T*>(ring);
  T* ring_out = reinterpret_cast<T*>(ring + S::kRingInCols * S::kColBytes);
  uint64_t* mb = reinterpret_cast<uint64_t*>(ring + (S::kRingInCols + S::kRingOutCols) * S::kColBytes);
  constexpr unsigned kChunkBytes = 32u * S::kColBytes;
  unsigned phase = 0;     // lane 0: bit h = parity of ring half h's next completion
  bool bulk_ok = true;    // lane 0: every bulk wait completed
  if constexpr (MULTI) {
    static_assert(CH == 32, "multi-strip runs 32-step chunks");
    // Lane 0 needs, at step s, buffer row s + 32 (column s + 1); those rows
    // are streamed into a 64-row ring: chunk k (steps 32k..32k+31) uses ring
    // half k&1, prefetched by a bulk copy during chunk k-1.  Step 0's
    // diagonal is row 31.  The boundary rows were written by every lane
    // (previous strip, or the zeroing): each lane fences them towards the
    // async proxy before lane 0 issues the copies.
    fence_for_bulk();
    __syncwarp();
    if (lane == 0) {
      mbar_init(mb, 1);
      mbar_init(mb + 1, 1);
      fence_for_bulk();
      bulk_g2s(ring_in, bnd + (size_t)32 * 4, kChunkBytes, mb);
      dM = bnd[31 * 4 + 0]; dX = bnd[31 * 4 + 1]; dY = bnd[31 * 4 + 2];
      if constexpr (kScale) { dM *= in_scale; dX *= in_scale; dY *= in_scale; }
      bulk_ok &= mbar_wait(mb, 0);
      phase ^= 1u;
    }
    __syncwarp();
  } else if constexpr (!SumRow<T>::value) {
    if (lane == 0) { upM = T(0); dM = T(0); }
  }

  for (int s0 = 0; s0 < nsteps; s0 += CH) {
    if constexpr (MULTI) {
      const int nk = s0 / 32 + 1;  // prefetch of the next chunk's rows into half nk & 1
      if (lane == 0) bulk_g2s(ring_in + (nk & 1) * 32 * 4, bnd + (size_t)(32 * nk + 32) * 4, kChunkBytes, mb + (nk & 1));
    }
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      const int s = s0 + u;
      if constexpr (MULTI) {
        if (lane == 0) {
          const T* rin = ring_in + ((((s0 >> 5) & 1) * 32) + u) * 4;
          upM = rin[0]; upX = rin[1]; upY = rin[2];
          if constexpr (kScale) { upM *= in_scale; upX *= in_scale; upY *= in_scale; }
        }
      }
      T e[RT];
      load_emissions<T, RT>(el, (unsigned)hc_lane[s] * S::kCodeStride, e);
      T um = upM, ux = upX;
      T dm = dM, dx = dX, dy = dY;
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        T mn, xn, yn;
        if constexpr (ScaledXY<T>::value && FOLD) {
          mn = e[j] * fma_(rw.cy[j], dy, fma_(rw.cx[j], dx, dm));
          xn = fma_(rw.kap[j], ux, um);
          yn = fma_(rw.g[j], Y[j], M[j]);
        } else if constexpr (ScaledXY<T>::value) {
          mn = e[j] * fma_(rw.mm[j], dm, fma_(rw.cx[j], dx, rw.cy[j] * dy));
          xn = fma_(rw.kap[j], ux, um);
          yn = fma_(rw.g[j], Y[j], M[j]);
        } else {
          mn = e[j] * fma_(rw.mm[j], dm, fma_(rw.cx[j], dx, rw.cy[j] * dy));
          xn = fma_(rw.gx[j], ux, rw.kap[j] * um);
          yn = fma_(rw.g[j], Y[j], rw.my[j] * M[j]);
        }
        dm = M[j]; dx = X[j]; dy = Y[j];
        um = mn; ux = xn;
        M[j] = mn; X[j] = xn; Y[j] = yn;
      }
      if constexpr (kSums) {
        sumM += M[RT - 1];
        sumX += X[RT - 1];
      }
      const T nM = __shfl_up_sync(0xffffffffu, M[RT - 1], 1);
      const T nX = __shfl_up_sync(0xffffffffu, X[RT - 1], 1);
      const T nY = __shfl_up_sync(0xffffffffu, Y[RT - 1], 1);
      if constexpr (MULTI) {
        if (lane == kWarp - 1) {
          T* ro = ring_out + u * 4;
          ro[0] = M[RT - 1]; ro[1] = X[RT - 1]; ro[2] = Y[RT - 1];
          if constexpr (kScale) bmax = fmax(bmax, fmax(M[RT - 1], fmax(X[RT - 1], Y[RT - 1])));
        }
      }
      dM = upM; dX = upX; dY = upY;
      upM = nM; upX = nX; upY = nY;
      if constexpr (!MULTI && !SumRow<T>::value) {
        if (lane == 0) upM = T(0);
      }
    }
    if constexpr (MULTI) {
      // End of a 32-step chunk: flush its bottom row (buffer rows s0+1 ..
      // s0+32; ring slot u holds step s0+u, i.e. column s0+u-30) and make the
      // prefetched chunk visible.
      __syncwarp();
      T* dstb = bnd + (size_t)(s0 + 1 + lane) * 4;
      const T* srco = ring_out + lane * 4;
      if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(dstb) = *reinterpret_cast<const float4*>(srco);
      } else {
        reinterpret_cast<double2*>(dstb)[0] = reinterpret_cast<const double2*>(srco)[0];
        reinterpret_cast<double2*>(dstb)[1] = reinterpret_cast<const double2*>(srco)[1];
      }
      __threadfence_block();
      if (lane == 0) {
        const int h = (s0 / 32 + 1) & 1;  // the prefetched half
        bulk_ok &= mbar_wait(mb + h, (phase >> h) & 1u);
        phase ^= 1u << h;
      }
      __syncwarp();
    }
  }
  if constexpr (MULTI) {
    // Every copy has been waited for (the last chunk waits for the half it
    // prefetched), unless a wait gave up; then the copy may still land, and
    // the barriers stay as they are (the status already fails the call).
    if (lane == 0) {
      if (bulk_ok) {
        mbar_inval(mb);
        mbar_inval(mb + 1);
      } else if (status) {
        atomicOr(status, 8ull);
      }
    }
    __syncwarp();
  }
  lastM = M[RT - 1];
  lastY = Y[RT - 1];
}

// Two haplotypes of one read in one warp (FP32 single strip).  Both pairs
// share the read's row constants and emission table; their states are the
// two halves of float2 values, so the transition arithmetic runs as packed
// FP32x2 instructions (fma.rn.f32x2 / mul.rn.f32x2 of sm_100), which halves
// the issue slots the FP32 pipe needs and leaves them to the shuffles and
// shared-memory loads.  Each half follows run_strip's operation order
// exactly, so a paired result equals the single-haplotype result bit for bit.
__device__ __forceinline__ float2 shfl_up2(float2 v) {
  return make_float2(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1));
}

// The lane above sends, instead of its bottom row's M, X and Y, the two sums
// this lane's top row r consumes (two shuffles per haplotype and step
// instead of three):
//   zx = kap(r) Xh(r-1,c) + M(r-1,c)                              (X of row r)
//   zm = pMM(r) M(r-1,c-1) + cx(r) Xh(r-1,c-1) + cy(r) Yh(r-1,c-1)  (M of row r / e)
// computed from the row-r constants the lane above holds (mmN, cxN, cyN,
// kapN), with the operations and operands of the top row's own update.
// Lane 0 receives its own sums: its top row is padding (e = 0) and the row
// below has zero X coefficient, so they reach no real row.
template <int RT, bool FOLD>
__device__ __forceinline__ void run_strip_pair(const Rows<float, RT>& rw, const float* __restrict__ y0a,
                                               const float* __restrict__ y0b, const ELane el,
                                               const uint32_t* __restrict__ hcp_lane, int nsteps,
                                               float2& lastM, float2& lastY) {
  constexpr int CH = 8;
  float2 mm[RT], cx[RT], cy[RT], kap[RT], g[RT];
  float2 M[RT], X[RT], Y[RT];
#pragma unroll
  for (int j = 0; j < RT; ++j) {
    mm[j] = make_float2(rw.mm[j], rw.mm[j]);
    cx[j] = make_float2(rw.cx[j], rw.cx[j]);
    cy[j] = make_float2(rw.cy[j], rw.cy[j]);
    kap[j] = make_float2(rw.kap[j], rw.kap[j]);
    g[j] = make_float2(rw.g[j], rw.g[j]);
    M[j] = make_float2(0.f, 0.f);
    X[j] = make_float2(0.f, 0.f);
    Y[j] = make_float2(y0a[j], y0b[j]);
  }
  // the next lane's top-row constants
  const float mmN1 = __shfl_down_sync(0xffffffffu, rw.mm[0], 1), cxN1 = __shfl_down_sync(0xffffffffu, rw.cx[0], 1);
  const float cyN1 = __shfl_down_sync(0xffffffffu, rw.cy[0], 1), kapN1 = __shfl_down_sync(0xffffffffu, rw.kap[0], 1);
  const float2 mmN = make_float2(mmN1, mmN1), cxN = make_float2(cxN1, cxN1);
  const float2 cyN = make_float2(cyN1, cyN1), kapN = make_float2(kapN1, kapN1);
  // sums for step 0 from the column-0 boundary state (M = X = 0, Y = y0)
  // (the folded form drops pMM: mmN is 1 there and unused)
  auto msum = [&](float2 m, float2 x, float2 y) {
    if constexpr (FOLD) return __ffma2_rn(cyN, y, __ffma2_rn(cxN, x, m));
    else return __ffma2_rn(mmN, m, __ffma2_rn(cxN, x, __fmul2_rn(cyN, y)));
  };
  float2 zx = shfl_up2(__ffma2_rn(kapN, X[RT - 1], M[RT - 1]));
  float2 zm = shfl_up2(msum(M[RT - 1], X[RT - 1], Y[RT - 1]));
  for (int s0 = 0; s0 < nsteps; s0 += CH) {
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      const int s = s0 + u;
      const uint32_t offs = hcp_lane[s];
      float ea[RT], eb[RT];
      load_emissions<float, RT>(el, offs & 0xffffu, ea);
      load_emissions<float, RT>(el, offs >> 16, eb);
      // top row from the lane above's sums
      const float2 mn0 = make_float2(ea[0] * zm.x, eb[0] * zm.y);
      const float2 yn0 = __ffma2_rn(g[0], Y[0], M[0]);
      float2 dm = M[0], dx = X[0], dy = Y[0];
      float2 um = mn0, ux = zx;
      M[0] = mn0; X[0] = zx; Y[0] = yn0;
#pragma unroll
      for (int j = 1; j < RT; ++j) {
        float2 t;
        if constexpr (FOLD) {
          t = __ffma2_rn(cx[j], dx, dm);
          t = __ffma2_rn(cy[j], dy, t);
        } else {
          t = __fmul2_rn(cy[j], dy);
          t = __ffma2_rn(cx[j], dx, t);
          t = __ffma2_rn(mm[j], dm, t);
        }
        const float2 mn = make_float2(ea[j] * t.x, eb[j] * t.y);
        const float2 xn = __ffma2_rn(kap[j], ux, um);
        const float2 yn = __ffma2_rn(g[j], Y[j], M[j]);
        dm = M[j]; dx = X[j]; dy = Y[j];
        um = mn; ux = xn;
        M[j] = mn; X[j] = xn; Y[j] = yn;
      }
      // dm/dx/dy: the bottom row at column c-1; M/X/Y[RT-1]: at column c
      zx = shfl_up2(__ffma2_rn(kapN, X[RT - 1], M[RT - 1]));
      zm = shfl_up2(msum(dm, dx, dy));
    }
  }
  lastM = M[RT - 1];
  lastY = Y[RT - 1];
}

template <typename T> __device__ __forceinline__ T log10_(T v);
template <> __device__ __forceinline__ float log10_(float v) { return log10f(v); }
template <> __device__ __forceinline__ double log10_(double v) { return log10(v); }

// Work items: full-DP units (a read against consecutive haplotypes) or single
// pairs from the FP64 list.
struct Item {
  int read, hap0, nh;
  long long out0;
};

// Writes one pair's log10 likelihood (lane 31 holds the result).  FP32:
// values below MIN_ACCEPTED or not finite go to the FP64 list (or NaN when
// the launch has none); FP64: log10 of the renormalised sum, -inf when it
// stayed non-positive.
template <typename T>
__device__ __forceinline__ void write_result(const KernelParams& p, int read, int hap, long long o, T res,
                                             long long kexp) {
  if (sizeof(T) == 4) {
    if (!p.rescue && (!(res >= (T)kMinAccepted) || isinf((double)res))) {
      p.out[o] = __longlong_as_double(0x7ff8000000000000ll);
    } else if (!(res >= (T)kMinAccepted) || isinf((double)res)) {
      // reads of at least long_rows bases go to the long list, filled from the
      // list's far end for the several-warps-per-pair FP64 kernel
      const bool lng = p.long_rows > 0 && p.batch.read_off[read + 1] - p.batch.read_off[read] >= p.long_rows;
      const unsigned long long slot = atomicAdd(lng ? &p.ctr->rescue_long_count : &p.ctr->rescue_count, 1ull);
      if (slot < (unsigned long long)p.rescue_cap) {
        const long long at = lng ? p.rescue_cap - 1 - (long long)slot : (long long)slot;
        p.rescue[at].read = read;
        p.rescue[at].hap = hap;
        p.rescue[at].out = o;
      } else {
        atomicOr(&p.ctr->status, 1ull);
      }
      p.out[o] = __longlong_as_double(0x7ff8000000000000ll);
    } else {
      p.out[o] = (double)(log10_((float)res) - p.tables->log10_init_f);
    }
  } else {
    const double rd = (double)res;
    if (rd > 0.0 && isfinite(rd)) {
      p.out[o] = log10(rd) + (double)kexp * 0.30102999566398119521 - p.tables->log10_init_d;
    } else {
      atomicAdd(&p.ctr->underflow_count, 1ull);
      p.out[o] = -INFINITY;
    }
  }
}

// Whether an FP32 multi-strip pair's result is certain to fall below
// kMinAccepted, from its last strip's bottom row in the boundary buffer
// (column c at buffer row c + 31; values M, X/pMX, Y/pMY).  The mass a row
// passes to the next one is at most its own (every state's transitions into
// the next row sum to <= 1 and emissions are <= 1); only the in-row deletion
// chain adds, at most a factor 1 + pMY/(1 - pYY) per row.  The bottom row's
// M + X/pMX + Y/pMY bounds its M + X + Y from above; times the chain factor
// over all rows, and twice that against the rounding of the FP32 sums, it
// bounds the result.  Kept out of line: it runs once per strip.
static __device__ __noinline__ bool fp32_result_below_threshold(const Tables* tb, const float* bnd, int H,
                                                         const uchar4* quals, int R, int lane) {
  float mass = 0.f;
  for (int c = 1 + lane; c <= H; c += kWarp) {
    const float4 v = *reinterpret_cast<const float4*>(bnd + (size_t)(c + 31) * 4);
    mass += v.x + v.y + v.z;
  }
  for (int o = 16; o > 0; o >>= 1) mass += __shfl_xor_sync(0xffffffffu, mass, o);
  if (!(isfinite(mass) && mass < (float)kMinAccepted)) return false;
  float growth = 0.f;  // log2 of the deletion-chain factor
  for (int r = lane; r < R; r += kWarp) {
    float pmy, pyy;
    if (tb->const_mode) { pmy = tb->cf[2]; pyy = tb->cf[6]; }
    else { pmy = tb->ph2pr_f[quals[r].z & kQualMask]; pyy = tb->ph2pr_f[quals[r].w & kQualMask]; }
    growth += pyy < 1.f ? __log2f(1.f + pmy / (1.f - pyy)) * 1.0001f + 1e-6f : 1e30f;
  }
  for (int o = 16; o > 0; o >>= 1) growth += __shfl_xor_sync(0xffffffffu, growth, o);
  return growth < 100.f && 2.f * mass * exp2f(growth) < (float)kMinAccepted;
}

template <typename T, int RT, bool MULTI, bool PAIR = false>
__device__ void process_item(const KernelParams& p, const Item& it, unsigned char* wsm, int lane, T* bnd) {
  using S = WarpSmem<T, RT>;
  const DeviceBatch& b = p.batch;
  const int64_t ro = b.read_off[it.read];
  const int R = (int)(b.read_off[it.read + 1] - ro);
  const uchar4* quals = b.read_quals + ro;
  const uint8_t* bases = b.read_bases + ro;
  // Padded row space: padding rows on top, row 0, rows 1..R, and (FP32) the
  // summing row; the host chose RT so that single-strip FP32 keeps >= 1
  // padding row on top.
  const int rows = R + 1 + (SumRow<T>::value ? 1 : 0);
  const int strip_rows = kWarp * RT;
  const int nstrips = (rows_needed(R, SumRow<T>::value, !MULTI) + strip_rows - 1) / strip_rows;
  const int pad = nstrips * strip_rows - rows;
  unsigned char* hc = wsm;
  unsigned char* etab = wsm + p.hap_bytes;
  const ELane el = elane<T, RT>(etab, lane);
  unsigned char* ring = etab + S::kEtabBytes;
  const bool is_f64 = sizeof(T) == 8;
  Rows<T, RT> rw;
  bool fold = false;
  if (!MULTI) {
    // single strip: rows and emission table are shared by all haplotypes
    fold = setup_rows<T, RT>(p.tables, quals, bases, R, lane * RT - pad, T(0), rw, etab, lane);
  }
  for (int k = 0; k < it.nh; ++k) {
    const int h = it.hap0 + k;
    const int64_t ho = b.hap_off[h];
    const int H = (int)(b.hap_off[h + 1] - ho);
    if constexpr (PAIR && !MULTI && sizeof(T) == 4) {
      if (k + 1 < it.nh && R > 0) {
        const int64_t ho2 = b.hap_off[h + 1];
        const int H2 = (int)(b.hap_off[h + 2] - ho2);
        if (H > 0 && H2 > 0) {
          const int Hm = H > H2 ? H : H2;
          const int nsteps = (Hm + kWarp + 7) / 8 * 8;  // as the single path: H + 31 + 1 (summing row), to 8
          uint32_t* hcp = reinterpret_cast<uint32_t*>(hc);
          __syncwarp();
          stage_hap_pair<S::kCodeStride>(b.hap_bases + ho, H, b.hap_bases + ho2, H2, hcp, nsteps + kHapLead, lane);
          const T init = (T)p.tables->init_f;
          const int r0j = pad - lane * RT;
          float y0a[RT], y0b[RT];
#pragma unroll
          for (int j = 0; j < RT; ++j) {
            y0a[j] = (j == r0j) ? init / (T)H : 0.f;
            y0b[j] = (j == r0j) ? init / (T)H2 : 0.f;
          }
          __syncwarp();
          float2 lastM, lastY;
          if (fold) run_strip_pair<RT, true>(rw, y0a, y0b, el, hcp + kHapLead - lane, nsteps, lastM, lastY);
          else run_strip_pair<RT, false>(rw, y0a, y0b, el, hcp + kHapLead - lane, nsteps, lastM, lastY);
          if (lane == kWarp - 1) {
            write_result<float>(p, it.read, h, it.out0 + k, lastY.x + lastM.x, 0);
            write_result<float>(p, it.read, h + 1, it.out0 + k + 1, lastY.y + lastM.y, 0);
          }
          ++k;
          continue;
        }
      }
    }
    if (H == 0 || R == 0) {
      // An empty read or haplotype has no alignment: likelihood 0.
      if (lane == kWarp - 1) p.out[it.out0 + k] = -INFINITY;
      continue;
    }
    const T init = is_f64 ? (T)p.tables->init_d : (T)p.tables->init_f;
    const T init_y = init / (T)H;
    const int CHK = MULTI ? 32 : 8;
    // lane 31 reaches column H at step H+30; the FP32 summing row trails the
    // last read row by one column, so FP32 runs one step more.
    const int nsteps = (H + kWarp - 1 + (SumRow<T>::value ? 1 : 0) + CHK - 1) / CHK * CHK;
    __syncwarp();
    stage_hap(b.hap_bases + ho, H, hc, nsteps + kHapLead, lane);
    if (!MULTI) {
      // the initial row's Y depends on the haplotype length
      const int r0j = pad - lane * RT;  // j of row 0 within this lane, if here
#pragma unroll
      for (int j = 0; j < RT; ++j) rw.y0[j] = (j == r0j) ? init_y : T(0);
    }
    __syncwarp();
    T lastM, lastY, sumM, sumX, bmax;
    long long kexp = 0;  // stored values are true values * 2^-kexp
    bool handed_over = false;  // FP32: the pair went to the FP64 list before its last strip
    if constexpr (MULTI) {
      // boundary row of "strip -1": all zero
      for (int x = lane; x < nsteps + 96; x += kWarp) {
        bnd[(size_t)x * 4 + 0] = T(0); bnd[(size_t)x * 4 + 1] = T(0); bnd[(size_t)x * 4 + 2] = T(0);
      }
      // FP32 early hand-off: once a strip's bottom row proves that the FP32
      // result will fall below kMinAccepted (fp32_result_below_threshold), the
      // reference's rule sends the pair to FP64; it goes there now instead of
      // after its remaining strips.
      T in_scale = T(1);
      for (int st = 0; st < nstrips; ++st) {
        __syncwarp();
        fold = setup_rows<T, RT>(p.tables, quals, bases, R, st * strip_rows + lane * RT - pad, init_y, rw, etab, lane);
        __syncwarp();
        if (fold)
          run_strip<T, RT, true, 32, true>(rw, el, hc + kHapLead - lane, nsteps, lane, bnd, ring, in_scale, lastM,
                                           lastY, sumM, sumX, bmax, &p.ctr->status);
        else
          run_strip<T, RT, true, 32>(rw, el, hc + kHapLead - lane, nsteps, lane, bnd, ring, in_scale, lastM,
                                     lastY, sumM, sumX, bmax, &p.ctr->status);
        __syncwarp();
        if constexpr (sizeof(T) == 4) {
          if (st + 1 < nstrips && p.rescue &&
              fp32_result_below_threshold(p.tables, reinterpret_cast<const float*>(bnd), H, quals, R, lane)) {
            handed_over = true;
            // read rows 1 .. R sit at padded rows pad + 1 .. pad + R; strips 0 .. st covered those below (st + 1) strip_rows
            const int done = min(R, (st + 1) * strip_rows - pad - 1);
            if (lane == kWarp - 1 && done < R)
              atomicAdd(&p.ctr->fp32_skipped_cells, (unsigned long long)(R - done) * (unsigned long long)H);
            break;
          }
        }
        in_scale = T(1);
        if (p.rescale && st + 1 < nstrips) {
          const T m = __shfl_sync(0xffffffffu, bmax, kWarp - 1);
          if (m > T(0)) {
            int e2;
            frexp((double)m, &e2);
            // keep the row maximum near 2^(target) so the next strip has headroom
            const int shift = e2 - p.rescale_target;
            kexp += shift;
            in_scale = (T)ldexp(1.0, -shift);
          }
        }
      }
    } else {
      if (fold)
        run_strip<T, RT, false, 8, true>(rw, el, hc + kHapLead - lane, nsteps, lane, nullptr, nullptr, T(1), lastM,
                                         lastY, sumM, sumX, bmax);
      else
        run_strip<T, RT, false, 8>(rw, el, hc + kHapLead - lane, nsteps, lane, nullptr, nullptr, T(1), lastM,
                                   lastY, sumM, sumX, bmax);
    }
    if (lane == kWarp - 1) {
      // FP32: the summing row's Y + M; FP64: the accumulated last-row sums;
      // a pair handed over early counts as below the rescue threshold.
      const T res = handed_over ? T(0) : SumRow<T>::value ? lastY + lastM : sumM + sumX;
      write_result<T>(p, it.read, h, it.out0 + k, res, kexp);
      if (is_f64 && p.cells_ctr) atomicAdd(p.cells_ctr, (unsigned long long)R * (unsigned long long)H);
    }
  }
}

}  // namespace bvphmm
