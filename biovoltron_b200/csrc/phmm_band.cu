// phmm_band.cu -- learned-band PairHMM path (see phmm_band.h for the pipeline).
//
// The reference computes every pair over its full read x haplotype matrix
// (avx-pairhmm-template.h:210-346).  Here a pair whose alignment is confined
// to a narrow diagonal band is scored on that band only: cells with diagonal
// d = c - r in [d_lo, d_lo + W) follow the reference recurrence, cells outside
// are zero.  The band comes from the 11-mer seed diagonal d* of the pair and
// from a small MLP that predicts the band's lower and upper edge relative to
// d*; the full DP takes every pair the band path cannot vouch for.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>

#include "phmm_band.h"
#include "phmm_common.h"
#include "phmm_kernels.h"
#include "phmm_rows.h"

namespace bvphmm {
namespace {

constexpr uint32_t kEmpty = 0xffffffffu;  // free hash-table slot

__device__ __forceinline__ int kmer_code(uint8_t b) {
  // 2-bit code for A C T G (ConvertChar's order); -1 for anything else.
  return b == 'A' ? 0 : b == 'C' ? 1 : b == 'T' ? 2 : b == 'G' ? 3 : -1;
}

// One-hot nibble used by the banded kernel's match test: a read or haplotype
// N matches everything (0xF), other unknown bytes read as A (ConvertChar).
__device__ __forceinline__ uint32_t onehot(uint8_t b) {
  return b == 'C' ? 2u : b == 'T' ? 4u : b == 'G' ? 8u : b == 'N' ? 15u : 1u;
}

__global__ void k_pairs_from_units(const Unit* __restrict__ units, long long n_units, int32_t* pair_read,
                                   int32_t* pair_hap) {
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < n_units;
       u += (long long)gridDim.x * blockDim.x) {
    const Unit un = units[u];
    for (int k = 0; k < un.nh; ++k) {
      pair_read[un.out0 + k] = un.read;
      pair_hap[un.out0 + k] = un.hap0 + k;
    }
  }
}

// Per haplotype h: a bucketed hash table of its 11-mers at
// table + tbl_base(h): (H + 1) / 2 buckets of 4 slots (load factor <= 1/2);
// a key lives in its hash bucket or, when that is full, in the next bucket
// with a free slot.  An entry is (code << 10) | position; kEmpty marks a free
// slot.  Built in shared memory, written out coalesced.  Haplotypes longer
// than kBandMaxHap get no table (the featuriser routes their pairs to the
// full DP).
// A table starts on a 16-byte boundary (its buckets are read as uint4 from
// global memory): word 2 hap_off + 8 h rounded up to a multiple of 4.  Table
// h spans at most 2 H + 2 words, which ends before table h + 1 starts; the
// buffer holds 2 n_hap_bytes + 8 n_haps + 4 words (kHapTableWords).
__device__ __forceinline__ int64_t tbl_base(int64_t hap_off, long long h) { return (2 * hap_off + 8 * h + 3) & ~3ll; }
__device__ __forceinline__ uint32_t tbl_bucket(uint32_t code, uint32_t nb) {
  return (uint32_t)(((uint64_t)(code * 0x9E3779B1u) * nb) >> 32);
}

// A warp per haplotype: lane l takes a run of consecutive positions and rolls
// the 11-mer code along it (one new base per position; an 11-bit shift
// register marks windows holding a non-ACGT byte), inserting with atomicCAS
// into the warp's table in shared memory; the table then goes out coalesced.
// Insertion order does not matter to the lookups: a key sits in its bucket
// or in a later one that was full when it was inserted, and buckets only
// fill up, so a probe that stops at the first bucket with a free slot sees it.
constexpr int kHapTblWarps = 4;
constexpr int kHapTblWords = 2 * kBandMaxHap + 4;

__global__ void __launch_bounds__(kHapTblWarps * 32) k_hap_table(const uint8_t* __restrict__ hap_bases,
                                                                 const int64_t* __restrict__ hap_off, long long n_haps,
                                                                 uint32_t* __restrict__ table) {
  __shared__ uint32_t s_tbl[kHapTblWarps][kHapTblWords];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t* st = s_tbl[wib];
  const long long nwarps = (long long)gridDim.x * kHapTblWarps;
  for (long long h = blockIdx.x * (long long)kHapTblWarps + wib; h < n_haps; h += nwarps) {
    const int64_t off = hap_off[h];
    const int H = (int)(hap_off[h + 1] - off);
    if (H > kBandMaxHap || H < kK) continue;
    const uint32_t nb = (uint32_t)(H + 1) / 2;
    for (uint32_t x = lane; x < 4 * nb; x += 32) st[x] = kEmpty;
    __syncwarp();
    const uint8_t* hb = hap_bases + off;
    const int npos = H - kK + 1;
    const int seg = (npos + 31) / 32;
    const int x0 = lane * seg, x1 = min(npos, x0 + seg);
    if (x0 < x1) {
      uint32_t code = 0, bad = 0;
      for (int t = 0; t < kK - 1; ++t) {
        const int c = kmer_code(hb[x0 + t]);
        code = (code << 2) | (uint32_t)(c & 3);
        bad = (bad << 1) | (c < 0 ? 1u : 0u);
      }
      for (int x = x0; x < x1; ++x) {
        const int c = kmer_code(hb[x + kK - 1]);
        code = ((code << 2) | (uint32_t)(c & 3)) & ((1u << (2 * kK)) - 1u);
        bad = ((bad << 1) | (c < 0 ? 1u : 0u)) & ((1u << kK) - 1u);
        if (bad) continue;
        const uint32_t e = (code << 10) | (uint32_t)x;
        uint32_t bk = tbl_bucket(code, nb);
        bool done = false;
        for (uint32_t tries = 0; tries < nb && !done; ++tries, bk = bk + 1 == nb ? 0 : bk + 1)
          for (int t = 0; t < 4 && !done; ++t) done = atomicCAS(&st[4 * bk + t], kEmpty, e) == kEmpty;
      }
    }
    __syncwarp();
    uint32_t* dst = table + tbl_base(off, h);
    for (uint32_t x = lane; x < 4 * nb; x += 32) dst[x] = st[x];
    __syncwarp();
  }
}


// The haplotype bases' one-hot nibbles (onehot): base x of the batch's
// haplotype buffer at bits 4 (x & 7) .. 4 (x & 7) + 3 of word x >> 3, with
// kNibPad zero words after the last.  The featuriser counts a pair's read-end
// mismatches from 16 of them at a time (end_mismatches).
__global__ void k_hap_nibbles(const uint8_t* __restrict__ hap_bases, long long n_bytes, uint32_t* __restrict__ nib) {
  const long long nw = (n_bytes + 7) / 8 + kNibPad;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < nw; w += (long long)gridDim.x * blockDim.x) {
    uint32_t v = 0;
    const long long x0 = 8 * w;
    if (x0 + 8 <= n_bytes) {
      const uint2 b = *reinterpret_cast<const uint2*>(hap_bases + x0);  // 8-byte aligned: x0 is a multiple of 8
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        v |= onehot((uint8_t)(b.x >> (8 * t))) << (4 * t);
        v |= onehot((uint8_t)(b.y >> (8 * t))) << (4 * (t + 4));
      }
    } else {
      for (int t = 0; t < 8 && x0 + t < n_bytes; ++t) v |= onehot(hap_bases[x0 + t]) << (4 * t);
    }
    nib[w] = v;
  }
}

// Mismatches of n <= 16 read bases against haplotype bases j0 .. j0 + n - 1
// (the haplotype starts at base index ho of the nibble image and has H
// bases); rn holds the read bases' one-hot nibbles (nibble l: the base facing
// haplotype base j0 + l).  A base matches when the nibbles share a bit (N
// matches everything); a position outside the haplotype is a mismatch.  One
// lane, three word loads.
__device__ __forceinline__ int end_mismatches(const uint32_t* __restrict__ nib, int64_t ho, int H, int j0, uint64_t rn,
                                              int n) {
  const int lo = max(0, -j0), hi = min(n, H - j0);  // read positions l in [lo, hi) face the haplotype
  if (hi <= lo) return n;
  const long long x = ho + j0 + lo;                 // >= ho >= 0
  const long long w = x >> 3;
  const int sh = (int)(x & 7) * 4;
  const uint64_t a = (uint64_t)__ldg(nib + w) | ((uint64_t)__ldg(nib + w + 1) << 32);
  const uint64_t c = __ldg(nib + w + 2);
  const uint64_t win = sh ? (a >> sh) | (c << (64 - sh)) : a;  // nibble t: haplotype base j0 + lo + t
  uint64_t t = win & (rn >> (4 * lo));
  t |= t >> 2;
  t |= t >> 1;
  const int len = hi - lo;
  const uint64_t keep = (len >= 16 ? ~0ull : ((1ull << (4 * len)) - 1ull)) & 0x1111111111111111ull;
  return n - __popcll(t & keep);
}

// One-hot nibbles of a read's first and last n = min(16, R) bases (nibble l:
// base l, and base R - n + l), assembled by the warp (lane l < n loads base l
// and base R - n + l).
__device__ __forceinline__ void read_end_nibbles(const uint8_t* __restrict__ rb, int R, bool ok, const uint8_t* oh,
                                                 int lane, uint64_t& pre, uint64_t& suf) {
  const int n = min(16, R);
  const bool on = ok && lane < n;
  const uint32_t np = on ? (uint32_t)oh[rb[lane]] << (4 * (lane & 7)) : 0u;
  const uint32_t ns = on ? (uint32_t)oh[rb[R - n + lane]] << (4 * (lane & 7)) : 0u;
  const uint32_t p_lo = __reduce_or_sync(0xffffffffu, lane < 8 ? np : 0u);
  const uint32_t p_hi = __reduce_or_sync(0xffffffffu, lane < 8 ? 0u : np);
  const uint32_t s_lo = __reduce_or_sync(0xffffffffu, lane < 8 ? ns : 0u);
  const uint32_t s_hi = __reduce_or_sync(0xffffffffu, lane < 8 ? 0u : ns);
  pre = (uint64_t)p_lo | ((uint64_t)p_hi << 32);
  suf = (uint64_t)s_lo | ((uint64_t)s_hi << 32);
}

// Per read: the 2-bit code of the 11-mer starting at each position (or
// kNoCode when it holds a byte other than A/C/G/T), computed once per read
// rather than once per pair.
constexpr uint32_t kNoCode = 0xffffffffu;

__global__ void k_read_kmers(const uint8_t* __restrict__ read_bases, long long n_bytes, uint32_t* __restrict__ codes) {
  // Four positions per thread from four aligned 32-bit loads (bytes x0 ..
  // x0+15; the buffer carries 16 bytes of tail padding), four bytes at a time:
  // the 2-bit code of A C T G is (byte >> 1) & 3 (ConvertChar's order), byte
  // compares give the valid mask.  lo holds base k's code at bits 2k, 2k+1.
  const long long n4 = (n_bytes + 3) / 4;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n4; t += (long long)gridDim.x * blockDim.x) {
    const long long x0 = 4 * t;
    uint32_t lo = 0, valid = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const long long rem = n_bytes - (x0 + 4 * j);
      const uint32_t w = rem > 0 ? *reinterpret_cast<const uint32_t*>(read_bases + x0 + 4 * j) : 0u;
      const uint32_t c4 = (w >> 1) & 0x03030303u;
      uint32_t v4 = __vcmpeq4(w, 0x41414141u) | __vcmpeq4(w, 0x43434343u) | __vcmpeq4(w, 0x47474747u) |
                    __vcmpeq4(w, 0x54545454u);
      if (rem < 4) v4 &= rem <= 0 ? 0u : (0xFFFFFFFFu >> (8 * (4 - rem)));  // bytes past the end
      const uint32_t y = c4 | (c4 >> 6);
      lo |= ((y | (y >> 12)) & 0xFFu) << (8 * j);
      valid |= (((v4 & 0x01010101u) * 0x01020408u) >> 24) << (4 * j);
    }
    uint32_t out[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool ok = x0 + q + kK <= n_bytes && ((valid >> q) & 0x7ffu) == 0x7ffu;
      // bases q .. q+10, first base highest: reverse the 2-bit groups
      uint32_t r = __brev((lo >> (2 * q)) & ((1u << (2 * kK)) - 1u)) >> (32 - 2 * kK);
      r = ((r >> 1) & 0x155555u) | ((r & 0x155555u) << 1);
      out[q] = ok ? r : kNoCode;
    }
    // positions too close to a read's end are masked by the caller
    if (x0 + 4 <= n_bytes) {
      *reinterpret_cast<uint4*>(codes + x0) = make_uint4(out[0], out[1], out[2], out[3]);
    } else {
      for (int q = 0; q < 4 && x0 + q < n_bytes; ++q) codes[x0 + q] = out[q];
    }
  }
}

// Features of a pair.  The read's 11-mers at positions 0, kSeedStride,
// 2 kSeedStride, ... and R - 11 are looked up in the haplotype's table, and
// every shared occurrence votes for diagonal d = j - i; per voted diagonal
// the votes and the first and last sampled read position voting for it are
// kept.  d* is the most voted diagonal (smallest on ties); the features are
// the 64 bins d* - 32 .. d* + 31 divided by the number of read 11-mers, and 16
// scalars: vote totals, lengths, d*'s position, the uncovered read ends
// (t_pre, t_suf), the diagonals of the first and last hit relative to d*, the
// mismatches of the first and last 16 read bases along those diagonals, and
// the voted extent relative to d*.  kmin/kmax are the extreme voted diagonals
// widened by the read ends' triangles: an insertion run in a read end moves
// the alignment one diagonal per row, so below a diagonal whose last hit
// leaves t read bases uncovered (t <= kEndRows, or any t for the read's last
// hit) the band reaches t diagonals down, and likewise up from a diagonal
// whose first hit starts h bases into the read.  Two kernels give the same
// results: a warp per work unit with at most one vote per lane and pair
// (k_featurize_u, below) and, for pairs with repeated 11-mers, a warp per pair
// with a histogram over all diagonals (featurize_pair, k_featurize_slow); both
// share feature_summary.
constexpr int kFeatWarps = kFeatWarpsPerBlock;
constexpr int kHitCap = 256;
constexpr int kEndRows = 24;   // horizon of the per-diagonal end triangles
constexpr int kHistSlots = kBandMaxRead + kBandMaxHap;  // d + R in [0, R + H)
// histogram slot: votes << 18 | first read position << 9 | last read position
// (read positions < 2^9 because reads over kBandMaxRead bases are not banded)
static_assert(kBandMaxRead < 512, "histogram slot packing");

__device__ __forceinline__ void no_seed(const BandParams& p, long long pi, int lane) {
  if (lane == 0) { p.dstar[pi] = INT32_MIN; p.kmin[pi] = INT32_MIN; p.kmax[pi] = INT32_MAX; }
  __nv_bfloat16* f = p.feat + pi * kFeat;
  for (int x = lane; x < kFeat; x += 32) f[x] = __float2bfloat16(0.f);
}

// Sampling stride of a read of R bases: kSeedStride, or wider so that at
// most 32 positions (0, stride, 2 stride, ... and R - 11) are sampled.
__device__ __forceinline__ int seed_stride(int last_pos) { return max(kSeedStride, (last_pos + 30) / 31); }

// The 16 scalar features of a pair (after the 64 histogram bins), as two
// 16-byte stores of BF16 pairs: hits, hits outside the window, read length,
// haplotype length, d*'s position, a constant, the mode's hits, the window's
// non-empty bins, the uncovered read ends, the first and last hit's diagonal
// and the mismatches of the read ends along them, the voted extent.  Both
// featurisers call it, so their outputs agree bit for bit.
__device__ __forceinline__ void write_scalars(__nv_bfloat16* f, int total, int win, int R, int H, int ds, int peak,
                                              int nonzero, float inv, int t_pre, int t_suf, int d_first, int d_last,
                                              int mis_pre, int mis_suf, bool overflow, int dmin, int dmax) {
  const float v[16] = {(float)total * inv,
                       (float)(total - win) * inv,
                       (float)R / 256.f,
                       (float)H / 1024.f,
                       __fdiv_rn((float)(ds + R), (float)(R + H)),
                       1.f,
                       (float)peak * inv,
                       (float)nonzero / (float)kHistBins,
                       (float)t_pre / 32.f,
                       (float)t_suf / 32.f,
                       (float)(d_first - ds) / 32.f,
                       (float)(d_last - ds) / 32.f,
                       (float)mis_pre / 16.f,
                       (float)mis_suf / 16.f,
                       overflow ? -2.f : fmaxf((float)(dmin - ds) / 32.f, -2.f),
                       overflow ? 2.f : fminf((float)(dmax - ds) / 32.f, 2.f)};
  uint32_t w[8];
#pragma unroll
  for (int x = 0; x < 8; ++x) {
    const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * x], v[2 * x + 1]);
    w[x] = *reinterpret_cast<const uint32_t*>(&b2);
  }
  uint4* dst = reinterpret_cast<uint4*>(f + kHistBins);
  dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
  dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

// A seeded pair's scalar block and band bounds, as the summary leaves them to
// one lane (the unit featuriser collects a unit's pairs in lanes 0.. and
// writes them together).  The lane that writes them also counts the read
// ends' mismatches (from the read's end nibbles pre / suf, read_end_nibbles).
// The read (R bases, n_samp sampled positions) is the same for all pairs a
// warp emits together, and the unit featuriser's lane k holds its unit's
// k-th pair (pair index and haplotype follow from k), so none of these is
// part of the block; H = 0 marks an empty one.
struct alignas(16) PairScalars {
  int total, win, H, ds, peak, nonzero, t_pre, t_suf, d_first, d_last, dmin, dmax, kmin, kmax;
  int overflow;
};
__device__ __forceinline__ void emit_scalars(const BandParams& p, const PairScalars& c, long long pi, int h, int R,
                                             int n_samp, uint64_t pre, uint64_t suf) {
  // mismatches of the first / last n read bases along the first / last hit's diagonal
  const int n = min(16, R);
  const int64_t ho = p.batch.hap_off[h];
  const int mis_pre = end_mismatches(p.hap_nib, ho, c.H, c.d_first, pre, n);
  const int mis_suf = end_mismatches(p.hap_nib, ho, c.H, R - n + c.d_last, suf, n);
  write_scalars(p.feat + pi * kFeat, c.total, c.win, R, c.H, c.ds, c.peak, c.nonzero, __frcp_rn((float)n_samp),
                c.t_pre, c.t_suf, c.d_first, c.d_last, mis_pre, mis_suf, c.overflow, c.dmin, c.dmax);
  p.dstar[pi] = c.ds;
  p.kmin[pi] = c.kmin;
  p.kmax[pi] = c.kmax;
}

// The votes of one sampled 11-mer (lane): its table's bucket `bk`, already
// loaded into q, and the buckets after it while they are full; nv counts the
// entries holding the code, v0 is the first one's slot d + R.
__device__ __forceinline__ void probe_votes(const uint32_t* tbl, uint32_t nb, uint32_t code, int i, int R, uint4 q,
                                            uint32_t bk, int& v0, int& nv) {
  v0 = -1;
  nv = 0;
  if (code == kNoCode) return;
  for (uint32_t guard = 0; guard < nb; ++guard) {
    const uint32_t e4[4] = {q.x, q.y, q.z, q.w};
    bool has_free = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (e4[k] == kEmpty) { has_free = true; continue; }
      if ((e4[k] >> 10) == code) {
        if (nv == 0) v0 = (int)(e4[k] & 1023u) - i + R;
        ++nv;
      }
    }
    if (has_free) break;
    bk = bk + 1 == nb ? 0 : bk + 1;
    q = __ldg(reinterpret_cast<const uint4*>(tbl + 4 * bk));
  }
}

__device__ __forceinline__ bool feature_summary(const BandParams& p, long long pi, int R, int H, int h,
                                                const uint32_t* tbl, uint32_t nb, uint32_t code, int i, int stride,
                                                int last_pos, int n_samp, int v0, int nv, uint32_t* hist, int* hits,
                                                int* nhit, uint64_t pre, uint64_t suf, int lane,
                                                PairScalars* out = nullptr, int out_lane = 0);

__device__ void featurize_pair(const BandParams& p, long long pi, int r, int h, const uint32_t* tbl, uint32_t* hist,
                               int* hits, int* nhit, const uint8_t* oh, int lane) {
  const int64_t ro = p.batch.read_off[r], ho = p.batch.hap_off[h];
  const int R = (int)(p.batch.read_off[r + 1] - ro), H = (int)(p.batch.hap_off[h + 1] - ho);
  const uint32_t nb = (uint32_t)(H + 1) / 2;
  const int last_pos = R - kK;
  const int stride = seed_stride(last_pos);
  const int q_s = stride == kSeedStride ? last_pos / kSeedStride : last_pos / stride;
  const int n_samp = q_s + 1 + (q_s * stride != last_pos);  // <= 32
  // lane t looks up the 11-mer at sampled position i: every occurrence in
  // the haplotype is a vote for slot d + R (d = j - i)
  const int i = min(lane * stride, last_pos);
  const uint32_t code = lane < n_samp ? p.read_kmers[ro + i] : kNoCode;
  int v0, nv;
  const uint32_t bk = code != kNoCode ? tbl_bucket(code, nb) : 0u;
  const uint4 q = code != kNoCode ? __ldg(reinterpret_cast<const uint4*>(tbl + 4 * bk)) : make_uint4(0, 0, 0, 0);
  probe_votes(tbl, nb, code, i, R, q, bk, v0, nv);
  uint64_t pre, suf;
  read_end_nibbles(p.batch.read_bases + ro, R, true, oh, lane, pre, suf);
  feature_summary(p, pi, R, H, h, tbl, nb, code, i, stride, last_pos, n_samp, v0, nv, hist, hits, nhit, pre, suf, lane);
}

// Everything after the probes, for both featurisers: the fast path (at most
// one vote per lane) groups lanes by slot; repeated 11-mers (hist != null
// only) build a per-warp histogram over all slots.  Writes the 64 histogram
// features; the pair's scalar block goes to out[out_lane] (shared memory, the
// unit featuriser writes it later) or, without `out`, straight to the pair
// (lane 0).  Returns whether the pair had a seed (false: no_seed wrote it).
__device__ __forceinline__ bool feature_summary(const BandParams& p, long long pi, int R, int H, int h,
                                                const uint32_t* tbl, uint32_t nb, uint32_t code, int i, int stride,
                                                int last_pos, int n_samp, int v0, int nv, uint32_t* hist, int* hits,
                                                int* nhit, uint64_t pre, uint64_t suf, int lane, PairScalars* out,
                                                int out_lane) {
  __nv_bfloat16* f = p.feat + pi * kFeat;
  // summary of the votes: mode (most votes, smallest slot on ties), voted
  // extent, first and last sampled hit (smallest slot on ties), per-diagonal
  // end triangles, vote total, and the 64 histogram bins around the mode
  uint32_t best = 0u, fkey = 0xffffffffu, lkey = 0u;
  int smin = INT32_MAX, smax = -1, tri_lo = INT32_MAX, tri_hi = INT32_MIN, total = 0;
  bool overflow = false;
  int fwin = 0, fnonzero = 0;  // fast path: votes and distinct slots inside the window
  int* wbin = hits;  // 64 bins (fast path)
  const bool fast = !__any_sync(0xffffffffu, nv > 1);
  if (fast) {
    // at most one vote per lane: group the lanes by slot
    const bool valid = nv == 1;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    const unsigned peers = __match_any_sync(0xffffffffu, valid ? v0 : -1);
    const bool lead = valid && (__ffs(peers) - 1) == lane;
    if (valid) {
      const uint32_t c = (uint32_t)__popc(peers);
      best = (c << 16) | (0xffffu - (uint32_t)v0);
      fkey = ((uint32_t)i << 16) | (uint32_t)v0;
      lkey = ((uint32_t)i << 16) | (0xffffu - (uint32_t)v0);
      smin = smax = v0;
    }
    if (lead) {  // the leader is the group's first sampled position, its highest lane the last
      const int la = min((31 - __clz(peers)) * stride, last_pos);
      const int d = v0 - R, tail = R - kK - la, head = i;
      if (tail <= kEndRows) tri_lo = d - tail;
      if (head <= kEndRows) tri_hi = d + head;
    }
    total = __popc(vmask);
    // the first and last sampled hit are the lowest and highest voting lane
    // (sampled positions grow with the lane); the rest are warp reductions
    fkey = __shfl_sync(0xffffffffu, fkey, vmask ? __ffs(vmask) - 1 : 0);
    lkey = __shfl_sync(0xffffffffu, lkey, vmask ? 31 - __clz(vmask) : 0);
    best = __reduce_max_sync(0xffffffffu, best);
    smin = __reduce_min_sync(0xffffffffu, smin);
    smax = __reduce_max_sync(0xffffffffu, smax);
    tri_lo = __reduce_min_sync(0xffffffffu, tri_lo);
    tri_hi = __reduce_max_sync(0xffffffffu, tri_hi);
    {
      const int bs = (int)(0xffffu - (best & 0xffffu));
      const bool inwin = valid && (unsigned)(v0 - (bs - kHistBins / 2)) < (unsigned)kHistBins;
      fwin = __popc(__ballot_sync(0xffffffffu, inwin));
      fnonzero = __popc(__ballot_sync(0xffffffffu, inwin && lead));
    }
    wbin[lane] = 0;
    wbin[lane + 32] = 0;
    __syncwarp();
    if (lead && best != 0u) {
      const int b = v0 - ((int)(0xffffu - (best & 0xffffu)) - kHistBins / 2);
      if (b >= 0 && b < kHistBins) wbin[b] = __popc(peers);
    }
    __syncwarp();
  } else {
    // repeated 11-mers: per-warp histogram in shared memory
    if (lane == 0) *nhit = 0;
    __syncwarp();
    int bk = code != kNoCode ? (int)tbl_bucket(code, nb) : -1;
    for (;;) {
      uint32_t hitmask = 0u;  // slots of the loaded bucket holding this code
      uint4 q = make_uint4(0, 0, 0, 0);
      if (bk >= 0) {
        q = *reinterpret_cast<const uint4*>(tbl + 4 * bk);
        hitmask = ((q.x >> 10) == code && q.x != kEmpty ? 1u : 0u) | ((q.y >> 10) == code && q.y != kEmpty ? 2u : 0u) |
                  ((q.z >> 10) == code && q.z != kEmpty ? 4u : 0u) | ((q.w >> 10) == code && q.w != kEmpty ? 8u : 0u);
        const bool has_free = q.x == kEmpty || q.y == kEmpty || q.z == kEmpty || q.w == kEmpty;
        bk = has_free ? -1 : (bk + 1 == (int)nb ? 0 : bk + 1);
      }
      while (__any_sync(0xffffffffu, hitmask != 0u)) {
        int vote = -1;
        if (hitmask) {
          const int k = __ffs(hitmask) - 1;
          hitmask &= hitmask - 1u;
          const uint32_t e = k == 0 ? q.x : k == 1 ? q.y : k == 2 ? q.z : q.w;
          vote = (int)(e & 1023u) - i + R;  // d + R
        }
        const unsigned vm = __ballot_sync(0xffffffffu, vote >= 0);
        if (vote >= 0) {
          const unsigned peers = __match_any_sync(vm, vote);
          if ((__ffs(peers) - 1) == lane) {
            // one leader per slot; peers' sampled positions are those of their lanes
            const int hl = 31 - __clz(peers);
            const uint32_t n = (uint32_t)__popc(peers);
            const uint32_t i_hi = (uint32_t)min(hl * stride, last_pos);
            const uint32_t old = hist[vote];
            if (old == 0u) {
              hist[vote] = (n << 18) | ((uint32_t)i << 9) | i_hi;
              const int qn = atomicAdd(nhit, 1);
              if (qn < kHitCap) hits[qn] = vote;
            } else {
              const uint32_t fi = min((old >> 9) & 511u, (uint32_t)i), la = max(old & 511u, i_hi);
              hist[vote] = (((old >> 18) + n) << 18) | (fi << 9) | la;
            }
          }
        }
        __syncwarp();
      }
      if (!__any_sync(0xffffffffu, bk >= 0)) break;
    }
    __syncwarp();
    const int nh = min(*nhit, kHitCap);
    overflow = *nhit > kHitCap;
    for (int x = lane; x < nh; x += 32) {
      const int sl = hits[x];
      const uint32_t v = hist[sl], c = v >> 18, fi = (v >> 9) & 511u, la = v & 511u;
      best = max(best, (c << 16) | (0xffffu - (uint32_t)sl));
      fkey = min(fkey, (fi << 16) | (uint32_t)sl);
      lkey = max(lkey, (la << 16) | (0xffffu - (uint32_t)sl));
      smin = min(smin, sl);
      smax = max(smax, sl);
      const int d = sl - R, tail = R - kK - (int)la, head = (int)fi;
      if (tail <= kEndRows) tri_lo = min(tri_lo, d - tail);
      if (head <= kEndRows) tri_hi = max(tri_hi, d + head);
      total += (int)c;
    }
    best = __reduce_max_sync(0xffffffffu, best);
    fkey = __reduce_min_sync(0xffffffffu, fkey);
    lkey = __reduce_max_sync(0xffffffffu, lkey);
    smin = __reduce_min_sync(0xffffffffu, smin);
    smax = __reduce_max_sync(0xffffffffu, smax);
    tri_lo = __reduce_min_sync(0xffffffffu, tri_lo);
    tri_hi = __reduce_max_sync(0xffffffffu, tri_hi);
    total = __reduce_add_sync(0xffffffffu, total);
  }
  if (best == 0u) {
    no_seed(p, pi, lane);
  } else {
    const int best_slot = (int)(0xffffu - (best & 0xffffu));
    const int ds = best_slot - R;
    const int first_i = (int)(fkey >> 16), first_s = (int)(fkey & 0xffffu);
    const int last_i = (int)(lkey >> 16), last_s = (int)(0xffffu - (lkey & 0xffffu));
    const int t_pre = first_i, t_suf = R - kK - last_i;
    const int d_first = first_s - R, d_last = last_s - R;
    tri_lo = min(tri_lo, d_last - t_suf);
    tri_hi = max(tri_hi, d_first + t_pre);
    // 64 histogram bins d* - 32 .. d* + 31, two adjacent bins per lane
    int win = 0, nonzero = 0, peak = 0;
    const float inv = __frcp_rn((float)n_samp);
    int cb[2];
    for (int t = 0; t < 2; ++t) {
      const int s = best_slot - kHistBins / 2 + 2 * lane + t;
      cb[t] = fast ? wbin[2 * lane + t] : (s >= 0 && s < R + H) ? (int)(hist[s] >> 18) : 0;
      win += cb[t];
      nonzero += cb[t] > 0;
      peak = max(peak, cb[t]);
    }
    *reinterpret_cast<__nv_bfloat162*>(f + 2 * lane) = __floats2bfloat162_rn((float)cb[0] * inv, (float)cb[1] * inv);
    if (fast) {
      win = fwin;
      nonzero = fnonzero;
      peak = (int)(best >> 16);  // the mode lies inside the window and has the most votes
    } else {
      win = __reduce_add_sync(0xffffffffu, win);
      nonzero = __reduce_add_sync(0xffffffffu, nonzero);
      peak = __reduce_max_sync(0xffffffffu, peak);
    }
    if (overflow) total = max(total, win);
    // voted extent and end triangles (a hit list overflow widens it to everything)
    const PairScalars c{total, win, H, ds, peak, nonzero, t_pre, t_suf, d_first, d_last,
                        smin - R, smax - R, overflow ? INT32_MIN : min(smin - R, tri_lo),
                        overflow ? INT32_MAX : max(smax - R, tri_hi), overflow};
    if (out) {
      if (lane == 0) out[out_lane] = c;  // the block is warp-uniform
    } else if (lane == 0) {
      emit_scalars(p, c, pi, h, R, n_samp, pre, suf);
    }
  }
  __syncwarp();
  if (!fast) {
    if (overflow) {
      for (int x = lane; x < R + H; x += 32) hist[x] = 0u;
    } else {
      for (int x = lane, nh = min(*nhit, kHitCap); x < nh; x += 32) hist[hits[x]] = 0u;
    }
  }
  __syncwarp();
  return best != 0u;
}

// Slow path: the pairs the unit featuriser handed back (repeated 11-mers,
// diagonals than it keeps), one warp per pair, each warp with a histogram of
// kHistSlots words in global scratch (zero between pairs) and its slot list in
// shared memory; the haplotype tables are read from global memory.
__global__ void __launch_bounds__(kFeatWarps * 32) k_featurize_slow(BandParams p) {
  __shared__ int s_hits[kFeatWarps][kHitCap + 1];
  __shared__ uint8_t s_oh[256];
  for (int x = threadIdx.x; x < 256; x += blockDim.x) s_oh[x] = (uint8_t)onehot((uint8_t)x);
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t* hist = p.feat_hist + ((size_t)blockIdx.x * kFeatWarps + wib) * kHistSlots;
  int* hits = s_hits[wib];
  int* nhit = hits + kHitCap;
  const unsigned long long n = min(p.bctr->feat_slow_count, (unsigned long long)max(p.n_pairs, 1ll));
  if (n == 0) return;
  for (int x = lane; x < kHistSlots; x += 32) hist[x] = 0u;
  __syncwarp();
  for (;;) {
    unsigned long long w = 0;
    if (lane == 0) w = atomicAdd(&p.bctr->feat_slow_next, 1ull);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= n) break;
    const long long pi = p.feat_slow[w];
    const int r = p.pair_read[pi], h = p.pair_hap[pi];
    featurize_pair(p, pi, r, h, p.hap_table + tbl_base(p.batch.hap_off[h], h), hist, hits, nhit, s_oh, lane);
  }
}

// ---------------------------------------------------------------------------
// Unit featuriser: one warp per work unit (a read and up to haps_per_unit of
// its region's haplotypes).  The warp loads the read's sampled 11-mer codes
// once (lane t: sample t), then, kFeatUBatch haplotypes at a time, issues
// every lane's first bucket load for each haplotype before it summarises them
// one by one with the warp featuriser's fast path (match_any groups, one
// REDUX per summary key; the first and last hit by lane).  A pair's scalar
// block waits in shared memory; 32 pairs (or the unit's last) are written
// together, lane k writing pair k and counting its read-end mismatches from
// the haplotype nibble image (end_mismatches) -- one lane per pair instead of
// a warp-wide load and ballot.  A pair for which some lane sees the same
// 11-mer more than once goes to the slow list (k_featurize_slow).
// Grid-strided over the units: consecutive warps take consecutive units, so a
// region's tables are read by warps running at the same time and stay in L2.
// Four blocks per SM (64 registers, a few spilled) beat three (80, none):
// the kernel is issue-bound and more warps hide the bucket loads.
// ---------------------------------------------------------------------------
constexpr int kFeatUWarps = 8;   // warps per block
constexpr int kFeatUBatch = 2;   // haplotypes whose bucket loads are in flight together
constexpr int kFeatUBlocksPerSm = 4;

__global__ void __launch_bounds__(kFeatUWarps * 32, kFeatUBlocksPerSm) k_featurize_u(BandParams p) {
  __shared__ int s_bins[kFeatUWarps][kHistBins];
  __shared__ PairScalars s_ps[kFeatUWarps][32];  // the scalar blocks of a warp's current 32 pairs
  __shared__ uint8_t s_oh[256];
  for (int x = threadIdx.x; x < 256; x += blockDim.x) s_oh[x] = (uint8_t)onehot((uint8_t)x);
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int* bins = s_bins[wib];
  const long long nwarps = (long long)gridDim.x * kFeatUWarps;
  for (long long u = blockIdx.x * (long long)kFeatUWarps + wib; u < p.n_units; u += nwarps) {
    const Unit un = p.units[u];
    const int64_t ro = p.batch.read_off[un.read];
    const int R = (int)(p.batch.read_off[un.read + 1] - ro);
    const bool read_ok = R >= kK && R <= kBandMaxRead;
    const int last_pos = R - kK;
    const int stride = read_ok ? seed_stride(last_pos) : 1;
    const int q_s = read_ok ? last_pos / stride : 0;
    const int n_samp = read_ok ? q_s + 1 + (q_s * stride != last_pos) : 0;  // <= 32
    const int i = read_ok ? min(lane * stride, last_pos) : 0;
    const uint32_t code = lane < n_samp ? __ldg(p.read_kmers + ro + i) : kNoCode;
    // once per unit: lane k's haplotype offset hap_off[hap0 + k] (k <= 31),
    // and the one-hot nibbles of the read's first and last 16 bases for the
    // end-mismatch counts
    const int64_t unit_off = lane <= min(un.nh, 31) ? p.batch.hap_off[un.hap0 + lane] : 0;
    uint64_t pre, suf;
    read_end_nibbles(p.batch.read_bases + ro, R, read_ok, s_oh, lane, pre, suf);
    // the scalar block of the unit's pair k waits in slot k & 31 until 32
    // pairs (or the unit's last) are written together, lane k writing pair k
    PairScalars* ps = s_ps[wib];
    unsigned filled = 0u;  // slots holding a seeded pair
    for (int k0 = 0; k0 < un.nh; k0 += kFeatUBatch) {
      uint4 q[kFeatUBatch];
      uint32_t bk[kFeatUBatch];
      int64_t hos[kFeatUBatch];
      int Hs[kFeatUBatch];
#pragma unroll
      for (int t = 0; t < kFeatUBatch; ++t) {
        const int k = k0 + t;
        const int kk = min(k, un.nh - 1);
        const int h = un.hap0 + kk;
        const int64_t o0 = __shfl_sync(0xffffffffu, unit_off, kk & 31), o1 = __shfl_sync(0xffffffffu, unit_off, (kk + 1) & 31);
        hos[t] = kk + 1 <= 31 ? o0 : p.batch.hap_off[h];
        Hs[t] = (int)((kk + 1 <= 31 ? o1 : p.batch.hap_off[h + 1]) - hos[t]);
        const bool ok = k < un.nh && read_ok && Hs[t] >= kK && Hs[t] <= kBandMaxHap && code != kNoCode;
        bk[t] = ok ? tbl_bucket(code, (uint32_t)(Hs[t] + 1) / 2) : 0u;
        q[t] = ok ? __ldg(reinterpret_cast<const uint4*>(p.hap_table + tbl_base(hos[t], h) + 4 * bk[t]))
                  : make_uint4(0, 0, 0, 0);
      }
#pragma unroll
      for (int t = 0; t < kFeatUBatch; ++t) {
        const int k = k0 + t;
        if (k >= un.nh) break;
        const int h = un.hap0 + k;
        const long long pi = un.out0 + k;
        const int64_t ho = hos[t];
        const int H = Hs[t];
        if (!read_ok || H < kK || H > kBandMaxHap) {
          no_seed(p, pi, lane);
          continue;
        }
        const uint32_t* tbl = p.hap_table + tbl_base(ho, h);
        const uint32_t nb = (uint32_t)(H + 1) / 2;
        int v0, nv;
        probe_votes(tbl, nb, code, i, R, q[t], bk[t], v0, nv);
        if (__any_sync(0xffffffffu, nv > 1)) {
          if (lane == 0) {
            const unsigned long long at = atomicAdd(&p.bctr->feat_slow_count, 1ull);
            if (at < (unsigned long long)p.n_pairs) p.feat_slow[at] = pi;
          }
          continue;
        }
        if (feature_summary(p, pi, R, H, h, tbl, nb, code, i, stride, last_pos, n_samp, v0, nv, nullptr, bins, nullptr,
                            pre, suf, lane, ps, k & 31))
          filled |= 1u << (k & 31);

        if ((k & 31) == 31) {
          __syncwarp();
          if (filled >> lane & 1u) emit_scalars(p, ps[lane], un.out0 + (k - 31) + lane, un.hap0 + (k - 31) + lane, R, n_samp, pre, suf);
          filled = 0u;
          __syncwarp();
        }
      }
    }
    __syncwarp();
    if (filled >> lane & 1u) {
      const int base = (un.nh - 1) & ~31;  // the last round's first pair
      emit_scalars(p, ps[lane], un.out0 + base + lane, un.hap0 + base + lane, R, n_samp, pre, suf);
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Routing.  Pass 0 counts band items per (width class, read-length bucket)
// and writes full-DP fallback units; pass 1 places band items at their
// bucket's offset so that each warp of the banded kernel gets reads of nearly
// equal length.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int full_variant(int R) {
  const int rt = (rows_needed(R, true, true) + 31) / 32;
  return rt <= 8 ? rt - 1 : 8;  // k_forward<float, rt, single> or the multi-strip variant
}

__device__ __forceinline__ bool route_band(const BandParams& p, long long pi, int R, int H, int& cls, int& d_lo) {
  const int ds = p.dstar[pi];
  if (ds == INT32_MIN || R > kBandMaxRead || R == 0 || H == 0) return false;
  float lo, hi;
  if (p.use_mlp) {
    lo = p.mlp_out[pi * kOut + 0];
    hi = p.mlp_out[pi * kOut + 1];
    if (!(lo <= hi) || !isfinite(lo) || !isfinite(hi)) return false;
  } else {
    lo = -(float)p.fixed_half;
    hi = (float)p.fixed_half;
  }
  // band in absolute diagonals, widened to hold every shared 11-mer diagonal
  const int km = p.kmin[pi], kx = p.kmax[pi];
  if (km == INT32_MIN || kx == INT32_MAX) return false;
  const int blo = min(ds + (int)floorf(lo) - p.margin, km), bhi = max(ds + (int)ceilf(hi) + p.margin, kx);
  const int width = bhi - blo + 1;
  if (width > band_width(kBandWidths - 1) || width < 1) return false;
  cls = (width - 1) / 8;  // band_width(cls) = 8 (cls + 1) >= width
  d_lo = blo - (band_width(cls) - width) / 2;
  return true;
}

// Block-aggregated: per-block shared counters, one global atomic per
// (counter, block); pass 1 reserves each bucket's range for the block at once.
constexpr int kSlotFull = kBandWidths * kRBuckets;
constexpr int kRouteSlots = kSlotFull + 9;

__global__ void __launch_bounds__(256) k_band_route(BandParams p, int pass) {
  __shared__ unsigned int cnt[kRouteSlots];
  __shared__ unsigned long long base[kRouteSlots];
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long pi0 = blockIdx.x * (long long)blockDim.x; pi0 < p.n_pairs; pi0 += stride) {
    for (int x = threadIdx.x; x < kRouteSlots; x += blockDim.x) cnt[x] = 0;
    __syncthreads();
    const long long pi = pi0 + threadIdx.x;
    int slot = -1;
    unsigned local = 0;
    int r = 0, h = 0, d_lo = 0, R = 0, cls = 0;
    bool band = false;
    if (pi < p.n_pairs) {
      r = p.pair_read[pi];
      h = p.pair_hap[pi];
      R = (int)(p.batch.read_off[r + 1] - p.batch.read_off[r]);
      const int H = (int)(p.batch.hap_off[h + 1] - p.batch.hap_off[h]);
      band = route_band(p, pi, R, H, cls, d_lo);
      slot = band ? cls * kRBuckets + min(R / kRBucketRows, kRBuckets - 1) : kSlotFull + full_variant(R);
      if (pass == 0 && p.banded) p.banded[pi] = 0;  // set by band_outcome when the band's result stands
      if (pass == 0 || band) local = atomicAdd(&cnt[slot], 1u);
    }
    __syncthreads();
    for (int x = threadIdx.x; x < kRouteSlots; x += blockDim.x) {
      const unsigned c = cnt[x];
      if (c == 0) continue;
      if (x < kSlotFull) {
        const int cl = x / kRBuckets, bucket = x % kRBuckets;
        if (pass == 0) atomicAdd(&p.bctr->band_count[cl][bucket], (unsigned long long)c);
        else base[x] = atomicAdd(&p.bctr->band_fill[cl][bucket], (unsigned long long)c);
      } else if (pass == 0) {
        base[x] = atomicAdd(&p.bctr->full_count[x - kSlotFull], (unsigned long long)c);
        atomicAdd(&p.bctr->fallback_route, (unsigned long long)c);
      }
    }
    __syncthreads();
    if (pi < p.n_pairs) {
      if (band && pass == 1) {
        BandItem it;
        it.read = r; it.hap = h; it.out = pi; it.d_lo = d_lo; it.pad_ = 0;
        p.items[(size_t)cls * p.item_cap + base[slot] + local] = it;
      } else if (!band && pass == 0) {
        const int v = slot - kSlotFull;
        const unsigned long long q = base[slot] + local;
        if (q < (unsigned long long)p.full_cap) {
          Unit u{};
          u.read = r; u.hap0 = h; u.nh = 1; u.out0 = pi;
          p.full_items[(size_t)v * p.full_cap + q] = u;
        } else {
          atomicOr(&p.ctr->status, 4ull);
        }
      }
      if (band && pass == 0 && p.audit_period > 0 && pi % p.audit_period == 0) {
        const unsigned long long a = atomicAdd(&p.bctr->audit_count, 1ull);
        if (a < (unsigned long long)p.audit_cap) p.audit_pairs[a] = pi;
      }
    }
    __syncthreads();
  }
}

// exclusive prefix over buckets, per width class
__global__ void k_band_scan(BandCounters* c) {
  if (threadIdx.x < kBandWidths) {
    unsigned long long acc = 0;
    for (int b = 0; b < kRBuckets; ++b) {
      c->band_fill[threadIdx.x][b] = acc;
      acc += c->band_count[threadIdx.x][b];
    }
    c->band_total[threadIdx.x] = acc;
  }
}

// A banded pair's outcome: promotion to the next wider class (a single item
// centred on this band), the full DP (edge check failed at W = 32, or the
// banded sum is not positive -- NaN included), the FP64 list, or its log10
// result.
__device__ __forceinline__ void band_outcome(const BandParams& p, int cls, const BandItem& it, int R, float tot,
                                             bool fall_back, bool rescue) {
  if (fall_back && cls + 1 < kBandWidths) {
    const unsigned long long q = atomicAdd(&p.bctr->promoted[cls + 1], 1ull);
    const unsigned long long at = p.bctr->band_total[cls + 1] + q;
    if (at < (unsigned long long)p.item_cap) {
      BandItem ni = it;
      ni.d_lo = it.d_lo - (band_width(cls + 1) - band_width(cls)) / 2;
      p.items[(size_t)(cls + 1) * p.item_cap + at] = ni;
    } else {
      atomicOr(&p.ctr->status, 4ull);
    }
  } else if (fall_back) {
    const int v = full_variant(R);
    const unsigned long long q = atomicAdd(&p.bctr->full_count[v], 1ull);
    atomicAdd(&p.bctr->fallback_edge, 1ull);
    if (q < (unsigned long long)p.full_cap) {
      Unit u{};
      u.read = it.read; u.hap0 = it.hap; u.nh = 1; u.out0 = it.out;
      p.full_items[(size_t)v * p.full_cap + q] = u;
    } else {
      atomicOr(&p.ctr->status, 4ull);
    }
  } else if (rescue) {
    const unsigned long long slot = atomicAdd(&p.ctr->rescue_count, 1ull);
    if (slot < (unsigned long long)p.rescue_cap) {
      p.rescue[slot].read = it.read;
      p.rescue[slot].hap = it.hap;
      p.rescue[slot].out = it.out;
    } else {
      atomicOr(&p.ctr->status, 1ull);
    }
    p.out[it.out] = __longlong_as_double(0x7ff8000000000000ll);
  } else {
    p.out[it.out] = (double)(log10f(tot) - p.tables->log10_init_f);
    if (p.banded) p.banded[it.out] = 1;
  }
}

// Row constants of the banded recurrence, from the row's quality bytes and
// the row above's pMX / pMY.  The kernels compute them one row ahead, with the
// quality bytes loaded two rows ahead, so the table lookups overlap the
// previous row's cells.
__device__ __forceinline__ int mm_index(int qi, int qd) {
  const int mx = max(qi, qd), mn = min(qi, qd);
  return ((mx * (mx + 1)) >> 1) + mn;
}

// Folded form (as the full-DP kernels): pMM(r) is folded into the row's
// emissions and cx, cy carry 1/pMM, so an M update is two FMAs and a
// multiply.  A row whose pMM is below kFoldMin cannot be folded: its 1/pMM
// table entry is NaN, which makes the banded sums NaN, and such pairs end in
// the full DP (which keeps the plain form for them) like any pair whose
// banded sum is not positive.
// Stages the probability tables the band kernels read per row into shared memory.
struct BandSmem {
  QProb qp[128];
  uint8_t oh[256];  // one-hot nibble of every byte (onehot)
  float mm[kMMEntries];
};
__device__ __forceinline__ void stage_band_tables(BandSmem& sm, const Tables* tb) {
  for (int x = threadIdx.x; x < 128; x += blockDim.x) sm.qp[x] = tb->qp[x];
  for (int x = threadIdx.x; x < 256; x += blockDim.x) sm.oh[x] = (uint8_t)onehot((uint8_t)x);
  for (int x = threadIdx.x; x < kMMEntries; x += blockDim.x) sm.mm[x] = tb->mm_f[x];
  __syncthreads();
}
struct FwdRow {
  float cx, cy, kap, g, pmx, pmy, em, ex;
  uint32_t rb;  // the read base's one-hot nibble, replicated 8 times
};
__device__ __forceinline__ FwdRow fwd_row(const BandSmem& sm, const float* __restrict__ minv, uchar4 qv, uint8_t base,
                                          float ap, float bp) {
  const QProb* qp = sm.qp;
  const float* mmt = sm.mm;
  FwdRow c;
  const int qi = qv.y & kQualMask, qd = qv.z & kQualMask;
  const QProb qpi = qp[qi], qpg = qp[qv.w & kQualMask], qpb = qp[qv.x & kQualMask];
  c.pmx = qpi.p;
  c.pmy = qp[qd].p;
  c.g = qpg.p;
  const float gp = qpg.q;
  const int mi = mm_index(qi, qd);
  const float mm = mmt[mi], inv = __ldg(minv + mi);
  c.cx = gp * ap * inv;
  c.cy = gp * bp * inv;
  c.kap = c.g * ap * qpi.inv;
  c.em = qpb.q * mm;
  c.ex = qpb.third * mm;
  c.rb = (uint32_t)sm.oh[base] * 0x11111111u;
  return c;
}

// Rows 2 .. R of a read whose insertion, deletion and gap-continuation
// qualities are the same on every base (the batch's, checked by k_gap_check):
// the transition constants of those rows are those of fwd_row with the
// previous row's pMX / pMY equal to this row's, computed once (u); only the
// emissions follow the base and its quality -- the same operations on the
// same values as fwd_row, so the same bits.
struct UniRows {
  FwdRow u;  // transition constants of rows >= 2
  float mm;  // the rows' match-to-match probability
};
__device__ __forceinline__ UniRows uni_rows(const BandSmem& sm, const float* __restrict__ minv, uchar4 q0) {
  const int qi = q0.y & kQualMask, qd = q0.z & kQualMask;
  UniRows r;
  r.u = fwd_row(sm, minv, q0, (uint8_t)'A', sm.qp[qi].p, sm.qp[qd].p);
  r.mm = sm.mm[mm_index(qi, qd)];
  return r;
}
__device__ __forceinline__ FwdRow uni_row(const BandSmem& sm, const UniRows& ur, uchar4 qv, uint8_t base) {
  FwdRow c = ur.u;
  const QProb qpb = sm.qp[qv.x & kQualMask];
  c.em = qpb.q * ur.mm;
  c.ex = qpb.third * ur.mm;
  c.rb = (uint32_t)sm.oh[base] * 0x11111111u;
  return c;
}

// ---------------------------------------------------------------------------
// Ring test.  A pair banded on [d_lo, d_lo + W) is also scored on the band
// widened by a ring of four diagonals on each side (eight for W >= 16); the
// wider band's likelihood is the result, and the pair is promoted to the next
// class (whose band is centred on this one) when the ring adds more than
// edge_threshold of it.  Unlike a posterior test on the band's edge
// diagonals, the ring also sees mass that enters the band from outside (an
// alignment start or end on a diagonal next to the band), which a banded
// model cannot represent.  W = 8, 16 run both bands in one row sweep (shared
// row constants and emissions); W = 24, 32 run them one after the other.
// ---------------------------------------------------------------------------
template <int WB, int WI, bool UNI>
__device__ __forceinline__ float2 band_forward_body(const BandSmem& sm, const Tables* tb, const uchar4* __restrict__ quals,
                                               const uint8_t* __restrict__ rbase, const uint8_t* __restrict__ hap,
                                               int R, int H, int d, const UniRows& ur) {
  constexpr int NW = WB / 8;
  constexpr int OFF = (WB - WI) / 2;  // inner band = outer diagonals OFF .. OFF + WI - 1
  constexpr int WIN = WI > 0 ? WI : 1;
  float M[WB], X[WB], Y[WB], Mi[WIN], Xi[WIN], Yi[WIN];
  const float init_y = tb->init_f / (float)H;
#pragma unroll
  for (int k = 0; k < WB; ++k) {
    const int c = d + k;
    M[k] = 0.f; X[k] = 0.f;
    Y[k] = (c >= 0 && c <= H) ? init_y : 0.f;
  }
#pragma unroll
  for (int k = 0; k < WIN; ++k) {
    const int c = d + OFF + k;
    Mi[k] = 0.f; Xi[k] = 0.f;
    Yi[k] = (WI > 0 && c >= 0 && c <= H) ? init_y : 0.f;
  }
  uint32_t win[NW];  // row 1: columns d + 1 + k
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    uint32_t v = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const int c = d + 1 + w * 8 + t;
      v |= ((c >= 1 && c <= H) ? (uint32_t)sm.oh[hap[c - 1]] : 0u) << (4 * t);
    }
    win[w] = v;
  }
  float pmx_last = 1.f;
  FwdRow cur = fwd_row(sm, tb->mm_inv_f, quals[0], rbase[0], 1.f, 1.f);  // row 1; row 0 has pMX = pMY = 1
  uchar4 qn = quals[min(1, R - 1)];
  uint8_t bn = rbase[min(1, R - 1)];
  for (int r = 1; r <= R; ++r) {
    // row r + 1 (unused after row R)
    const FwdRow nxt = UNI ? uni_row(sm, ur, qn, bn) : fwd_row(sm, tb->mm_inv_f, qn, bn, cur.pmx, cur.pmy);
    {
      const int rn = min(r + 1, R - 1);  // row r + 2
      qn = quals[rn];
      bn = rbase[rn];
    }
    const int cn = r + 1 + d + WB - 1;  // next row's window: shift, append column cn
    const uint8_t hb = (cn >= 1 && cn <= H) ? hap[cn - 1] : (uint8_t)0;
    float lm = 0.f, ly = 0.f, lmi = 0.f, lyi = 0.f;
#pragma unroll
    for (int k = 0; k < WB; ++k) {
      const bool match = (win[k >> 3] & cur.rb & (0xFu << (4 * (k & 7)))) != 0u;
      const float e = match ? cur.em : cur.ex;
      {
        const float upm = (k + 1 < WB) ? M[k + 1] : 0.f;
        const float upx = (k + 1 < WB) ? X[k + 1] : 0.f;
        const float mn = e * __fmaf_rn(cur.cy, Y[k], __fmaf_rn(cur.cx, X[k], M[k]));
        const float xn = __fmaf_rn(cur.kap, upx, upm);
        const float yn = __fmaf_rn(cur.g, ly, lm);
        M[k] = mn; X[k] = xn; Y[k] = yn;
        lm = mn; ly = yn;
      }
      if constexpr (WI > 0) {
        if (k >= OFF && k < OFF + WI) {
          const int ki = k - OFF;
          const float upm = (ki + 1 < WI) ? Mi[ki + 1] : 0.f;
          const float upx = (ki + 1 < WI) ? Xi[ki + 1] : 0.f;
          const float mn = e * __fmaf_rn(cur.cy, Yi[ki], __fmaf_rn(cur.cx, Xi[ki], Mi[ki]));
          const float xn = __fmaf_rn(cur.kap, upx, upm);
          const float yn = __fmaf_rn(cur.g, lyi, lmi);
          Mi[ki] = mn; Xi[ki] = xn; Yi[ki] = yn;
          lmi = mn; lyi = yn;
        }
      }
    }
    const uint32_t nib = (cn >= 1 && cn <= H) ? (uint32_t)sm.oh[hb] : 0u;
#pragma unroll
    for (int w = 0; w < NW - 1; ++w) win[w] = __funnelshift_r(win[w], win[w + 1], 4);
    win[NW - 1] = (win[NW - 1] >> 4) | (nib << 28);
    pmx_last = cur.pmx;
    cur = nxt;
  }
  float tot = 0.f, toti = 0.f;
#pragma unroll
  for (int k = 0; k < WB; ++k) {
    const int c = R + d + k;
    tot += (c >= 1 && c <= H) ? M[k] + pmx_last * X[k] : 0.f;
  }
#pragma unroll
  for (int k = 0; k < WIN; ++k) {
    const int c = R + d + OFF + k;
    toti += (WI > 0 && c >= 1 && c <= H) ? Mi[k] + pmx_last * Xi[k] : 0.f;
  }
  return make_float2(tot, toti);
}

// The same two sweeps with the inner band's cells packed beside the outer
// band's: the inner band (diagonals OFF .. OFF + WI - 1 of the outer band) is
// the same matrix cells under another DP, with the same emission and row
// constants, so each such cell updates both DPs with packed FP32x2
// operations (fma.rn.f32x2 of sm_100) -- each half the scalar operation
// sequence, so the results are bit-identical to band_forward_body.  Outer
// cells without an inner twin (the rings) stay scalar.
template <int WB, int WI, bool UNI>
__device__ __forceinline__ float2 band_forward_paired(const BandSmem& sm, const Tables* tb,
                                                      const uchar4* __restrict__ quals,
                                                      const uint8_t* __restrict__ rbase, const uint8_t* __restrict__ hap,
                                                      int R, int H, int d, const UniRows& ur) {
  constexpr int NW = WB / 8;
  constexpr int OFF = (WB - WI) / 2;   // outer cells 0 .. OFF-1: lower ring; OFF+WI .. WB-1: upper ring
  constexpr int NHI = WB - OFF - WI;
  static_assert(WI > 0 && OFF > 0 && NHI > 0, "paired sweep needs rings on both sides");
  float Ml[OFF], Xl[OFF], Yl[OFF];     // lower ring (outer only)
  float2 P_M[WI], P_X[WI], P_Y[WI];    // .x outer cell OFF + k, .y inner cell k
  float Mh[NHI], Xh[NHI], Yh[NHI];     // upper ring (outer only)
  const float init_y = tb->init_f / (float)H;
  auto y0 = [&](int k) { const int c = d + k; return (c >= 0 && c <= H) ? init_y : 0.f; };
#pragma unroll
  for (int k = 0; k < OFF; ++k) { Ml[k] = 0.f; Xl[k] = 0.f; Yl[k] = y0(k); }
#pragma unroll
  for (int k = 0; k < WI; ++k) {
    P_M[k] = make_float2(0.f, 0.f);
    P_X[k] = make_float2(0.f, 0.f);
    const float y = y0(OFF + k);
    P_Y[k] = make_float2(y, y);
  }
#pragma unroll
  for (int k = 0; k < NHI; ++k) { Mh[k] = 0.f; Xh[k] = 0.f; Yh[k] = y0(OFF + WI + k); }
  uint32_t win[NW];  // row 1: columns d + 1 + k
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    uint32_t v = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const int c = d + 1 + w * 8 + t;
      v |= ((c >= 1 && c <= H) ? (uint32_t)sm.oh[hap[c - 1]] : 0u) << (4 * t);
    }
    win[w] = v;
  }
  float pmx_last = 1.f;
  FwdRow cur = fwd_row(sm, tb->mm_inv_f, quals[0], rbase[0], 1.f, 1.f);
  uchar4 qn = quals[min(1, R - 1)];
  uint8_t bn = rbase[min(1, R - 1)];
  for (int r = 1; r <= R; ++r) {
    const FwdRow nxt = UNI ? uni_row(sm, ur, qn, bn) : fwd_row(sm, tb->mm_inv_f, qn, bn, cur.pmx, cur.pmy);
    {
      const int rn = min(r + 1, R - 1);
      qn = quals[rn];
      bn = rbase[rn];
    }
    const int cn = r + 1 + d + WB - 1;
    const uint8_t hb = (cn >= 1 && cn <= H) ? hap[cn - 1] : (uint8_t)0;
    const float2 cx2 = make_float2(cur.cx, cur.cx), cy2 = make_float2(cur.cy, cur.cy);
    const float2 kap2 = make_float2(cur.kap, cur.kap), g2 = make_float2(cur.g, cur.g);
    auto emis = [&](int k) {
      const bool match = (win[k >> 3] & cur.rb & (0xFu << (4 * (k & 7)))) != 0u;
      return match ? cur.em : cur.ex;
    };
    float lm = 0.f, ly = 0.f;
    // lower ring
#pragma unroll
    for (int k = 0; k < OFF; ++k) {
      const float e = emis(k);
      const float upm = k + 1 < OFF ? Ml[k + 1] : P_M[0].x;
      const float upx = k + 1 < OFF ? Xl[k + 1] : P_X[0].x;
      const float mn = e * __fmaf_rn(cur.cy, Yl[k], __fmaf_rn(cur.cx, Xl[k], Ml[k]));
      const float xn = __fmaf_rn(cur.kap, upx, upm);
      const float yn = __fmaf_rn(cur.g, ly, lm);
      Ml[k] = mn; Xl[k] = xn; Yl[k] = yn;
      lm = mn; ly = yn;
    }
    // paired cells: the inner band's row starts with no left neighbour
    float2 lm2 = make_float2(lm, 0.f), ly2 = make_float2(ly, 0.f);
#pragma unroll
    for (int k = 0; k < WI; ++k) {
      const float e = emis(OFF + k);
      const float2 upm = k + 1 < WI ? P_M[k + 1] : make_float2(Mh[0], 0.f);
      const float2 upx = k + 1 < WI ? P_X[k + 1] : make_float2(Xh[0], 0.f);
      const float2 t = __ffma2_rn(cy2, P_Y[k], __ffma2_rn(cx2, P_X[k], P_M[k]));
      const float2 mn = make_float2(e * t.x, e * t.y);
      const float2 xn = __ffma2_rn(kap2, upx, upm);
      const float2 yn = __ffma2_rn(g2, ly2, lm2);
      P_M[k] = mn; P_X[k] = xn; P_Y[k] = yn;
      lm2 = mn; ly2 = yn;
    }
    lm = lm2.x;
    ly = ly2.x;
    // upper ring
#pragma unroll
    for (int k = 0; k < NHI; ++k) {
      const float e = emis(OFF + WI + k);
      const float upm = k + 1 < NHI ? Mh[k + 1] : 0.f;
      const float upx = k + 1 < NHI ? Xh[k + 1] : 0.f;
      const float mn = e * __fmaf_rn(cur.cy, Yh[k], __fmaf_rn(cur.cx, Xh[k], Mh[k]));
      const float xn = __fmaf_rn(cur.kap, upx, upm);
      const float yn = __fmaf_rn(cur.g, ly, lm);
      Mh[k] = mn; Xh[k] = xn; Yh[k] = yn;
      lm = mn; ly = yn;
    }
    const uint32_t nib = (cn >= 1 && cn <= H) ? (uint32_t)sm.oh[hb] : 0u;
#pragma unroll
    for (int w = 0; w < NW - 1; ++w) win[w] = __funnelshift_r(win[w], win[w + 1], 4);
    win[NW - 1] = (win[NW - 1] >> 4) | (nib << 28);
    pmx_last = cur.pmx;
    cur = nxt;
  }
  // last row sums, in the scalar body's order (outer cells 0 .. WB-1, then inner 0 .. WI-1)
  float tot = 0.f, toti = 0.f;
#pragma unroll
  for (int k = 0; k < WB; ++k) {
    const int c = R + d + k;
    const float m = k < OFF ? Ml[k] : k < OFF + WI ? P_M[k - OFF].x : Mh[k - OFF - WI];
    const float x = k < OFF ? Xl[k] : k < OFF + WI ? P_X[k - OFF].x : Xh[k - OFF - WI];
    tot += (c >= 1 && c <= H) ? m + pmx_last * x : 0.f;
  }
#pragma unroll
  for (int k = 0; k < WI; ++k) {
    const int c = R + d + OFF + k;
    toti += (c >= 1 && c <= H) ? P_M[k].y + pmx_last * P_X[k].y : 0.f;
  }
  return make_float2(tot, toti);
}

// One band alone, not inlined: the two passes of the wider classes then hold
// one band's state at a time.
template <int WB, bool UNI>
__device__ __noinline__ float band_forward_pass(const BandSmem& sm, const Tables* tb, const uchar4* quals,
                                                const uint8_t* rbase, const uint8_t* hap, int R, int H, int d,
                                                const UniRows& ur) {
  return band_forward_body<WB, 0, UNI>(sm, tb, quals, rbase, hap, R, H, d, ur).x;
}

// W = 8 keeps three blocks per SM (up to 168 registers); the wider classes two.
template <int W>
__global__ void __launch_bounds__(128, W <= 8 ? 3 : 2) k_band_ring_f32(BandParams p, int cls) {
  constexpr bool kDual = W <= 16;  // both bands in one sweep
  // ring width on each side: pairs routed to wider bands have indel-rich alignments whose
  // alternatives lie farther out, so W >= 16 test eight diagonals
  constexpr int kRing = W >= 16 ? 8 : 4;
  const Tables* tb = p.tables;
  __shared__ BandSmem sm;
  stage_band_tables(sm, tb);
  // uniform gap qualities over the batch (k_gap_check ran): one set of row constants.  Not for
  // W = 16: compiled with both row paths it holds 227 registers instead of 219 and ran slower
  const bool uni = W != 16 && p.bctr->gap_checked != 0u && p.bctr->gap_mixed == 0u;
  const UniRows ur = uni_rows(sm, tb->mm_inv_f, p.batch.read_quals[0]);
  // routed items (bucketed by read length), then items promoted from the next narrower class
  const unsigned long long total =
      p.bctr->band_total[cls] + min(p.bctr->promoted[cls], (unsigned long long)p.item_cap - p.bctr->band_total[cls]);
  const BandItem* items = p.items + (size_t)cls * p.item_cap;
  const unsigned long long nthreads = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  unsigned long long cells = 0, rcells = 0;
  for (unsigned long long ii = tid; ii < total; ii += nthreads) {
    const BandItem it = items[ii];
    const int64_t ro = p.batch.read_off[it.read], ho = p.batch.hap_off[it.hap];
    const int R = (int)(p.batch.read_off[it.read + 1] - ro), H = (int)(p.batch.hap_off[it.hap + 1] - ho);
    const uchar4* quals = p.batch.read_quals + ro;
    const uint8_t* rbase = p.batch.read_bases + ro;
    const uint8_t* hap = p.batch.hap_bases + ho;
    float lin, lout;
    if constexpr (kDual) {
      const float2 t = uni ? band_forward_paired<W + 2 * kRing, W, true>(sm, tb, quals, rbase, hap, R, H, it.d_lo - kRing, ur)
                           : band_forward_paired<W + 2 * kRing, W, false>(sm, tb, quals, rbase, hap, R, H, it.d_lo - kRing, ur);
      lout = t.x;
      lin = t.y;
    } else if (uni) {
      lin = band_forward_pass<W, true>(sm, tb, quals, rbase, hap, R, H, it.d_lo, ur);
      lout = band_forward_pass<W + 2 * kRing, true>(sm, tb, quals, rbase, hap, R, H, it.d_lo - kRing, ur);
    } else {
      lin = band_forward_pass<W, false>(sm, tb, quals, rbase, hap, R, H, it.d_lo, ur);
      lout = band_forward_pass<W + 2 * kRing, false>(sm, tb, quals, rbase, hap, R, H, it.d_lo - kRing, ur);
    }
    cells += (unsigned long long)R * (2 * W + 2 * kRing);
    rcells += (unsigned long long)R * (W + 2 * kRing);
    bool fall_back = !(lout > 0.f);
    const bool rescue = !fall_back && (!(lout >= (float)kMinAccepted) || isinf(lout));
    // the ring's share of the outer likelihood (NaN or a negative share fall back too)
    if (!fall_back && !rescue) fall_back = !(lout - lin <= p.edge_threshold * lout && lin >= 0.f);
    band_outcome(p, cls, it, R, lout, fall_back, rescue);
  }
  for (int o = 16; o > 0; o >>= 1) {
    cells += __shfl_xor_sync(0xffffffffu, cells, o);
    rcells += __shfl_xor_sync(0xffffffffu, rcells, o);
  }
  if ((threadIdx.x & 31) == 0 && cells) {
    atomicAdd(&p.bctr->band_cells, cells);
    atomicAdd(&p.bctr->band_result_cells, rcells);
  }
}

// Marks the batch whose read bases all carry the first base's insertion,
// deletion and gap-continuation qualities (Biovoltron's SamRecord fills those
// from constant strings): the banded kernels then take every row's transition
// constants from one set (uni_rows).  Four bases per 16-byte load; byte 0 of
// each packed base is its base quality, which may differ.
__global__ void k_gap_check(const uchar4* __restrict__ quals, long long n, BandCounters* c) {
  const uint32_t ref = *reinterpret_cast<const uint32_t*>(quals) & 0x7f7f7f00u;
  const long long n4 = n / 4;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x, nt = (long long)gridDim.x * blockDim.x;
  bool mixed = false;
  for (long long x = tid; x < n4; x += nt) {
    const uint4 v = reinterpret_cast<const uint4*>(quals)[x];  // quals is 16-byte aligned (start of its allocation)
    mixed |= ((v.x & 0x7f7f7f00u) != ref) | ((v.y & 0x7f7f7f00u) != ref) | ((v.z & 0x7f7f7f00u) != ref) |
             ((v.w & 0x7f7f7f00u) != ref);
  }
  for (long long x = 4 * n4 + tid; x < n; x += nt)
    mixed |= (*reinterpret_cast<const uint32_t*>(quals + x) & 0x7f7f7f00u) != ref;
  if (__any_sync(0xffffffffu, mixed) && (threadIdx.x & 31) == 0) c->gap_mixed = 1u;
  if (tid == 0) c->gap_checked = 1u;
}

// Rescore: a read's pairs are consecutive result slots.  The thread at a
// read's first slot takes the best result over the read's pairs (NaN: an FP64
// rescue still to come, left out) and sends every banded pair more than
// cap_margin log10 units below it to the full DP: such a pair is a read
// scored against a haplotype it does not come from, and a stretch of the read
// that does not belong to the haplotype is then partly explained by paths off
// the band (a long insertion run, or a start far off the diagonal), which the
// ring test does not see.  The full DP's result replaces the banded one.
__global__ void k_band_cap(BandParams p) {
  for (long long pi = blockIdx.x * (long long)blockDim.x + threadIdx.x; pi < p.n_pairs;
       pi += (long long)gridDim.x * blockDim.x) {
    const int r = p.pair_read[pi];
    if (pi > 0 && p.pair_read[pi - 1] == r) continue;
    long long end = pi;
    double best = -INFINITY;
    for (; end < p.n_pairs && p.pair_read[end] == r; ++end) {
      const double v = p.out[end];
      if (v > best) best = v;  // NaN compares false
    }
    const double cut = best - (double)p.cap_margin;
    const int R = (int)(p.batch.read_off[r + 1] - p.batch.read_off[r]);
    const int v = full_variant(R);
    for (long long j = pi; j < end; ++j) {
      if (!p.banded[j] || !(p.out[j] < cut)) continue;
      const unsigned long long q = atomicAdd(&p.bctr->cap_count[v], 1ull);
      atomicAdd(&p.bctr->cap_flagged, 1ull);
      if (q < (unsigned long long)p.item_cap) {
        Unit u{};
        u.read = r; u.hap0 = p.pair_hap[j]; u.nh = 1; u.out0 = j;
        p.cap_items[(size_t)v * p.item_cap + q] = u;
      } else {
        atomicOr(&p.ctr->status, 4ull);
      }
    }
  }
}

__global__ void k_audit_units(BandParams p, Unit* units) {
  const unsigned long long n = min(p.bctr->audit_count, (unsigned long long)p.audit_cap);
  for (unsigned long long a = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; a < n;
       a += (unsigned long long)gridDim.x * blockDim.x) {
    const long long pi = p.audit_pairs[a];
    Unit u{};
    u.read = p.pair_read[pi]; u.hap0 = p.pair_hap[pi]; u.nh = 1; u.out0 = (long long)a;
    const int R = (int)(p.batch.read_off[u.read + 1] - p.batch.read_off[u.read]);
    const int v = full_variant(R);
    const unsigned long long q = atomicAdd(&p.bctr->audit_var[v], 1ull);
    units[(size_t)v * p.audit_cap + q] = u;  // q < n <= audit_cap
  }
}

__global__ void k_audit_compare(BandParams p, double* err) {
  const unsigned long long n = min(p.bctr->audit_count, (unsigned long long)p.audit_cap);
  for (unsigned long long a = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; a < n;
       a += (unsigned long long)gridDim.x * blockDim.x) {
    const double b = p.out[p.audit_pairs[a]], f = p.audit_out[a];
    // NaN where the full DP's FP32 value needed the FP64 pass (not audited)
    err[a] = (isfinite(b) && isfinite(f)) ? fabs(b - f) : (isinf(b) && isinf(f) ? 0.0 : __longlong_as_double(0x7ff8000000000000ll));
  }
}

}  // namespace

cudaError_t launch_gap_check(const uchar4* quals, long long n_bases, BandCounters* c, int sms, cudaStream_t st) {
  if (n_bases <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((n_bases / 4 + 255) / 256 + 1, (long long)sms * 8);
  k_gap_check<<<(int)blocks, 256, 0, st>>>(quals, n_bases, c);
  return cudaGetLastError();
}

cudaError_t launch_band_cap(const BandParams& p, int sms, cudaStream_t st) {
  if (p.n_pairs <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((p.n_pairs + 255) / 256, (long long)sms * 8);
  k_band_cap<<<(int)blocks, 256, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_audit_units(const BandParams& p, Unit* units, cudaStream_t st) {
  k_audit_units<<<64, 256, 0, st>>>(p, units);
  return cudaGetLastError();
}

cudaError_t launch_audit_compare(const BandParams& p, double* err, cudaStream_t st) {
  k_audit_compare<<<64, 256, 0, st>>>(p, err);
  return cudaGetLastError();
}

cudaError_t launch_pairs_from_units(const Unit* units, long long n_units, int32_t* pair_read, int32_t* pair_hap,
                                    int sms, cudaStream_t st) {
  if (n_units <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((n_units + 255) / 256, (long long)sms * 8);
  k_pairs_from_units<<<(int)blocks, 256, 0, st>>>(units, n_units, pair_read, pair_hap);
  return cudaGetLastError();
}

cudaError_t launch_read_kmers(const uint8_t* read_bases, long long n_bytes, uint32_t* codes, int sms, cudaStream_t st) {
  if (n_bytes <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>(((n_bytes + 3) / 4 + 255) / 256, (long long)sms * 16);
  k_read_kmers<<<(int)blocks, 256, 0, st>>>(read_bases, n_bytes, codes);
  return cudaGetLastError();
}

cudaError_t launch_hap_table(const uint8_t* hap_bases, const int64_t* hap_off, long long n_haps, long long n_hap_bytes,
                             uint32_t* table, uint32_t* nib, int sms, cudaStream_t st) {
  if (n_haps <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((n_haps + kHapTblWarps - 1) / kHapTblWarps, (long long)sms * 6);
  k_hap_table<<<(int)blocks, kHapTblWarps * 32, 0, st>>>(hap_bases, hap_off, n_haps, table);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long long nw = hap_nibble_words(n_hap_bytes);
  const long long nblk = std::min<long long>((nw + 255) / 256, (long long)sms * 8);
  k_hap_nibbles<<<(int)nblk, 256, 0, st>>>(hap_bases, n_hap_bytes, nib);
  return cudaGetLastError();
}

cudaError_t prepare_band_kernels() { return prepare_mlp_tc(); }

cudaError_t launch_featurize(const BandParams& p, int sms, cudaStream_t st) {
  if (p.n_units <= 0) return cudaSuccess;
  const long long need = (p.n_units + kFeatUWarps - 1) / kFeatUWarps;
  const long long blocks = std::min<long long>(need, (long long)sms * kFeatUBlocksPerSm);
  k_featurize_u<<<(int)blocks, kFeatUWarps * 32, 0, st>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // the slow list's length is known only on the device: the warp featuriser
  // reads it and returns at once when it is empty
  k_featurize_slow<<<feat_blocks(sms), kFeatWarps * 32, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const BandParams& p, int sms, cudaStream_t st) {
  return launch_mlp_forward_tc(p, sms, st);
}

cudaError_t launch_band_route(const BandParams& p, int pass, int sms, cudaStream_t st) {
  if (p.n_pairs <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((p.n_pairs + 255) / 256, (long long)sms * 8);
  k_band_route<<<(int)blocks, 256, 0, st>>>(p, pass);
  return cudaGetLastError();
}

cudaError_t launch_band_scan(BandCounters* c, cudaStream_t st) {
  k_band_scan<<<1, 32, 0, st>>>(c);
  return cudaGetLastError();
}

cudaError_t launch_band_dp(const BandParams& p, int cls, int sms, cudaStream_t st) {
  const int blocks = band_dp_blocks(sms, cls);
  if (cls == 0) {
    k_band_ring_f32<8><<<blocks, 128, 0, st>>>(p, 0);
  } else if (cls == 1) {
    k_band_ring_f32<16><<<blocks, 128, 0, st>>>(p, 1);
  } else if (cls == 2) {
    k_band_ring_f32<24><<<blocks, 128, 0, st>>>(p, 2);
  } else {
    k_band_ring_f32<32><<<blocks, 128, 0, st>>>(p, 3);
  }
  return cudaGetLastError();
}

}  // namespace bvphmm
