// phmm_band.h -- learned-band path: launch interface (host <-> kernels).
//
// Pipeline, all on the context's stream:
//   k_pairs_from_units  expand work units into one (read, hap) per result slot
//   k_hap_table         per haplotype: 11-mer hash table (code -> positions)
//   k_read_kmers        per read position: 11-mer code
//   k_featurize_t       one thread per pair: shared 11-mer diagonal votes ->
//                       features, seed diagonal d* (the votes' mode), band
//                       extent (voted diagonals and read-end triangles); a
//                       pair voting for more diagonals than a thread keeps
//                       goes to k_featurize_slow (one warp per pair, a
//                       histogram in global scratch), with the same results
//   k_mlp_forward       per pair: BF16 MLP 80-128-128-2 (FP32 accumulation) ->
//                       lower and upper band edge relative to d*
//   k_band_route        band (by width class and read-length bucket) or full DP
//   k_band_ring_f32<W>  banded forward pass, one thread per pair, on the band
//                       and on the band widened by a ring of 4 (W = 8) or 8
//                       diagonals per side; the wider band is the result and a
//                       ring share above the threshold promotes the pair to the
//                       next class; classes W = 8, 16, 24, 32 run in that order
// Pairs that leave the band path (routed out, or failing at W = 32) go to the
// full-DP kernels through per-variant device lists; FP32 results below 1e-28
// go to the FP64 list as before.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "phmm_common.h"

namespace bvphmm {

constexpr int kK = 11;                 // k-mer length of the featuriser
constexpr int kSeedStride = 5;         // read 11-mers sampled every kSeedStride positions (and the last one)
constexpr int kFeat = 80;              // MLP input width (64 histogram bins + 16 scalars, zero padded)
constexpr int kHid = 128;              // hidden width
constexpr int kOut = 2;                // outputs: lower and upper band edge (diagonals, relative to d*)
constexpr int kHistBins = 64;          // histogram window: d* - 32 .. d* + 31
constexpr int kBandMaxSpan = 2048;     // read_len + hap_len limit of the featuriser (per-warp histogram)
constexpr int kBandMaxHap = 1024;      // haplotype limit of the k-mer sort and the featuriser's staging
constexpr int kBandWidths = 4;         // width classes of the banded kernel
#if defined(__CUDACC__)
__host__ __device__
#endif
constexpr int band_width(int cls) { return 8 * (cls + 1); }  // 8, 16, 24, 32 diagonals
constexpr int kRBuckets = 64;          // read-length buckets (8 rows each) for warp-uniform band launches
constexpr int kRBucketRows = 8;
constexpr int kBandMaxRead = kRBuckets * kRBucketRows - 1;

// MLP parameters, device layout: weights as [out][in] (row = output unit).
struct MlpParams {
  __nv_bfloat16 w1[kHid * kFeat];
  __nv_bfloat16 w2[kHid * kHid];
  __nv_bfloat16 w3[kOut * kHid];
  float b1[kHid];
  float b2[kHid];
  float b3[kOut];
};

// One banded-DP work item.
struct BandItem {
  int32_t read;
  int32_t hap;
  int64_t out;
  int32_t d_lo;  // first diagonal of the band (c - r)
  int32_t pad_;
};

struct BandCounters {
  unsigned long long band_count[kBandWidths][kRBuckets];  // items per (width, bucket)
  unsigned long long band_fill[kBandWidths][kRBuckets];
  unsigned long long band_next[kBandWidths];              // work-queue heads of the band launches
  unsigned long long band_total[kBandWidths];             // routed items per width class
  unsigned long long promoted[kBandWidths];               // items promoted from the next narrower class
  unsigned long long full_count[16];                      // fallback items per full-DP variant
  unsigned long long audit_count;
  unsigned long long audit_var[16];                       // audit units per full-DP variant
  unsigned long long fallback_edge;                       // pairs sent back by the edge check
  unsigned long long fallback_route;                      // pairs routed to the full DP up front
  unsigned long long band_cells;                          // cells of both sweeps (result band and inner band)
  unsigned long long band_result_cells;                   // cells of the result band (band plus ring)
  unsigned long long feat_slow_count;                     // pairs left to the warp featuriser (many distinct diagonals)
  unsigned long long feat_slow_next;                      // its work-queue head
  unsigned int gap_checked;                               // k_gap_check ran on this batch
  unsigned int gap_mixed;                                 // some base's gap qualities differ from the first base's
  unsigned long long cap_count[16];                       // banded pairs rescored by the full DP, per variant
  unsigned long long cap_flagged;                         // their total
};
// work-queue slots of the rescore launches (the fallback launches use 0 .. 8, the audit 16 .. 24)
constexpr int kCapSlot0 = 32;

struct BandParams {
  DeviceBatch batch;
  const Tables* tables;
  long long n_pairs;
  const int32_t* pair_read;   // [n_pairs]
  const int32_t* pair_hap;    // [n_pairs]
  const uint32_t* hap_table;  // 11-mer hash tables, 16-byte aligned, hap_table_words() words
  const uint32_t* hap_nib;    // one-hot nibbles of the haplotype bases, hap_nibble_words() words
  const Unit* units;          // work units (featuriser order)
  long long n_units;
  const uint32_t* read_kmers; // 11-mer code per read position
  uint32_t* feat_hist;        // featuriser scratch: one histogram of kBandMaxRead + kBandMaxHap slots per warp
  int64_t* feat_slow;         // [n_pairs] pairs the unit featuriser hands to the slow featuriser
  int32_t* dstar;             // [n_pairs] seed diagonal (INT32_MIN: no seed)
  int32_t* kmin;              // [n_pairs] lowest / highest diagonal of a shared 11-mer
  int32_t* kmax;
  __nv_bfloat16* feat;        // [n_pairs, kFeat]
  float* mlp_out;             // [n_pairs, kOut]
  const MlpParams* mlp;
  int use_mlp;                // 0: fixed band half-width `fixed_half` around d*
  int fixed_half;
  int margin;                 // diagonals added on both sides of the predicted band
  float edge_threshold;       // promotion when the ring adds more than this share of the likelihood
  float cap_margin;           // > 0: banded pairs this many log10 units below their read's best are rescored
  uint8_t* banded;            // [n_pairs] 1 where the result came from the banded kernel
  Unit* cap_items;            // [9][item_cap] rescore units per full-DP variant
  int audit_period;           // every audit_period-th pair is also scored by the full DP (0: off)
  BandCounters* bctr;
  Counters* ctr;
  BandItem* items;            // [kBandWidths][capacity]
  long long item_cap;
  Unit* full_items;           // [16][capacity] fallback units (nh = 1), per full-DP variant
  long long full_cap;
  int64_t* audit_pairs;       // [audit capacity]
  long long audit_cap;
  double* out;                // log10 per result slot
  double* audit_out;          // full-DP log10 of the audit pairs
  PairRef* rescue;
  long long rescue_cap;
};

// Words of the per-haplotype 11-mer hash tables of a batch.
inline long long hap_table_words(long long n_hap_bytes, long long n_haps) { return 2 * n_hap_bytes + 8 * n_haps + 4; }
// Words of the haplotype bases' nibble image (8 bases a word, then kNibPad zero words).
constexpr int kNibPad = 4;
inline long long hap_nibble_words(long long n_hap_bytes) { return (n_hap_bytes + 7) / 8 + kNibPad; }

cudaError_t launch_pairs_from_units(const Unit* units, long long n_units, int32_t* pair_read, int32_t* pair_hap,
                                    int sms, cudaStream_t st);
cudaError_t launch_read_kmers(const uint8_t* read_bases, long long n_bytes, uint32_t* codes, int sms, cudaStream_t st);
// The 11-mer tables and the nibble image of the batch's haplotypes (n_hap_bytes bases).
cudaError_t launch_hap_table(const uint8_t* hap_bases, const int64_t* hap_off, long long n_haps, long long n_hap_bytes,
                             uint32_t* table, uint32_t* nib, int sms, cudaStream_t st);
cudaError_t launch_featurize(const BandParams& p, int sms, cudaStream_t st);
// Whether every read base has the first base's insertion, deletion and gap-continuation
// qualities (BandCounters::gap_checked / gap_mixed; the counters must be zero before).
cudaError_t launch_gap_check(const uchar4* quals, long long n_bases, BandCounters* c, int sms, cudaStream_t st);
cudaError_t launch_mlp_forward(const BandParams& p, int sms, cudaStream_t st);
cudaError_t launch_band_route(const BandParams& p, int pass, int sms, cudaStream_t st);
cudaError_t launch_band_scan(BandCounters* c, cudaStream_t st);
cudaError_t launch_band_dp(const BandParams& p, int width_class, int sms, cudaStream_t st);
// After the fallback full DP: per read, the banded pairs whose result lies more than cap_margin
// log10 units below the read's best result go to the rescore lists (cap_items, cap_count).
cudaError_t launch_band_cap(const BandParams& p, int sms, cudaStream_t st);
// banded kernels: 128-thread blocks, as many as fit at once (3 per SM for W = 8, 2 for the wider classes)
inline int band_dp_blocks(int sms, int width_class) { return sms * (width_class == 0 ? 3 : 2); }
// warp featuriser (the slow path) grid and its per-warp scratch histograms (words)
constexpr int kFeatWarpsPerBlock = 4;
inline int feat_blocks(int sms) { return sms * 4; }
inline long long feat_hist_words(int sms) { return (long long)feat_blocks(sms) * kFeatWarpsPerBlock * (kBandMaxRead + kBandMaxHap); }
// Sets the dynamic shared-memory limits of the band kernels (before any capture).
cudaError_t prepare_band_kernels();
// The MLP inference kernel on tcgen05 tensor cores (phmm_mlp_tc.cu).
cudaError_t prepare_mlp_tc();
cudaError_t launch_mlp_forward_tc(const BandParams& p, int sms, cudaStream_t st);
// audit: full-DP units for the sampled pairs (out = audit slot), listed per full-DP
// variant ([9][audit_cap]), then the differences
cudaError_t launch_audit_units(const BandParams& p, Unit* units, cudaStream_t st);
cudaError_t launch_audit_compare(const BandParams& p, double* err, cudaStream_t st);

}  // namespace bvphmm
