// phmm_common.h -- types shared by the PairHMM kernels and the host engine.
#pragma once
#include <cstdint>
#include <vector_types.h>

namespace bvphmm {

// Quality bytes are masked to 0..127 (avx-pairhmm-template.h:110-126), so the
// match-to-match table is only ever indexed up to max*(max+1)/2+min with
// max, min <= 127 (Context.h:121-133): 127*128/2 + 127 + 1 entries.
constexpr int kQualMask = 127;
constexpr int kMMEntries = 127 * 128 / 2 + 127 + 1;

// Haplotype column codes.  0..4 follow ConvertChar (pairhmm_common.h:26-44:
// A0 C1 T2 G3 N4, every other byte 0); 5 marks a column outside the
// haplotype, whose emission is 0 so the wavefront's ramp-up and ramp-down
// columns carry exact boundary values.
constexpr int kCodes = 6;
constexpr int kPadCode = 5;

constexpr int kWarp = 32;
// Leading and trailing padding of the staged haplotype code row (bytes).
constexpr int kHapLead = 32;
constexpr int kHapTail = 48;

// Reference constants (Context.h:104-110, 144-150; pairhmm_common.h:16).
constexpr double kMinAccepted = 1e-28;

// The FP32 kernels fold pMM(r) into row r's emissions (five operations per
// cell instead of six) when every row involved has pMM >= kFoldMin; pMM is
// that small only for indel qualities of a few units.
constexpr float kFoldMin = 0.5f;

// Per-quality FP32 probabilities for the banded kernel: p = 10^(-q/10),
// 1 - p, p / 3 and 1 / p, one 16-byte load per quality byte.
struct alignas(16) QProb {
  float p, q, third, inv;
};

struct Tables {
  QProb qp[128];
  float ph2pr_f[128];
  float mm_f[kMMEntries];
  float mm_inv_f[kMMEntries];  // 1 / mm_f where mm_f >= kFoldMin, else NaN
  double ph2pr_d[128];
  double mm_d[kMMEntries];
  // Constant transitions (the scalar PairHMM model, pairhmm.hpp:32-33, 56-80):
  // const_mode = 1 takes every row's transitions from cf / cd instead of the
  // quality bytes: [0] M->M, [1] M->I, [2] M->D, [3] I->M, [4] I->I, [5] D->M,
  // [6] D->D (PairHMM::TrasMatrx order); cf[7] = 1 / cf[0] when the folded form
  // applies, else NaN.  Only the base qualities are read then.
  int32_t const_mode;
  float cf[8];
  double cd[8];
  float init_f;          // 2^120
  float log10_init_f;    // log10f(2^120), evaluated on the host as the reference does
  double init_d;         // 2^1020
  double log10_init_d;
};

// One unit of full-DP work: a read scored against `nh` consecutive haplotypes
// whose results are consecutive in the output.
struct Unit {
  int32_t read;
  int32_t hap0;
  int32_t nh;
  int32_t pad_;
  int64_t out0;
};

// A pair routed to the FP64 kernel.
struct PairRef {
  int32_t read;
  int32_t hap;
  int64_t out;
};

struct DeviceBatch {
  const uint8_t* read_bases;
  const uchar4* read_quals;  // (q, i, d, c) per read position
  const int64_t* read_off;
  const uint8_t* hap_bases;
  const int64_t* hap_off;
};

// Device-side counters and status, one block of memory per call.
struct Counters {
  unsigned long long unit_next[48];  // work-queue heads, one per launch slot
  unsigned long long rescue_count;
  unsigned long long rescue_next;
  unsigned long long underflow_count;  // FP64 results that stayed non-positive
  unsigned long long status;           // nonzero: a kernel met an inconsistent input
  unsigned long long rescued_cells;    // DP cells the FP64 pass computed
  unsigned long long rescue_long_count;  // FP64 list entries of long reads (at the list's far end)
  unsigned long long rescue_long_next;
  unsigned long long fp32_skipped_cells;  // cells of strips the FP32 pass skipped by handing a pair over early
};

}  // namespace bvphmm
