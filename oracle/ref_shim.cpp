// ref_shim.cpp -- C entry points around Biovoltron's own PairHMM kernel.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's headers where they lie (lib/intel_native/pairhmm/*.h) into
// oracle/_ref/libref_pairhmm.so.  Nothing of the reference is copied here: the
// kernel bodies come from the included headers, which define non-inline
// functions and therefore live in exactly this one translation unit.
//
// The entry points reproduce what AvxPairHMM does around the kernel
// (include/biovoltron/algo/align/inexact_match/pairhmm_avx.hpp):
//   initNative          :83-119  FTZ on, ConvertChar::init, Context ctors
//   computeLikelihoods  :121-157 OpenMP dynamic loop, FP32 then FP64 below
//                                MIN_ACCEPTED, log10 minus the scale constant
// but take testcases directly, so reads longer than the 256-byte SAM penalty
// strings get well-defined penalty arrays.
#include <cmath>
#include <cstdint>
#include <algorithm>
#include <omp.h>

#include "intel_native/pairhmm/avx-pairhmm.h"

namespace {
struct RefInit {
  Context<float> ctxf;
  Context<double> ctxd;
  RefInit() { ConvertChar::init(); }
};
RefInit &ref_init() {
  static RefInit r;
  return r;
}
void set_ftz() { _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON); }
}  // namespace

extern "C" {

float ref_prob_f32(testcase *tc) {
  ref_init();
  set_ftz();
  return compute_full_prob_avxs<float>(tc);
}

double ref_prob_f64(testcase *tc) {
  ref_init();
  set_ftz();
  return compute_full_prob_avxd<double>(tc);
}

// computeLikelihoodsNative's loop body and OpenMP schedule, over a flat list.
void ref_batch_log10(long n, testcase *tcs, double *out, int *used_f64, int nthreads) {
  RefInit &ri = ref_init();
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (long k = 0; k < n; k++) {
    set_ftz();
    const float rf = compute_full_prob_avxs<float>(&tcs[k]);
    double res;
    int dbl = 0;
    if (rf < MIN_ACCEPTED) {
      const double rd = compute_full_prob_avxd<double>(&tcs[k]);
      res = std::log10(rd) - ri.ctxd.LOG10_INITIAL_CONSTANT;
      dbl = 1;
    } else {
      res = ::log10f(rf) - ri.ctxf.LOG10_INITIAL_CONSTANT;
    }
    out[k] = res;
    if (used_f64) used_f64[k] = dbl;
  }
}

// The static tables the kernel reads (Context.h:17-23), for table-identity tests.
const float *ref_table_ph2pr_f32() { ref_init(); return Context<float>::ph2pr; }
const double *ref_table_ph2pr_f64() { ref_init(); return Context<double>::ph2pr; }
const float *ref_table_mm_f32() { ref_init(); return Context<float>::matchToMatchProb; }
const double *ref_table_mm_f64() { ref_init(); return Context<double>::matchToMatchProb; }
int ref_table_mm_size() { return ((MAX_QUAL + 1) * (MAX_QUAL + 2)) >> 1; }
int ref_threads() { return omp_get_max_threads(); }

}  // extern "C"
