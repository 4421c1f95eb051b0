// ref_scalar_shim.cpp -- C entry point around Biovoltron's scalar PairHMM.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file against the
// reference's headers where they lie (include/biovoltron/...) into
// oracle/_ref/libref_scalar.so; nothing of the reference is copied here.
//
// PairHMM::compute_likelihoods (include/biovoltron/algo/align/inexact_match/
// pairhmm.hpp:116-141) normalises and filters its matrix, and the filter
// drops well-modelled reads, so the shim calls the per-pair step
// sub_compute_likelihood (:56-80) directly; the access specifier is lifted
// for this one translation unit to reach it.
// The standard headers the reference's headers use come first, so the
// lifted access specifier only reaches the reference's own types.
#include <algorithm>
#include <array>
#include <cassert>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cwctype>
#include <ios>
#include <iostream>
#include <istream>
#include <limits>
#include <map>
#include <ostream>
#include <ranges>
#include <span>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <tuple>
#include <vector>
#define private public
#include <biovoltron/algo/align/inexact_match/pairhmm.hpp>
#undef private

extern "C" double ref_scalar_log10(const char* read, const char* qual, int rl, const char* hap, int hl,
                                   const double* trans /* 7 entries, NULL = ORIGINAL_DEFAULT */) {
  using namespace biovoltron;
  SamRecord<> r;
  r.seq.assign(read, read + rl);
  r.qual.assign(qual, qual + rl);
  const std::string h(hap, hap + hl);
  PairHMM::TrasMatrx t = PairHMM::ORIGINAL_DEFAULT;
  if (trans)
    for (int k = 0; k < PairHMM::TRANS_PROB_ARRAY_LENGTH; ++k) t[k] = trans[k];
  auto M = std::vector(rl + 1, std::vector(hl + 1, 0.0));
  auto I = M, D = M, prior = M;
  return PairHMM{}.sub_compute_likelihood(r, h, t, M, I, D, prior);
}
