// ref_genotyper_shim.cpp -- C entry points around Biovoltron's genotyper
// marginalisation and diploid genotype likelihoods.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file against the
// reference's headers where they lie into oracle/_ref/libref_genotyper.so;
// nothing of the reference is copied here.
//
// ref_genotype runs, on one window's raw [read][hap] log10 matrix, what
// HaplotypeCaller does with it: PairHMM::normalize_likelihoods and
// filter_poorly_modeled_reads (include/biovoltron/algo/align/inexact_match/
// pairhmm.hpp:83-114), the genotyper's read selection by overlap (here a mask
// over the window's original reads), Genotyper::marginal_likelihoods and
// calculate_genotype_likelihoods (include/biovoltron/applications/
// haplotypecaller/genotype/genotyper.hpp:223-240, 254-326).  Those two are
// private members of a class; an explicit template instantiation, which
// ignores access, names them.  MathUtils keeps its Jacobian log table in a
// private: section, which the lifted specifier below opens.
#include <algorithm>
#include <array>
#include <bitset>
#include <cassert>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cwctype>
#include <deque>
#include <functional>
#include <ios>
#include <iostream>
#include <istream>
#include <iterator>
#include <limits>
#include <list>
#include <map>
#include <memory>
#include <numbers>
#include <numeric>
#include <optional>
#include <ostream>
#include <queue>
#include <ranges>
#include <set>
#include <span>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <variant>
#include <vector>
#define private public
#include <biovoltron/algo/align/inexact_match/pairhmm.hpp>
#include <biovoltron/applications/haplotypecaller/genotype/genotyper.hpp>
#undef private

namespace {
using Mat = std::vector<std::vector<double>>;
using U32 = std::vector<std::uint32_t>;
struct MargTag {
  using type = Mat (biovoltron::Genotyper::*)(std::uint32_t, const U32&, const U32&, const Mat&) const;
  friend type get(MargTag);
};
struct GenoTag {
  using type = std::vector<double> (biovoltron::Genotyper::*)(const Mat&, std::uint32_t) const;
  friend type get(GenoTag);
};
template <typename Tag, typename Tag::type M>
struct Robber {
  friend typename Tag::type get(Tag) { return M; }
};
template struct Robber<MargTag, &biovoltron::Genotyper::marginal_likelihoods>;
template struct Robber<GenoTag, &biovoltron::Genotyper::calculate_genotype_likelihoods>;
}  // namespace

extern "C" {

int ref_jacobian_table(double* out, int n) {
  const auto& t = biovoltron::MathUtils::JacobianLogTable::cache;
  for (int k = 0; k < n && k < (int)t.size(); ++k) out[k] = t[k];
  return (int)t.size();
}

double ref_approximate_log10_sum_log10(double a, double b) {
  return biovoltron::MathUtils::approximate_log10_sum_log10(a, b);
}

// ll: [nreads][nhaps] raw log10; read_len: [nreads]; overlap: [nreads] 0/1;
// hap_allele: [nhaps].  Writes the kept reads' original indices, their allele
// likelihoods [nkept][allele_count] and the genotype likelihoods
// [allele_count (allele_count + 1) / 2]; returns nkept.
int ref_genotype(int nreads, int nhaps, const double* ll, const int* read_len, const unsigned char* overlap,
                 int allele_count, const unsigned* hap_allele, int* kept, double* allele_out, double* geno_out) {
  using namespace biovoltron;
  std::vector<SamRecord<>> reads(nreads);
  Mat m(nreads, std::vector<double>(nhaps));
  for (int r = 0; r < nreads; ++r) {
    reads[r].seq.assign(read_len[r], 'A');
    reads[r].qname = std::to_string(r);
    for (int h = 0; h < nhaps; ++h) m[r][h] = ll[(size_t)r * nhaps + h];
  }
  PairHMM::normalize_likelihoods(m);
  PairHMM::filter_poorly_modeled_reads(reads, m);
  U32 keep;
  for (int i = 0; i < (int)reads.size(); ++i)
    if (overlap[std::stoi(reads[i].qname)]) keep.push_back(i);
  U32 mapper(hap_allele, hap_allele + nhaps);
  Genotyper g;
  const Mat al = (g.*get(MargTag{}))(allele_count, mapper, keep, m);
  const std::vector<double> gl = (g.*get(GenoTag{}))(al, allele_count);
  for (size_t k = 0; k < keep.size(); ++k) {
    kept[k] = std::stoi(reads[keep[k]].qname);
    for (int a = 0; a < allele_count; ++a) allele_out[k * allele_count + a] = al[k][a];
  }
  for (size_t gi = 0; gi < gl.size(); ++gi) geno_out[gi] = gl[gi];
  return (int)keep.size();
}

}  // extern "C"
