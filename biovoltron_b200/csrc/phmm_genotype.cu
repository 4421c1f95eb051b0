// phmm_genotype.cu -- normalise, filter, marginalise and score diploid
// genotypes on the staged batch's [read][hap] log10 matrix, one warp per
// region.  The steps and their arithmetic are the reference's:
//   PairHMM::normalize_likelihoods / filter_poorly_modeled_reads
//     (include/biovoltron/algo/align/inexact_match/pairhmm.hpp:83-114),
//   Genotyper::marginal_likelihoods and the diploid genotype likelihoods
//     (include/biovoltron/applications/haplotypecaller/genotype/genotyper.hpp:
//     223-240, 254-326), with MathUtils::approximate_log10_sum_log10
//     (include/biovoltron/math/math_utils.hpp:112-118).
// Genotype sums run read by read in order (one lane per genotype), as
// std::accumulate does, so the results equal the reference's bit for bit.
#include <cfloat>
#include <cmath>

#include "phmm_genotype.h"

namespace bvphmm {
namespace {

constexpr double kTableStep = 0.0001;
constexpr double kMaxTolerance = 8.0;
constexpr double kBestAltDifference = -4.5;   // pairhmm.hpp:28
constexpr double kErrorRatePerBase = 0.02;    // pairhmm.hpp:29
constexpr double kLog10QualityPerBase = -4.0; // pairhmm.hpp:30
constexpr double kMaxErrorsPerRead = 2.0;     // pairhmm.hpp:31

__device__ __forceinline__ double approx_log10_sum_log10(double a, double b, const double* table) {
  if (a > b) {
    const double t = a;
    a = b;
    b = t;
  }
  const double diff = b - a;
  if (diff < kMaxTolerance) return b + table[(long long)round(diff * (1.0 / kTableStep))];
  return b;
}

__global__ void __launch_bounds__(128) k_genotype(GenotypeParams p) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long g = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); g < p.n_regions; g += warps) {
    const int64_t r0 = p.region_reads[g], nr = p.region_reads[g + 1] - r0;
    const int64_t h0 = p.region_haps[g], nh = p.region_haps[g + 1] - h0;
    const int A = p.allele_count[g];
    const double* ll = p.ll + p.res_off[g];
    double* al = p.allele_lik + p.al_off[g];
    int32_t* kr = p.kept_reads + r0;
    // reads in chunks of 32: keep test per lane, ballot compaction keeps the order
    int kept = 0;
    for (int64_t c = 0; c < nr; c += 32) {
      const int64_t r = c + lane;
      bool keep = false;
      double best = -INFINITY;
      if (r < nr && nh > 0) {
        best = ll[r * nh];
        for (int64_t h = 1; h < nh; ++h) best = fmax(best, ll[r * nh + h]);
        const double len = (double)(p.read_off[r0 + r + 1] - p.read_off[r0 + r]);
        const double thr = fmin(kMaxErrorsPerRead, ceil(len * kErrorRatePerBase)) * kLog10QualityPerBase;
        keep = best < thr && p.overlap[r0 + r] != 0;
      }
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int k = kept + __popc(m & ((1u << lane) - 1u));
        kr[k] = (int32_t)(r0 + r);
        const double cap = best + kBestAltDifference;
        for (int a = 0; a < A; ++a) al[(int64_t)k * A + a] = -DBL_MAX;
        for (int64_t h = 0; h < nh; ++h) {
          double v = ll[r * nh + h];
          if (v < cap) v = cap;
          const int a = p.hap_allele[h0 + h];
          if (a >= 0 && a < A && v > al[(int64_t)k * A + a]) al[(int64_t)k * A + a] = v;
        }
      }
      kept += __popc(m);
    }
    __syncwarp();
    const int G = A * (A + 1) / 2;
    for (int gi = lane; gi < G; gi += 32) {
      // genotype gi = (a1, a2), a1 <= a2, in the reference's order
      int a1 = 0, rem = gi;
      while (rem >= A - a1) {
        rem -= A - a1;
        ++a1;
      }
      const int a2 = a1 + rem;
      double s = 0.0;
      for (int k = 0; k < kept; ++k) {
        const double x1 = al[(int64_t)k * A + a1];
        s += a1 == a2 ? x1 + p.log10_2 : approx_log10_sum_log10(x1, al[(int64_t)k * A + a2], p.table);
      }
      p.genotype_lik[p.geno_off[g] + gi] = s - (double)kept * p.log10_2;
    }
    if (lane == 0) p.kept_count[g] = kept;
    __syncwarp();
  }
}

}  // namespace

cudaError_t launch_genotype(const GenotypeParams& p, int sms, cudaStream_t st) {
  if (p.n_regions <= 0) return cudaSuccess;
  const long long want = (p.n_regions + 3) / 4;
  const int blocks = (int)(want < (long long)sms * 16 ? want : (long long)sms * 16);
  k_genotype<<<blocks, 128, 0, st>>>(p);
  return cudaGetLastError();
}

}  // namespace bvphmm
