// phmm_genotype.h -- the genotyper steps that consume the PairHMM matrix, on
// the device, fused after a staged run (no D2H of the [read][hap] matrix).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace bvphmm {

constexpr int kJacobianEntries = 80001;  // MathUtils::JacobianLogTable: 8.0 / 1e-4 + 1 (math_utils.hpp:122-139)

struct GenotypeParams {
  const double* ll;            // the staged batch's log10 results, region-major [read][hap]
  const int64_t* read_off;     // read byte offsets (read lengths)
  const int64_t* region_reads; // [regions + 1]
  const int64_t* region_haps;  // [regions + 1]
  const int64_t* res_off;      // [regions]: first result slot of each region
  const int64_t* al_off;       // [regions]: first allele-likelihood slot (sum of reads * alleles before)
  const int64_t* geno_off;     // [regions]: first genotype slot
  const int32_t* allele_count; // [regions]
  const int32_t* hap_allele;   // [haps]
  const uint8_t* overlap;      // [reads]
  const double* table;         // Jacobian log table
  double log10_2;
  long long n_regions;
  int32_t* kept_count;         // [regions]
  int32_t* kept_reads;         // [reads]: per region block, the kept reads (batch read indices) in order
  double* allele_lik;          // per region block: kept x alleles
  double* genotype_lik;        // per region block: alleles (alleles + 1) / 2
};

cudaError_t launch_genotype(const GenotypeParams& p, int sms, cudaStream_t st);

// Host: the Jacobian log table, entries log10(1 + 10^(-1e-4 i)) rounded to
// double from 113-bit arithmetic (the correctly rounded values).
void build_jacobian_table(double* out);

}  // namespace bvphmm
