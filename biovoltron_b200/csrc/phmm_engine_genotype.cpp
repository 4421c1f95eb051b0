// phmm_engine_genotype.cpp -- host side of the device genotyper: region
// offsets, the Jacobian log table, uploads, one launch, result copies.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "phmm_engine.h"
#include "phmm_genotype.h"

namespace bvphmm {

#define BV_CUDA(call, what)                              \
  do {                                                   \
    cudaError_t e__ = (call);                            \
    if (e__ != cudaSuccess) return cuda_fail(e__, what); \
  } while (0)

bv_status Engine::genotype_staged(const bv_region_batch& b, const bv_genotype_batch& g, int32_t* kept_count,
                                  int32_t* kept_reads, double* allele_lik, double* genotype_lik, double* kernel_ms) {
  if (!staged_ || runs_since_stage_ == 0) return fail(BV_ERR_INVALID_ARG, "no staged batch has been run");
  if (!g.allele_count || (b.num_haps > 0 && !g.hap_allele) || (b.num_reads > 0 && !g.read_overlaps))
    return fail(BV_ERR_INVALID_ARG, "genotype inputs missing");
  bv_status s = validate(b);
  if (s != BV_OK) return s;
  if (b.num_reads != n_reads_ || b.num_haps != n_haps_) return fail(BV_ERR_INVALID_ARG, "not the staged batch");
  const int64_t G = b.num_regions;
  // offsets: results, allele likelihoods, genotypes
  std::vector<int64_t> off(3 * (size_t)std::max<int64_t>(G, 1), 0);
  int64_t res = 0, al = 0, ge = 0;
  for (int64_t r = 0; r < G; ++r) {
    const int64_t nr = b.region_reads[r + 1] - b.region_reads[r], nh = b.region_haps[r + 1] - b.region_haps[r];
    const int32_t A = g.allele_count[r];
    if (A < 1 || A > 64) return fail(BV_ERR_INVALID_ARG, "allele count outside 1..64");
    off[r] = res;
    off[G + r] = al;
    off[2 * G + r] = ge;
    res += nr * nh;
    al += nr * A;
    ge += (int64_t)A * (A + 1) / 2;
  }
  if (res != n_results_) return fail(BV_ERR_INVALID_ARG, "not the staged batch");
  if (G > 0 && (!kept_count || (b.num_reads > 0 && !kept_reads) || (al > 0 && !allele_lik) || !genotype_lik))
    return fail(BV_ERR_INVALID_ARG, "null output");
  BV_CUDA(cudaSetDevice(opt_.device), "cudaSetDevice");
  if (!jacobian_ready_) {
    std::vector<double> t(kJacobianEntries);
    build_jacobian_table(t.data());
    BV_CUDA(d_jacobian_.reserve(sizeof(double) * kJacobianEntries), "alloc table");
    BV_CUDA(cudaMemcpy(d_jacobian_.get(), t.data(), sizeof(double) * kJacobianEntries, cudaMemcpyHostToDevice),
            "table copy");
    jacobian_ready_ = true;
  }
  const size_t nG = (size_t)std::max<int64_t>(G, 1), nR = (size_t)std::max<int64_t>(b.num_reads, 1);
  const size_t nH = (size_t)std::max<int64_t>(b.num_haps, 1);
  BV_CUDA(d_gt_regions_.reserve(sizeof(int64_t) * 2 * (nG + 1)), "alloc");
  BV_CUDA(d_gt_offsets_.reserve(sizeof(int64_t) * 3 * nG), "alloc");
  BV_CUDA(d_gt_alleles_.reserve(sizeof(int32_t) * nG), "alloc");
  BV_CUDA(d_gt_hap_allele_.reserve(sizeof(int32_t) * nH), "alloc");
  BV_CUDA(d_gt_overlap_.reserve(nR), "alloc");
  BV_CUDA(d_gt_kept_count_.reserve(sizeof(int32_t) * nG), "alloc");
  BV_CUDA(d_gt_kept_reads_.reserve(sizeof(int32_t) * nR), "alloc");
  BV_CUDA(d_gt_allele_lik_.reserve(sizeof(double) * (size_t)std::max<int64_t>(al, 1)), "alloc");
  BV_CUDA(d_gt_geno_lik_.reserve(sizeof(double) * (size_t)std::max<int64_t>(ge, 1)), "alloc");
  if (G > 0) {
    int64_t* reg = d_gt_regions_.as<int64_t>();
    BV_CUDA(cudaMemcpyAsync(reg, b.region_reads, sizeof(int64_t) * (G + 1), cudaMemcpyHostToDevice, stream_), "H2D");
    BV_CUDA(cudaMemcpyAsync(reg + G + 1, b.region_haps, sizeof(int64_t) * (G + 1), cudaMemcpyHostToDevice, stream_),
            "H2D");
    BV_CUDA(cudaMemcpyAsync(d_gt_offsets_.get(), off.data(), sizeof(int64_t) * 3 * G, cudaMemcpyHostToDevice, stream_),
            "H2D");
    BV_CUDA(cudaMemcpyAsync(d_gt_alleles_.get(), g.allele_count, sizeof(int32_t) * G, cudaMemcpyHostToDevice, stream_),
            "H2D");
  }
  if (b.num_haps > 0)
    BV_CUDA(cudaMemcpyAsync(d_gt_hap_allele_.get(), g.hap_allele, sizeof(int32_t) * b.num_haps, cudaMemcpyHostToDevice,
                            stream_), "H2D");
  if (b.num_reads > 0)
    BV_CUDA(cudaMemcpyAsync(d_gt_overlap_.get(), g.read_overlaps, b.num_reads, cudaMemcpyHostToDevice, stream_), "H2D");
  GenotypeParams p{};
  p.ll = d_out_.as<double>();
  p.read_off = d_read_off_.as<int64_t>();
  p.region_reads = d_gt_regions_.as<int64_t>();
  p.region_haps = d_gt_regions_.as<int64_t>() + G + 1;
  p.res_off = d_gt_offsets_.as<int64_t>();
  p.al_off = d_gt_offsets_.as<int64_t>() + G;
  p.geno_off = d_gt_offsets_.as<int64_t>() + 2 * G;
  p.allele_count = d_gt_alleles_.as<int32_t>();
  p.hap_allele = d_gt_hap_allele_.as<int32_t>();
  p.overlap = d_gt_overlap_.as<uint8_t>();
  p.table = d_jacobian_.as<double>();
  p.log10_2 = std::log10(2.0);  // the reference's log10_frequency and denominator factor
  p.n_regions = G;
  p.kept_count = d_gt_kept_count_.as<int32_t>();
  p.kept_reads = d_gt_kept_reads_.as<int32_t>();
  p.allele_lik = d_gt_allele_lik_.as<double>();
  p.genotype_lik = d_gt_geno_lik_.as<double>();
  BV_CUDA(cudaEventRecord(ev_[0], stream_), "event");
  BV_CUDA(launch_genotype(p, sms_, stream_), "genotype");
  BV_CUDA(cudaEventRecord(ev_[1], stream_), "event");
  if (G > 0) {
    BV_CUDA(cudaMemcpyAsync(kept_count, p.kept_count, sizeof(int32_t) * G, cudaMemcpyDeviceToHost, stream_), "D2H");
    if (b.num_reads > 0)
      BV_CUDA(cudaMemcpyAsync(kept_reads, p.kept_reads, sizeof(int32_t) * b.num_reads, cudaMemcpyDeviceToHost, stream_),
              "D2H");
    if (al > 0)
      BV_CUDA(cudaMemcpyAsync(allele_lik, p.allele_lik, sizeof(double) * al, cudaMemcpyDeviceToHost, stream_), "D2H");
    BV_CUDA(cudaMemcpyAsync(genotype_lik, p.genotype_lik, sizeof(double) * ge, cudaMemcpyDeviceToHost, stream_), "D2H");
  }
  BV_CUDA(cudaStreamSynchronize(stream_), "genotype sync");
  if (kernel_ms) {
    float ms = 0;
    BV_CUDA(cudaEventElapsedTime(&ms, ev_[0], ev_[1]), "event time");
    *kernel_ms = ms;
  }
  return BV_OK;
}

}  // namespace bvphmm
