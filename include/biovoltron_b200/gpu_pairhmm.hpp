// gpu_pairhmm.hpp -- C++20 drop-in for biovoltron::AvxPairHMM / PairHMM.
//
// GpuPairHMM::compute_likelihoods(haplotypes, reads) has the signature, the
// [read][hap] result layout and the side effects of
// AvxPairHMM::compute_likelihoods (include/biovoltron/algo/align/
// inexact_match/pairhmm_avx.hpp:160-171), which HaplotypeCaller calls through
// PairHMM::compute_likelihoods (haplotypecaller.hpp:90):
//   1. the inputs are those AvxPairHMM::getData gathers (:38-81): read bases,
//      qual, insertion_gop(), deletion_gop(), overall_gcp() and each
//      haplotype's seq; the window goes to the device as one region (each
//      haplotype once, constant penalty views as three bytes);
//   2. log10 likelihoods come from the GPU (FP32, FP64 below 1e-28);
//   3. PairHMM::normalize_likelihoods (pairhmm.hpp:83-93) caps every value at
//      the row's best - 4.5;
//   4. PairHMM::filter_poorly_modeled_reads (pairhmm.hpp:95-114) keeps the
//      reads whose best likelihood is below min(2, ceil(0.02 len)) * -4 --
//      the reference's comparison, unchanged -- and removes the others from
//      `reads`.
// Read and haplotype types are template parameters, so Biovoltron's
// SamRecord<> / Haplotype work unchanged (they provide .seq, .qual and the
// three penalty views), as do any types with the same members.
//
// Errors from the C ABI are thrown as std::runtime_error.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "bv_pairhmm.h"

namespace biovoltron_b200 {

class GpuPairHMM {
 public:
  static constexpr double kMaximumBestAltLikelihoodDifference = -4.5;  // pairhmm.hpp:28
  static constexpr double kExpectedErrorRatePerBase = 0.02;             // pairhmm.hpp:29
  static constexpr double kLog10QualityPerBase = -4.0;                  // pairhmm.hpp:30
  static constexpr double kMaximumExpectedErrorPerRead = 2.0;           // pairhmm.hpp:31

  explicit GpuPairHMM(int device = 0, bool use_double = false) {
    bv_phmm_options o;
    bv_phmm_default_options(&o);
    o.device = device;
    o.precision = use_double ? BV_PRECISION_F64 : BV_PRECISION_AUTO;
    check(bv_phmm_create(&o, &ctx_), "bv_phmm_create");
  }
  ~GpuPairHMM() { bv_phmm_destroy(ctx_); }
  GpuPairHMM(const GpuPairHMM&) = delete;
  GpuPairHMM& operator=(const GpuPairHMM&) = delete;

  template <class HapVec, class ReadVec>
  std::vector<std::vector<double>> compute_likelihoods(const HapVec& haplotypes, ReadVec& reads) {
    const size_t nr = reads.size(), nh = haplotypes.size();
    std::vector<std::vector<double>> ll(nr, std::vector<double>(nh, 0.0));
    if (nr == 0 || nh == 0) return ll;
    score(haplotypes, reads, false, ll);
    normalize_likelihoods(ll);
    filter_poorly_modeled_reads(reads, ll);
    return ll;
  }

  static void normalize_likelihoods(std::vector<std::vector<double>>& log_likelihoods) {
    for (auto& row : log_likelihoods) {
      if (row.empty()) continue;
      const double cap = *std::max_element(row.begin(), row.end()) + kMaximumBestAltLikelihoodDifference;
      for (auto& v : row)
        if (v < cap) v = cap;
    }
  }

  template <class ReadVec>
  static void filter_poorly_modeled_reads(ReadVec& reads, std::vector<std::vector<double>>& log_likelihoods) {
    ReadVec kept_reads;
    std::vector<std::vector<double>> kept;
    for (size_t i = 0; i < log_likelihoods.size(); ++i) {
      const double best = *std::max_element(log_likelihoods[i].begin(), log_likelihoods[i].end());
      const double thr = std::min(kMaximumExpectedErrorPerRead,
                                  std::ceil(reads[i].seq.size() * kExpectedErrorRatePerBase)) *
                         kLog10QualityPerBase;
      if (best < thr) {
        kept_reads.push_back(std::move(reads[i]));
        kept.push_back(std::move(log_likelihoods[i]));
      }
    }
    reads.swap(kept_reads);
    log_likelihoods.swap(kept);
  }

  bv_phmm_ctx* context() const { return ctx_; }

 protected:
  // Scores every read against every haplotype into ll (no normalising or
  // filtering); `scalar` takes only the base qualities (constant
  // transitions).  The window is one region of bv_phmm_compute_regions, so
  // each haplotype crosses to the device once; when every read's three
  // penalty views hold one and the same byte (SamRecord fills them from
  // constant strings) they go as the batch's uniform gap penalties instead of
  // per-base arrays.
  template <class HapVec, class ReadVec>
  void score(const HapVec& haplotypes, const ReadVec& reads, bool scalar, std::vector<std::vector<double>>& ll) {
    const size_t nr = reads.size(), nh = haplotypes.size();
    std::vector<int64_t> region_reads{0, static_cast<int64_t>(nr)}, region_haps{0, static_cast<int64_t>(nh)};
    std::vector<int64_t> read_off{0}, hap_off{0};
    std::string rb, rq, ri, rd, rc, hb;
    int gap[3] = {-1, -1, -1};
    bool uniform = true;
    if (!scalar) {
      for (const auto& r : reads) {
        const size_t n = r.seq.size();
        const char* v[3] = {r.insertion_gop().data(), r.deletion_gop().data(), r.overall_gcp().data()};
        for (int k = 0; k < 3 && uniform; ++k)
          for (size_t x = 0; x < n && uniform; ++x) {
            const int b = static_cast<unsigned char>(v[k][x]);
            if (gap[k] < 0) gap[k] = b;
            uniform = b == gap[k];
          }
        if (!uniform) break;
      }
    }
    for (const auto& r : reads) {
      rb.append(r.seq.data(), r.seq.size());
      rq.append(r.qual.data(), r.qual.size());
      if (!scalar && !uniform) {
        ri.append(r.insertion_gop().data(), r.seq.size());
        rd.append(r.deletion_gop().data(), r.seq.size());
        rc.append(r.overall_gcp().data(), r.seq.size());
      }
      read_off.push_back(static_cast<int64_t>(rb.size()));
    }
    for (const auto& h : haplotypes) {
      hb.append(h.seq.data(), h.seq.size());
      hap_off.push_back(static_cast<int64_t>(hb.size()));
    }
    auto u8 = [](const std::string& x) { return reinterpret_cast<const uint8_t*>(x.data()); };
    bv_region_batch b{};
    b.num_regions = 1;
    b.region_reads = region_reads.data();
    b.region_haps = region_haps.data();
    b.num_reads = static_cast<int64_t>(nr);
    b.read_offsets = read_off.data();
    b.read_bases = u8(rb);
    b.read_q = u8(rq);
    if (scalar || uniform) {
      // the scalar model's transitions are constant; its gap bytes are unused
      b.gap_ins = static_cast<uint8_t>(gap[0] < 0 ? 0 : gap[0]);
      b.gap_del = static_cast<uint8_t>(gap[1] < 0 ? 0 : gap[1]);
      b.gap_gcp = static_cast<uint8_t>(gap[2] < 0 ? 0 : gap[2]);
    } else {
      b.read_i = u8(ri);
      b.read_d = u8(rd);
      b.read_c = u8(rc);
    }
    b.num_haps = static_cast<int64_t>(nh);
    b.hap_offsets = hap_off.data();
    b.hap_bases = u8(hb);
    std::vector<double> flat(nr * nh);
    check(bv_phmm_compute_regions(ctx_, &b, flat.data(), nullptr), "bv_phmm_compute_regions");
    for (size_t r = 0; r < nr; ++r)
      std::copy(flat.begin() + r * nh, flat.begin() + (r + 1) * nh, ll[r].begin());
  }

 private:
  void check(bv_status s, const char* what) {
    if (s != BV_OK) {
      std::string msg = std::string(what) + ": " + bv_phmm_status_string(s);
      if (ctx_) msg += std::string(" (") + bv_phmm_last_error(ctx_) + ")";
      throw std::runtime_error(msg);
    }
  }
  bv_phmm_ctx* ctx_ = nullptr;
};

// Drop-in for the scalar biovoltron::PairHMM (include/biovoltron/algo/align/
// inexact_match/pairhmm.hpp): compute_likelihoods(haplotypes, reads, trans)
// scores with seven constant transition probabilities (ORIGINAL_DEFAULT
// unless given, :32-33) and the base qualities' emission prior (:39-54), then
// normalises and filters as PairHMM does (:83-114).  Bases compare as
// A/C/G/T with N matching everything, which is the scalar model's raw-byte
// comparison for upper-case ACGTN sequences.
class GpuScalarPairHMM : public GpuPairHMM {
 public:
  using TransMatrix = std::array<double, 7>;  // M->M, M->I, M->D, I->M, I->I, D->M, D->D
  static constexpr TransMatrix kOriginalDefault = {0.9998, 0.0001, 0.0001, 0.9, 0.1, 0.9, 0.1};

  explicit GpuScalarPairHMM(int device = 0) : GpuPairHMM(device, false) {}

  template <class HapVec, class ReadVec>
  std::vector<std::vector<double>> compute_likelihoods(const HapVec& haplotypes, ReadVec& reads,
                                                       const TransMatrix& trans = kOriginalDefault) {
    const size_t nr = reads.size(), nh = haplotypes.size();
    std::vector<std::vector<double>> ll(nr, std::vector<double>(nh, 0.0));
    if (nr == 0 || nh == 0) return ll;
    check_status(bv_phmm_set_transitions(context(), trans.data()), "bv_phmm_set_transitions");
    score(haplotypes, reads, true, ll);
    normalize_likelihoods(ll);
    filter_poorly_modeled_reads(reads, ll);
    return ll;
  }

 private:
  void check_status(bv_status s, const char* what) {
    if (s != BV_OK)
      throw std::runtime_error(std::string(what) + ": " + bv_phmm_status_string(s) + " (" +
                               bv_phmm_last_error(context()) + ")");
  }
};

// Queues many windows (a window = the haplotypes and reads one
// compute_likelihoods call would take) and scores them in one
// bv_phmm_compute_regions call.  HaplotypeCaller::run calls the PairHMM once
// per window, one after another (haplotypecaller.hpp:126-151, the call at
// :90); with a batcher the caller adds the windows, runs once, and reads each
// window's [read][hap] matrix back, normalised and filtered exactly as a
// per-window compute_likelihoods call would (the filter edits that window's
// read vector, which must outlive run()).  scalar = true uses the scalar
// PairHMM's constant transitions.
template <class HapVec, class ReadVec>
class RegionBatcher {
 public:
  explicit RegionBatcher(GpuPairHMM& hmm, bool scalar = false,
                         const GpuScalarPairHMM::TransMatrix& trans = GpuScalarPairHMM::kOriginalDefault)
      : hmm_(hmm), scalar_(scalar), trans_(trans) {}

  size_t add(const HapVec& haplotypes, ReadVec& reads) {
    queue_.push_back({&haplotypes, &reads});
    results_.emplace_back();
    done_.push_back(false);
    return results_.size() - 1;
  }

  void run() {
    if (queue_.empty()) return;
    std::vector<int64_t> region_reads{0}, region_haps{0}, read_off{0}, hap_off{0};
    std::string rb, rq, ri, rd, rc, hb;
    // penalty views that hold one byte throughout go as uniform gap penalties
    // (the scalar model does not read them at all)
    int gap[3] = {-1, -1, -1};
    bool uniform = true;
    for (const auto& w : queue_) {
      for (const auto& r : *w.reads) {
        if (scalar_ || !uniform) break;
        const char* v[3] = {r.insertion_gop().data(), r.deletion_gop().data(), r.overall_gcp().data()};
        for (int k = 0; k < 3 && uniform; ++k)
          for (size_t x = 0; x < r.seq.size() && uniform; ++x) {
            const int b = static_cast<unsigned char>(v[k][x]);
            if (gap[k] < 0) gap[k] = b;
            uniform = b == gap[k];
          }
      }
    }
    for (const auto& w : queue_) {
      for (const auto& r : *w.reads) {
        rb.append(r.seq.data(), r.seq.size());
        rq.append(r.qual.data(), r.qual.size());
        if (!scalar_ && !uniform) {
          ri.append(r.insertion_gop().data(), r.seq.size());
          rd.append(r.deletion_gop().data(), r.seq.size());
          rc.append(r.overall_gcp().data(), r.seq.size());
        }
        read_off.push_back(static_cast<int64_t>(rb.size()));
      }
      for (const auto& h : *w.haps) {
        hb.append(h.seq.data(), h.seq.size());
        hap_off.push_back(static_cast<int64_t>(hb.size()));
      }
      region_reads.push_back(static_cast<int64_t>(read_off.size() - 1));
      region_haps.push_back(static_cast<int64_t>(hap_off.size() - 1));
    }
    auto u8 = [](const std::string& x) { return reinterpret_cast<const uint8_t*>(x.data()); };
    bv_region_batch b{};
    b.num_regions = static_cast<int64_t>(queue_.size());
    b.region_reads = region_reads.data();
    b.region_haps = region_haps.data();
    b.num_reads = static_cast<int64_t>(read_off.size() - 1);
    b.read_offsets = read_off.data();
    b.read_bases = u8(rb);
    b.read_q = u8(rq);
    if (scalar_ || uniform) {
      b.gap_ins = static_cast<uint8_t>(gap[0] < 0 ? 0 : gap[0]);
      b.gap_del = static_cast<uint8_t>(gap[1] < 0 ? 0 : gap[1]);
      b.gap_gcp = static_cast<uint8_t>(gap[2] < 0 ? 0 : gap[2]);
    } else {
      b.read_i = u8(ri);
      b.read_d = u8(rd);
      b.read_c = u8(rc);
    }
    b.num_haps = static_cast<int64_t>(hap_off.size() - 1);
    b.hap_offsets = hap_off.data();
    b.hap_bases = u8(hb);
    std::vector<double> flat(static_cast<size_t>(std::max<int64_t>(bv_phmm_region_results(&b), 1)));
    bv_phmm_ctx* ctx = hmm_.context();
    if (scalar_) throw_if(bv_phmm_set_transitions(ctx, trans_.data()), "bv_phmm_set_transitions");
    const bv_status st = bv_phmm_compute_regions(ctx, &b, flat.data(), nullptr);
    if (scalar_) bv_phmm_set_transitions(ctx, nullptr);
    throw_if(st, "bv_phmm_compute_regions");
    size_t pos = 0, k0 = results_.size() - queue_.size();
    for (size_t k = 0; k < queue_.size(); ++k) {
      auto& w = queue_[k];
      const size_t nr = w.reads->size(), nh = w.haps->size();
      std::vector<std::vector<double>> ll(nr, std::vector<double>(nh, 0.0));
      for (size_t i = 0; i < nr; ++i)
        std::copy(flat.begin() + pos + i * nh, flat.begin() + pos + (i + 1) * nh, ll[i].begin());
      pos += nr * nh;
      if (nr && nh) {
        GpuPairHMM::normalize_likelihoods(ll);
        GpuPairHMM::filter_poorly_modeled_reads(*w.reads, ll);
      }
      results_[k0 + k] = std::move(ll);
      done_[k0 + k] = true;
    }
    queue_.clear();
  }

  const std::vector<std::vector<double>>& result(size_t handle) const {
    if (handle >= results_.size() || !done_[handle]) throw std::runtime_error("window not scored yet: call run()");
    return results_[handle];
  }

 private:
  struct Window {
    const HapVec* haps;
    ReadVec* reads;
  };
  void throw_if(bv_status s, const char* what) {
    if (s != BV_OK)
      throw std::runtime_error(std::string(what) + ": " + bv_phmm_status_string(s) + " (" +
                               bv_phmm_last_error(hmm_.context()) + ")");
  }
  GpuPairHMM& hmm_;
  bool scalar_;
  GpuScalarPairHMM::TransMatrix trans_;
  std::vector<Window> queue_;
  std::vector<std::vector<std::vector<double>>> results_;
  std::vector<bool> done_;
};

}  // namespace biovoltron_b200
