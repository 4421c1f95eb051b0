// adapter_check.cpp -- drives include/biovoltron_b200/gpu_pairhmm.hpp with
// record types shaped like Biovoltron's SamRecord<> / Haplotype.
// With the argument "scalar" it drives GpuScalarPairHMM (the scalar model);
// with "batch" it scores the window twice through RegionBatcher and prints
// both results one after the other.
// Input (stdin): lines "H <bases>" and "R <bases> <quals>"; quals are raw
// bytes given as printable characters.  Output: the kept reads' indices and
// the [read][hap] log10 matrix after normalize/filter, one row per line.
#include <cstdio>
#include <iostream>
#include <sstream>
#include <string>
#include <string_view>
#include <vector>

#include "biovoltron_b200/gpu_pairhmm.hpp"

struct Haplotype {
  std::string seq;
};

struct SamRecord {
  std::string seq, qual;
  int id = 0;
  std::string gop, gcp;  // full-length penalty strings ('!'+40, '!'+10)
  std::string_view insertion_gop() const { return gop; }
  std::string_view deletion_gop() const { return gop; }
  std::string_view overall_gcp() const { return gcp; }
};

int main(int argc, char** argv) {
  const bool scalar = argc > 1 && std::string(argv[1]) == "scalar";
  std::vector<Haplotype> haps;
  std::vector<SamRecord> reads;
  std::string line;
  while (std::getline(std::cin, line)) {
    std::istringstream ss(line);
    std::string tag;
    ss >> tag;
    if (tag == "H") {
      Haplotype h;
      ss >> h.seq;
      haps.push_back(h);
    } else if (tag == "R") {
      SamRecord r;
      ss >> r.seq >> r.qual;
      r.id = (int)reads.size();
      r.gop.assign(r.seq.size(), (char)(40 + '!'));
      r.gcp.assign(r.seq.size(), (char)(10 + '!'));
      reads.push_back(r);
    }
  }
  std::vector<std::vector<double>> ll;
  if (argc > 1 && std::string(argv[1]) == "batch") {
    // two copies of the window through the region batcher: both must equal one call
    biovoltron_b200::GpuPairHMM hmm(0);
    std::vector<SamRecord> copy = reads;
    biovoltron_b200::RegionBatcher<std::vector<Haplotype>, std::vector<SamRecord>> batcher(hmm);
    const size_t a = batcher.add(haps, reads), b = batcher.add(haps, copy);
    batcher.run();
    for (size_t w : {a, b}) {
      const auto& rr = w == a ? reads : copy;
      std::printf("kept");
      for (const auto& r : rr) std::printf(" %d", r.id);
      std::printf("\n");
      for (const auto& row : batcher.result(w)) {
        for (size_t j = 0; j < row.size(); ++j) std::printf(j ? " %.9f" : "%.9f", row[j]);
        std::printf("\n");
      }
    }
    return 0;
  }
  if (scalar) {
    biovoltron_b200::GpuScalarPairHMM hmm(0);
    ll = hmm.compute_likelihoods(haps, reads);
  } else {
    biovoltron_b200::GpuPairHMM hmm(0);
    ll = hmm.compute_likelihoods(haps, reads);
  }
  std::printf("kept");
  for (const auto& r : reads) std::printf(" %d", r.id);
  std::printf("\n");
  for (const auto& row : ll) {
    for (size_t j = 0; j < row.size(); ++j) std::printf(j ? " %.9f" : "%.9f", row[j]);
    std::printf("\n");
  }
  return 0;
}
