// phmm_pipeline.cpp -- region-chunked compute over two contexts of one GPU.
//
// compute() copies the whole batch to the device, runs it, and copies the
// results back, one after the other.  For large batches the copies (and the
// host's planning) cost about as much as the kernels, so compute_chunked
// splits the regions into chunks and alternates them between two contexts
// (two streams, two sets of buffers): chunk k's copies and planning run
// while chunk k-1's kernels run.  Every pair is scored exactly as in
// compute(); only the sampled band audit sees different samples.
#include <algorithm>
#include <chrono>
#include <vector>

#include "phmm_engine.h"

namespace bvphmm {

bv_status Engine::mirror_config(Engine& src) {
  double tr[7];
  const bool ct = src.constant_transitions(tr);
  band_opt_.enabled = 0;  // the transitions first: they refuse a band context
  bv_status st = set_transitions(ct ? tr : nullptr);
  if (st != BV_OK) return st;
  if (src.mlp_ready_) {
    bv_status s = install_weights(src.mlp_w_.data());
    if (s != BV_OK) return s;
  }
  band_opt_ = src.band_opt_;
  std::copy(src.tune_, src.tune_ + kTuneBins + 1, tune_);
  long_warps_ = src.long_warps_;
  staged_ = false;
  destroy_graph();
  mirrored_version_ = src.config_version_;
  return BV_OK;
}

void add_stats(bv_phmm_stats& t, const bv_phmm_stats& s) {
  t.pairs += s.pairs;
  t.cells += s.cells;
  t.rescued += s.rescued;
  t.rescued_cells += s.rescued_cells;
  t.band_result_cells += s.band_result_cells;
  t.fp32_skipped_cells += s.fp32_skipped_cells;
  t.band_rescored += s.band_rescored;
  t.underflow += s.underflow;
  t.band_pairs += s.band_pairs;
  t.band_fallback += s.band_fallback;
  t.band_cells += s.band_cells;
  t.kernel_launches += s.kernel_launches;
  t.ms_h2d += s.ms_h2d;
  t.ms_fp32 += s.ms_fp32;
  t.ms_fp64 += s.ms_fp64;
  t.ms_band += s.ms_band;
  t.band_routed_full += s.band_routed_full;
  t.audit_pairs += s.audit_pairs;
  t.audit_max_err = std::max(t.audit_max_err, s.audit_max_err);
  t.audit_p99_err = std::max(t.audit_p99_err, s.audit_p99_err);  // the largest chunk p99
  t.band_promoted += s.band_promoted;
  t.ms_seed += s.ms_seed;
  t.ms_full += s.ms_full;
}

std::vector<ChunkCut> plan_chunks(const bv_region_batch& b, int chunks) {
  int64_t total = 0;
  for (int64_t g = 0; g < b.num_regions; ++g)
    total += (b.region_reads[g + 1] - b.region_reads[g]) * (b.region_haps[g + 1] - b.region_haps[g]);
  std::vector<ChunkCut> cuts;
  const int64_t target = std::max<int64_t>(1, (total + chunks - 1) / std::max(chunks, 1));
  int64_t g0 = 0, acc = 0, out0 = 0;
  for (int64_t g = 0; g < b.num_regions; ++g) {
    acc += (b.region_reads[g + 1] - b.region_reads[g]) * (b.region_haps[g + 1] - b.region_haps[g]);
    if (acc >= target || g + 1 == b.num_regions) {
      cuts.push_back(ChunkCut{g0, g + 1, out0, acc});
      out0 += acc;
      acc = 0;
      g0 = g + 1;
    }
  }
  return cuts;
}

bv_status Engine::compute_chunked(Engine& other, const bv_region_batch& b, double* out, bv_phmm_stats* stats,
                                  int chunks) {
  const auto t0 = std::chrono::steady_clock::now();
  // The chunks' reads and haplotypes are validated as each chunk is staged
  // (an invalid one ends the call with the chunks before it already written).
  bv_status s = validate_outline(b);
  if (s != BV_OK) return s;
  // results per region and the chunk cuts (about equal numbers of pairs)
  int64_t total = 0;
  for (int64_t g = 0; g < b.num_regions; ++g)
    total += (b.region_reads[g + 1] - b.region_reads[g]) * (b.region_haps[g + 1] - b.region_haps[g]);
  if (total > 0 && !out) return fail(BV_ERR_INVALID_ARG, "null output");
  std::vector<Chunk> ck;
  for (const ChunkCut& cut : plan_chunks(b, chunks)) {
    Chunk c;
    c.g0 = cut.g0;
    c.g1 = cut.g1;
    c.out0 = cut.out0;
    c.n_out = cut.n_out;
    ck.push_back(std::move(c));
  }
  Engine* eng[2] = {this, &other};
  {
    int64_t most = 1;
    for (const Chunk& c : ck) most = std::max(most, c.n_off(b));
    for (Engine* e : eng) {
      s = e->reserve_chunk_offsets(most);
      if (s != BV_OK) return fail(s, e->last_error());
    }
  }
  std::vector<bv_phmm_stats> cs(ck.size());
  auto drain = [&](size_t k) -> bv_status {  // results and stats of chunk k
    Engine& e = *eng[k % 2];
    bv_status r = e.fetch(out + ck[k].out0, ck[k].n_out);
    if (r != BV_OK) return fail(r, e.last_error());
    r = e.finish(&cs[k]);
    return r == BV_OK ? r : fail(r, e.last_error());
  };
  auto abort = [&](bv_status r) {
    // no copy from the caller's arrays may outlive the call
    cudaStreamSynchronize(stream_);
    cudaStreamSynchronize(other.stream_);
    return r;
  };
  for (size_t k = 0; k < ck.size(); ++k) {
    Engine& e = *eng[k % 2];
    // here rather than up front: the host rebases chunk k while chunk k-1 runs; chunk k-2, the
    // last user of this context's offset buffer, has been drained
    ck[k].build(b, e.chunk_offsets());
    s = e.stage(ck[k].view, false);
    if (s == BV_OK) s = e.launch();
    if (s != BV_OK) return abort(fail(s, e.last_error()));
    if (k >= 1) {
      s = drain(k - 1);
      if (s != BV_OK) return abort(s);
    }
  }
  if (!ck.empty()) {
    s = drain(ck.size() - 1);
    if (s != BV_OK) return abort(s);
  }
  if (stats) {
    *stats = bv_phmm_stats{};
    for (const auto& c : cs) add_stats(*stats, c);
    stats->ms_d2h = 0;  // the result copies overlap the next chunk's work
    stats->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return BV_OK;
}

}  // namespace bvphmm
