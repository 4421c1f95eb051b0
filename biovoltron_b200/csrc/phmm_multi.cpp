// phmm_multi.cpp -- one region batch over several devices.
//
// Pairs and regions are independent, so several GPUs share a batch with no
// exchange between them.  The regions are cut into contiguous blocks of about
// equal DP cells (sum over the block's regions of read bases x haplotype
// bases) and the blocks are dealt to the devices by greedy LPT (longest
// processing time first): largest block first, each to the device with the
// fewest cells so far.  A block is a rebased view of the caller's arrays (no
// host copy); each device scores its blocks through its own context, one host
// thread per context, and every result lands at its region's offset, so the
// output is in region order exactly as one context would write it.
#include <algorithm>
#include <chrono>
#include <numeric>
#include <thread>
#include <vector>

#include "phmm_engine.h"

namespace bvphmm {

Partition plan_partition(const bv_region_batch& b, int n_parts, int n_blocks) {
  Partition pt;
  const int64_t ng = b.num_regions;
  std::vector<int64_t> cells(ng), pairs(ng);
  int64_t total = 0;
  for (int64_t g = 0; g < ng; ++g) {
    const int64_t r0 = b.region_reads[g], r1 = b.region_reads[g + 1];
    const int64_t h0 = b.region_haps[g], h1 = b.region_haps[g + 1];
    const int64_t rb = r1 > r0 ? b.read_offsets[r1] - b.read_offsets[r0] : 0;
    const int64_t hb = h1 > h0 ? b.hap_offsets[h1] - b.hap_offsets[h0] : 0;
    cells[g] = rb * hb;
    pairs[g] = (r1 - r0) * (h1 - h0);
    total += cells[g];
  }
  // contiguous blocks of about total / n_blocks cells (one region at least);
  // as many blocks as regions: one region per block
  const int64_t nb = std::max<int64_t>(1, std::min<int64_t>(n_blocks, ng));
  const int64_t target = std::max<int64_t>(1, (total + nb - 1) / nb);
  int64_t g0 = 0, acc = 0, out0 = 0, acc_pairs = 0;
  for (int64_t g = 0; g < ng; ++g) {
    acc += cells[g];
    acc_pairs += pairs[g];
    if (acc >= target || g + 1 == ng || nb == ng) {
      pt.block_start.push_back(g0);
      pt.block_cells.push_back(acc);
      pt.block_out0.push_back(out0);
      pt.block_pairs.push_back(acc_pairs);
      out0 += acc_pairs;
      g0 = g + 1;
      acc = 0;
      acc_pairs = 0;
    }
  }
  pt.block_start.push_back(ng);
  // greedy LPT: blocks by cells, largest first (lower index on ties), each to
  // the part with the fewest cells so far (lower index on ties)
  const size_t nblk = pt.block_cells.size();
  std::vector<size_t> order(nblk);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t x, size_t y) { return pt.block_cells[x] > pt.block_cells[y]; });
  pt.part_cells.assign(std::max(n_parts, 1), 0);
  pt.block_part.assign(nblk, 0);
  for (size_t k : order) {
    const int p = (int)(std::min_element(pt.part_cells.begin(), pt.part_cells.end()) - pt.part_cells.begin());
    pt.block_part[k] = p;
    pt.part_cells[p] += pt.block_cells[k];
  }
  return pt;
}

}  // namespace bvphmm

extern "C" int64_t bv_phmm_plan_partition(const bv_region_batch* batch, int32_t n_parts, int32_t n_blocks,
                                          int64_t* block_start, int32_t* block_part, int64_t* part_cells) {
  if (!batch || n_parts < 1 || n_blocks < 1 || batch->num_regions < 0 ||
      (batch->num_regions > 0 && (!batch->region_reads || !batch->region_haps || !batch->read_offsets ||
                                  !batch->hap_offsets)))
    return -1;
  const bvphmm::Partition pt = bvphmm::plan_partition(*batch, n_parts, n_blocks);
  const size_t nb = pt.block_part.size();
  if (block_start) std::copy(pt.block_start.begin(), pt.block_start.end(), block_start);
  if (block_part) std::copy(pt.block_part.begin(), pt.block_part.end(), block_part);
  if (part_cells) std::copy(pt.part_cells.begin(), pt.part_cells.end(), part_cells);
  return (int64_t)nb;
}

extern "C" bv_status bv_phmm_compute_regions_multi(bv_phmm_ctx* const* ctxs, int32_t n_ctx,
                                                   const bv_region_batch* batch, double* out_log10,
                                                   bv_phmm_stats* stats) {
  using namespace bvphmm;
  const auto t0 = std::chrono::steady_clock::now();
  if (!ctxs || n_ctx < 1 || !batch) return BV_ERR_INVALID_ARG;
  for (int k = 0; k < n_ctx; ++k) {
    if (!ctxs[k]) return BV_ERR_INVALID_ARG;
    for (int j = 0; j < k; ++j)
      if (ctxs[j] == ctxs[k]) return BV_ERR_INVALID_ARG;  // a context is not thread-safe
  }
  if (batch->num_regions < 0 ||
      (batch->num_regions > 0 && (!batch->region_reads || !batch->region_haps)) ||
      (batch->num_reads > 0 && !batch->read_offsets) || (batch->num_haps > 0 && !batch->hap_offsets))
    return BV_ERR_INVALID_ARG;
  for (int64_t g = 0; g < batch->num_regions; ++g)
    if (batch->region_reads[g] > batch->region_reads[g + 1] || batch->region_haps[g] > batch->region_haps[g + 1] ||
        batch->region_reads[g] < 0 || batch->region_haps[g] < 0 || batch->region_reads[g + 1] > batch->num_reads ||
        batch->region_haps[g + 1] > batch->num_haps)
      return BV_ERR_INVALID_ARG;
  if (bv_phmm_region_results(batch) > 0 && !out_log10) return BV_ERR_INVALID_ARG;
  // a few blocks per device so that LPT can even out uneven regions
  const Partition pt = plan_partition(*batch, n_ctx, 16 * n_ctx);
  const size_t nb = pt.block_part.size();
  std::vector<bv_status> status(n_ctx, BV_OK);
  std::vector<bv_phmm_stats> st(n_ctx);
  auto work = [&](int k) {
    bv_phmm_stats acc{};
    // runs of consecutive blocks on this device go as one view
    for (size_t x = 0; x < nb && status[k] == BV_OK;) {
      if (pt.block_part[x] != k) { ++x; continue; }
      size_t y = x + 1;
      while (y < nb && pt.block_part[y] == k) ++y;
      Chunk c;
      c.g0 = pt.block_start[x];
      c.g1 = pt.block_start[y];
      c.out0 = pt.block_out0[x];
      std::vector<int64_t> off((size_t)c.n_off(*batch));  // the view is copied from within the call below
      c.build(*batch, off.data());
      bv_phmm_stats s{};
      status[k] = bv_phmm_compute_regions(ctxs[k], &c.view, out_log10 ? out_log10 + c.out0 : nullptr, &s);
      add_stats(acc, s);
      x = y;
    }
    st[k] = acc;
  };
  std::vector<std::thread> th;
  for (int k = 1; k < n_ctx; ++k) th.emplace_back(work, k);
  work(0);
  for (auto& t : th) t.join();
  for (int k = 0; k < n_ctx; ++k)
    if (status[k] != BV_OK) return status[k];
  if (stats) {
    *stats = bv_phmm_stats{};
    for (const auto& s : st) add_stats(*stats, s);
    stats->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return BV_OK;
}
