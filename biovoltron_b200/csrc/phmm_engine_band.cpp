// phmm_engine_band.cpp -- the engine's learned-band path (see phmm_band.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "phmm_engine.h"
#include "phmm_rows.h"

namespace bvphmm {

#define BV_CUDA(call, what)                                  \
  do {                                                       \
    cudaError_t e__ = (call);                                \
    if (e__ != cudaSuccess) return cuda_fail(e__, what);     \
  } while (0)

namespace {
int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
}  // namespace

bv_status Engine::set_band_options(const bv_band_options& o) {
  if (o.struct_size != (int32_t)sizeof(bv_band_options)) return fail(BV_ERR_INVALID_ARG, "band options size");
  if (o.fixed_half < 0 || o.fixed_half > 15 || o.margin < 0 || o.margin > 15 || o.audit_period < 0 ||
      !(o.edge_threshold > 0) || !(o.cap_margin >= 0.f) || !(o.cap_margin < 1e30f))
    return fail(BV_ERR_INVALID_ARG, "band option out of range");
  if (o.enabled && o.use_mlp && !mlp_ready_) return fail(BV_ERR_INVALID_ARG, "no band MLP weights (train or load)");
  if (o.enabled && constant_transitions(nullptr))
    return fail(BV_ERR_UNSUPPORTED, "the band path takes its transitions from the quality bytes");
  band_opt_ = o;
  ++config_version_;
  staged_ = false;  // buffers and launch sequence depend on the mode: stage again
  destroy_graph();
  return BV_OK;
}

BandParams Engine::band_params() const {
  BandParams p{};
  p.batch.read_bases = d_read_bases_.as<uint8_t>();
  p.batch.read_quals = d_quals4_.as<uchar4>();
  p.batch.read_off = d_read_off_.as<int64_t>();
  p.batch.hap_bases = d_hap_bases_.as<uint8_t>();
  p.batch.hap_off = d_hap_off_.as<int64_t>();
  p.tables = d_tables_.as<Tables>();
  p.n_pairs = n_results_;
  p.pair_read = d_pair_read_.as<int32_t>();
  p.pair_hap = d_pair_hap_.as<int32_t>();
  p.hap_table = d_hap_table_.as<uint32_t>();
  p.hap_nib = d_hap_nib_.as<uint32_t>();
  p.units = d_units_.as<Unit>();
  p.n_units = (long long)units_.size();
  p.read_kmers = d_read_kmers_.as<uint32_t>();
  p.feat_hist = d_feat_hist_.as<uint32_t>();
  p.feat_slow = d_feat_slow_.as<int64_t>();
  p.dstar = d_dstar_.as<int32_t>();
  p.kmin = d_kmin_.as<int32_t>();
  p.kmax = d_kmax_.as<int32_t>();
  p.feat = d_feat_.as<__nv_bfloat16>();
  p.mlp_out = d_mlp_out_.as<float>();
  p.mlp = d_mlp_.as<MlpParams>();
  p.use_mlp = band_opt_.use_mlp;
  p.fixed_half = band_opt_.fixed_half;
  p.margin = band_opt_.margin;
  p.edge_threshold = (float)band_opt_.edge_threshold;
  p.audit_period = band_opt_.audit_period;
  p.cap_margin = band_opt_.cap_margin;
  p.banded = d_banded_.as<uint8_t>();
  p.cap_items = d_cap_items_.as<Unit>();
  p.bctr = d_bctr_.as<BandCounters>();
  p.ctr = d_counters_.as<Counters>();
  p.items = d_band_items_.as<BandItem>();
  p.item_cap = item_cap_;
  p.full_items = d_full_items_.as<Unit>();
  p.full_cap = full_cap_;
  p.audit_pairs = d_audit_pairs_.as<int64_t>();
  p.audit_cap = audit_cap_;
  p.out = d_out_.as<double>();
  p.audit_out = d_audit_out_.as<double>();
  p.rescue = d_rescue_.as<PairRef>();
  p.rescue_cap = std::max<int64_t>(n_results_, 1);
  return p;
}

bv_status Engine::band_prepare() {
  const int64_t n = std::max<int64_t>(n_results_, 1);
  BV_CUDA(prepare_band_kernels(), "band kernel attributes");
  BV_CUDA(d_pair_read_.reserve(sizeof(int32_t) * n), "alloc pairs");
  BV_CUDA(d_pair_hap_.reserve(sizeof(int32_t) * n), "alloc pairs");
  BV_CUDA(d_hap_table_.reserve(sizeof(uint32_t) * (size_t)hap_table_words(std::max<int64_t>(n_hap_bytes_, 1), n_haps_)),
          "alloc hap tables");
  BV_CUDA(d_hap_nib_.reserve(sizeof(uint32_t) * (size_t)hap_nibble_words(std::max<int64_t>(n_hap_bytes_, 1))),
          "alloc haplotype nibbles");
  BV_CUDA(d_read_kmers_.reserve(sizeof(uint32_t) * std::max<int64_t>(n_read_bytes_, 1)), "alloc kmers");
  BV_CUDA(d_feat_hist_.reserve(sizeof(uint32_t) * (size_t)feat_hist_words(sms_)), "alloc featuriser scratch");
  BV_CUDA(d_feat_slow_.reserve(sizeof(int64_t) * n), "alloc featuriser list");
  BV_CUDA(d_dstar_.reserve(sizeof(int32_t) * n), "alloc seeds");
  BV_CUDA(d_kmin_.reserve(sizeof(int32_t) * n), "alloc seeds");
  BV_CUDA(d_kmax_.reserve(sizeof(int32_t) * n), "alloc seeds");
  BV_CUDA(d_feat_.reserve(sizeof(__nv_bfloat16) * kFeat * n), "alloc features");
  BV_CUDA(d_mlp_out_.reserve(sizeof(float) * kOut * n), "alloc mlp out");
  BV_CUDA(d_mlp_.reserve(sizeof(MlpParams)), "alloc mlp");
  BV_CUDA(d_bctr_.reserve(sizeof(BandCounters)), "alloc band counters");
  item_cap_ = n;
  full_cap_ = n;
  audit_cap_ = band_opt_.audit_period > 0 ? n / band_opt_.audit_period + 1 : 1;
  BV_CUDA(d_band_items_.reserve(sizeof(BandItem) * kBandWidths * item_cap_), "alloc band items");
  BV_CUDA(d_full_items_.reserve(sizeof(Unit) * 9 * full_cap_), "alloc fallback units");
  BV_CUDA(d_banded_.reserve((size_t)n), "alloc band flags");
  BV_CUDA(d_cap_items_.reserve(sizeof(Unit) * 9 * (band_opt_.cap_margin > 0 ? full_cap_ : 1)), "alloc rescore units");
  BV_CUDA(d_audit_pairs_.reserve(sizeof(int64_t) * audit_cap_), "alloc audit");
  BV_CUDA(d_audit_units_.reserve(sizeof(Unit) * 9 * audit_cap_), "alloc audit");
  BV_CUDA(d_audit_out_.reserve(sizeof(double) * audit_cap_), "alloc audit");
  BV_CUDA(d_audit_err_.reserve(sizeof(double) * audit_cap_), "alloc audit");
  // Fallback launches: one persistent launch per full-DP variant, sized for the
  // batch's longest haplotype; the unit counts are known only on the device.
  size_t need32 = d_bnd32_.capacity();
  for (int v = 0; v < 9; ++v) {
    LaunchPlan lp;
    lp.variant = v;
    lp.slot = v;
    lp.multi = (v == 8);
    lp.hap_bytes = (int)round_up((int64_t)std::max(max_hap_, 1) + (kWarp - 1) + (lp.multi ? 32 : 8) + kHapLead + 16, 16);
    lp.warp_smem = warp_smem_bytes(v, lp.hap_bytes);
    const int smem_block = lp.warp_smem * (kThreadsPerBlock / kWarp);
    if (smem_block > 227 * 1024) return fail(BV_ERR_INVALID_ARG, "haplotype too long for shared-memory staging");
    BV_CUDA(prepare_variant(v, smem_block), "kernel attribute");
    lp.grid = sms_ * std::max(1, blocks_per_sm(v, smem_block));
    lp.bnd_cols = lp.multi ? round_up((int64_t)std::max(max_hap_, 1) + kWarp, 32) + 160 : 0;
    if (lp.multi) need32 = std::max<size_t>(need32, (size_t)lp.grid * (kThreadsPerBlock / kWarp) * lp.bnd_cols * 4 * sizeof(float));
    full_plans_[v] = lp;
  }
  if (need32 > d_bnd32_.capacity()) BV_CUDA(d_bnd32_.reserve(need32), "alloc boundary buffers");
  BV_CUDA(launch_pairs_from_units(d_units_.as<Unit>(), (long long)units_.size(), d_pair_read_.as<int32_t>(),
                                  d_pair_hap_.as<int32_t>(), sms_, stream_), "pairs");
  return BV_OK;
}

bv_status Engine::enqueue_band(bool capturing, KernelParams& kp) {
  auto rec = [&](cudaEvent_t ev) {
    return capturing ? cudaEventRecordWithFlags(ev, stream_, cudaEventRecordExternal) : cudaEventRecord(ev, stream_);
  };
  BandParams p = band_params();
  BV_CUDA(cudaMemsetAsync(d_bctr_.get(), 0, sizeof(BandCounters), stream_), "memset band counters");
  BV_CUDA(launch_hap_table(p.batch.hap_bases, p.batch.hap_off, n_haps_, n_hap_bytes_, d_hap_table_.as<uint32_t>(),
                           d_hap_nib_.as<uint32_t>(), sms_, stream_),
          "hap tables");
  BV_CUDA(launch_read_kmers(p.batch.read_bases, n_read_bytes_, d_read_kmers_.as<uint32_t>(), sms_, stream_), "kmers");
  BV_CUDA(launch_gap_check(p.batch.read_quals, n_read_bytes_, p.bctr, sms_, stream_), "gap check");
  BV_CUDA(launch_featurize(p, sms_, stream_), "featurize");
  if (p.use_mlp) BV_CUDA(launch_mlp_forward(p, sms_, stream_), "mlp");
  BV_CUDA(launch_band_route(p, 0, sms_, stream_), "route");
  BV_CUDA(launch_band_scan(p.bctr, stream_), "scan");
  BV_CUDA(launch_band_route(p, 1, sms_, stream_), "route");
  BV_CUDA(rec(ev_[5]), "event");
  for (int cls = 0; cls < kBandWidths; ++cls) BV_CUDA(launch_band_dp(p, cls, sms_, stream_), "band dp");
  BV_CUDA(rec(ev_[6]), "event");
  // full DP for everything the band path handed back
  for (int v = 0; v < 9; ++v) {
    const LaunchPlan& lp = full_plans_[v];
    kp.units = d_full_items_.as<Unit>() + (size_t)v * full_cap_;
    kp.unit_base = 0;
    kp.n_units = 0;
    kp.n_units_dev = &d_bctr_.as<BandCounters>()->full_count[v];
    kp.slot = lp.slot;
    kp.from_rescue = 0;
    kp.hap_bytes = lp.hap_bytes;
    kp.warp_smem_bytes = lp.warp_smem;
    kp.bnd = lp.multi ? d_bnd32_.get() : nullptr;
    kp.bnd_cols = lp.bnd_cols;
    kp.rescale = 0;
    kp.rescale_target = 0;
    BV_CUDA(launch_forward(v, kp, lp.grid, stream_), "fallback full DP");
  }
  if (band_opt_.cap_margin > 0) {
    // banded pairs far below their read's best result, scored again by the full DP
    BV_CUDA(launch_band_cap(p, sms_, stream_), "band cap");
    for (int v = 0; v < 9; ++v) {
      const LaunchPlan& lp = full_plans_[v];
      kp.units = d_cap_items_.as<Unit>() + (size_t)v * full_cap_;
      kp.unit_base = 0;
      kp.n_units = 0;
      kp.n_units_dev = &d_bctr_.as<BandCounters>()->cap_count[v];
      kp.slot = kCapSlot0 + v;
      kp.from_rescue = 0;
      kp.hap_bytes = lp.hap_bytes;
      kp.warp_smem_bytes = lp.warp_smem;
      kp.bnd = lp.multi ? d_bnd32_.get() : nullptr;
      kp.bnd_cols = lp.bnd_cols;
      kp.rescale = 0;
      kp.rescale_target = 0;
      BV_CUDA(launch_forward(v, kp, lp.grid, stream_), "rescore full DP");
    }
  }
  if (band_opt_.audit_period > 0) {
    BV_CUDA(launch_audit_units(p, d_audit_units_.as<Unit>(), stream_), "audit units");
    // the audit pairs' full DP, on the variant each read length takes
    for (int v = 0; v < 9; ++v) {
      KernelParams ak = kp;
      const LaunchPlan& lp = full_plans_[v];
      ak.units = d_audit_units_.as<Unit>() + (size_t)v * audit_cap_;
      ak.n_units_dev = &d_bctr_.as<BandCounters>()->audit_var[v];
      ak.slot = 16 + v;
      ak.hap_bytes = lp.hap_bytes;
      ak.warp_smem_bytes = lp.warp_smem;
      ak.bnd = lp.multi ? d_bnd32_.get() : nullptr;
      ak.bnd_cols = lp.bnd_cols;
      ak.out = d_audit_out_.as<double>();
      ak.rescue = nullptr;  // audit pairs that need FP64 are left out of the comparison
      BV_CUDA(launch_forward(v, ak, lp.grid, stream_), "audit full DP");
    }
  }
  kp.n_units_dev = nullptr;
  return BV_OK;
}

bv_status Engine::band_stats(bv_phmm_stats* st) {
  BandCounters bc{};
  BV_CUDA(cudaMemcpy(&bc, d_bctr_.get(), sizeof(bc), cudaMemcpyDeviceToHost), "band counters");
  long long banded = 0;
  for (int c = 0; c < kBandWidths; ++c)
    for (int b = 0; b < kRBuckets; ++b) banded += (long long)bc.band_count[c][b];
  st->band_pairs = banded;
  st->band_fallback = (int64_t)bc.fallback_edge;
  st->band_routed_full = (int64_t)bc.fallback_route;
  st->band_cells = (int64_t)bc.band_cells;
  st->band_result_cells = (int64_t)bc.band_result_cells;
  st->band_rescored = (int64_t)bc.cap_flagged;
  st->band_promoted = 0;
  for (int c = 0; c < kBandWidths; ++c) st->band_promoted += (int64_t)bc.promoted[c];
  const long long na = std::min<long long>((long long)bc.audit_count, audit_cap_);
  st->audit_pairs = band_opt_.audit_period > 0 ? na : 0;
  st->audit_max_err = 0;
  st->audit_p99_err = 0;
  if (band_opt_.audit_period > 0 && na > 0) {
    std::vector<double> err((size_t)na);
    BV_CUDA(cudaMemcpy(err.data(), d_audit_err_.get(), sizeof(double) * na, cudaMemcpyDeviceToHost), "audit errors");
    std::vector<double> e;
    e.reserve(err.size());
    for (double v : err)
      if (std::isfinite(v)) e.push_back(v);
    if (!e.empty()) {
      std::sort(e.begin(), e.end());
      st->audit_max_err = e.back();
      st->audit_p99_err = e[(size_t)std::min<double>(e.size() - 1, std::floor(0.99 * (e.size() - 1)))];
    }
    st->audit_pairs = (int64_t)e.size();
  }
  return BV_OK;
}

bv_status Engine::band_routes(int64_t n, int32_t* d_lo, int32_t* width, int32_t* route) {
  if (!band_enabled() || !staged_) return fail(BV_ERR_INVALID_ARG, "no band-mode batch has run");
  if (n != n_results_) return fail(BV_ERR_INVALID_ARG, "result count");
  BandCounters bc{};
  Counters cc{};
  BV_CUDA(cudaMemcpy(&bc, d_bctr_.get(), sizeof(bc), cudaMemcpyDeviceToHost), "band counters");
  BV_CUDA(cudaMemcpy(&cc, d_counters_.get(), sizeof(cc), cudaMemcpyDeviceToHost), "counters");
  std::fill(d_lo, d_lo + n, 0);
  std::fill(width, width + n, 0);
  std::fill(route, route + n, 1);
  for (int c = 0; c < kBandWidths; ++c) {
    unsigned long long cnt = bc.band_total[c] + bc.promoted[c];
    cnt = std::min<unsigned long long>(cnt, (unsigned long long)item_cap_);
    std::vector<BandItem> it(cnt);
    if (cnt) BV_CUDA(cudaMemcpy(it.data(), d_band_items_.as<BandItem>() + (size_t)c * item_cap_, sizeof(BandItem) * cnt,
                                cudaMemcpyDeviceToHost), "band items");
    for (const auto& x : it) {
      if (x.out < 0 || x.out >= n) continue;
      d_lo[x.out] = x.d_lo;
      width[x.out] = band_width(c);
      route[x.out] = 0;
    }
  }
  for (int v = 0; v < 9; ++v) {
    const unsigned long long cnt = std::min<unsigned long long>(bc.full_count[v], (unsigned long long)full_cap_);
    std::vector<Unit> u(cnt);
    if (cnt) BV_CUDA(cudaMemcpy(u.data(), d_full_items_.as<Unit>() + (size_t)v * full_cap_, sizeof(Unit) * cnt,
                                cudaMemcpyDeviceToHost), "fallback units");
    for (const auto& x : u)
      if (x.out0 >= 0 && x.out0 < n && route[x.out0] == 0) route[x.out0] = 2;
  }
  const unsigned long long nr = std::min<unsigned long long>(cc.rescue_count, (unsigned long long)std::max<int64_t>(n_results_, 1));
  std::vector<PairRef> rl(nr);
  if (nr) BV_CUDA(cudaMemcpy(rl.data(), d_rescue_.get(), sizeof(PairRef) * nr, cudaMemcpyDeviceToHost), "rescue list");
  const unsigned long long nl =
      std::min<unsigned long long>(cc.rescue_long_count, (unsigned long long)std::max<int64_t>(n_results_, 1) - nr);
  rl.resize(nr + nl);
  if (nl) BV_CUDA(cudaMemcpy(rl.data() + nr, d_rescue_.as<PairRef>() + (std::max<int64_t>(n_results_, 1) - (int64_t)nl),
                             sizeof(PairRef) * nl, cudaMemcpyDeviceToHost), "rescue list");
  if (band_opt_.cap_margin > 0) {
    for (int v = 0; v < 9; ++v) {
      const unsigned long long cnt = std::min<unsigned long long>(bc.cap_count[v], (unsigned long long)full_cap_);
      std::vector<Unit> u(cnt);
      if (cnt) BV_CUDA(cudaMemcpy(u.data(), d_cap_items_.as<Unit>() + (size_t)v * full_cap_, sizeof(Unit) * cnt,
                                  cudaMemcpyDeviceToHost), "rescore units");
      for (const auto& x : u)
        if (x.out0 >= 0 && x.out0 < n && route[x.out0] == 0) route[x.out0] = 4;
    }
  }
  for (const auto& x : rl)
    if (x.out >= 0 && x.out < n && (route[x.out] == 0 || route[x.out] == 4)) route[x.out] = 3;
  return BV_OK;
}

}  // namespace bvphmm
