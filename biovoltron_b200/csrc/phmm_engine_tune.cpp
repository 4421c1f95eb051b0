// phmm_engine_tune.cpp -- per-bin launch-shape autotuner of the full-DP kernels.
//
// A bin is the set of reads whose single-strip FP32 kernel has the same rows
// per lane.  The tuner stages the sample once per candidate shape (haplotypes
// per warp x warps per block), runs it directly (not from a graph) with
// events around every bin launch, and keeps per bin the shape with the
// smallest median time.
#include <algorithm>
#include <vector>

#include "phmm_engine.h"

namespace bvphmm {

#define BV_CUDA(call, what)                              \
  do {                                                   \
    cudaError_t e__ = (call);                            \
    if (e__ != cudaSuccess) return cuda_fail(e__, what); \
  } while (0)

bv_status Engine::set_tuning(const bv_phmm_tune_entry* e, int32_t n) {
  if (n < 0 || (n > 0 && !e)) return fail(BV_ERR_INVALID_ARG, "tuning entries");
  for (int32_t i = 0; i < n; ++i) {
    if (e[i].rows_per_lane < 1 || e[i].rows_per_lane > kTuneBins ||
        (e[i].haps_per_warp != 1 && e[i].haps_per_warp != 2) || e[i].warps_per_block < 1 ||
        e[i].warps_per_block > kThreadsPerBlock / kWarp)
      return fail(BV_ERR_INVALID_ARG, "tuning entry out of range");
  }
  for (int32_t i = 0; i < n; ++i) {
    tune_[e[i].rows_per_lane].haps_per_warp = e[i].haps_per_warp;
    tune_[e[i].rows_per_lane].warps_per_block = e[i].warps_per_block;
  }
  ++config_version_;
  staged_ = false;  // the launch plan depends on it: stage again
  destroy_graph();
  return BV_OK;
}

bv_status Engine::get_tuning(bv_phmm_tune_entry* out, int32_t* n_out) {
  if (!out || !n_out) return fail(BV_ERR_INVALID_ARG, "null output");
  for (int rt = 1; rt <= kTuneBins; ++rt) {
    bv_phmm_tune_entry t{};
    t.rows_per_lane = rt;
    t.haps_per_warp = tune_[rt].haps_per_warp;
    t.warps_per_block = tune_[rt].warps_per_block;
    out[rt - 1] = t;
  }
  *n_out = kTuneBins;
  return BV_OK;
}

bv_status Engine::autotune(const bv_region_batch& sample, int repeats, bv_phmm_tune_entry* out, int32_t* n_out) {
  if (!out || !n_out) return fail(BV_ERR_INVALID_ARG, "null output");
  if (repeats < 1 || repeats > 64) return fail(BV_ERR_INVALID_ARG, "repeats out of range");
  if (band_enabled()) return fail(BV_ERR_INVALID_ARG, "autotune runs the full-DP path: disable the band first");
  if (opt_.precision == BV_PRECISION_F64) return fail(BV_ERR_INVALID_ARG, "autotune needs FP32 precision");
  const int saved_hpw = opt_.haps_per_warp;
  opt_.haps_per_warp = 0;  // the per-bin table decides
  BinTune saved[kTuneBins + 1];
  std::copy(tune_, tune_ + kTuneBins + 1, saved);
  struct Cand {
    int hpw, wpb;
  };
  const Cand cands[] = {{2, 4}, {2, 2}, {2, 1}, {1, 4}, {1, 2}, {1, 1}};
  constexpr int kCands = (int)(sizeof(cands) / sizeof(cands[0]));
  double best[kTuneBins + 1];
  int best_c[kTuneBins + 1];
  for (int rt = 0; rt <= kTuneBins; ++rt) {
    best[rt] = 1e300;
    best_c[rt] = -1;
  }
  bv_status s = BV_OK;
  for (int c = 0; c < kCands && s == BV_OK; ++c) {
    for (int rt = 1; rt <= kTuneBins; ++rt) {
      tune_[rt].haps_per_warp = cands[c].hpw;
      tune_[rt].warps_per_block = cands[c].wpb;
    }
    s = stage(sample);
    if (s != BV_OK) break;
    std::vector<int> plan_rt(plans_.size(), 0);  // bin of each launch
    for (size_t i = 0; i < plans_.size(); ++i)
      for (int t = 1; t <= kTuneBins; ++t)
        if (plans_[i].variant == variant_index(false, t, false, false) ||
            plans_[i].variant == variant_index(false, t, false, true))
          plan_rt[i] = t;
    std::vector<std::vector<float>> times(plans_.size());
    tune_timing_ = true;
    for (int k = 0; k <= repeats && s == BV_OK; ++k) {  // the first run warms up
      s = enqueue_kernels(false);
      if (s != BV_OK) break;
      cudaError_t e = cudaStreamSynchronize(stream_);
      if (e != cudaSuccess) {
        s = cuda_fail(e, "tune sync");
        break;
      }
      Counters cc{};
      e = cudaMemcpy(&cc, d_counters_.get(), sizeof(cc), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) {
        s = cuda_fail(e, "tune counters");
        break;
      }
      if (cc.status != 0) {
        s = status_fail(cc.status);
        break;
      }
      if (k == 0) continue;
      for (size_t i = 0; i < plans_.size(); ++i) {
        float ms = 0;
        cudaEventElapsedTime(&ms, tune_ev_[2 * i], tune_ev_[2 * i + 1]);
        times[i].push_back(ms);
      }
    }
    tune_timing_ = false;
    if (s != BV_OK) break;
    for (size_t i = 0; i < plans_.size(); ++i) {
      if (!plan_rt[i] || times[i].empty()) continue;
      std::vector<float> t = times[i];
      std::nth_element(t.begin(), t.begin() + t.size() / 2, t.end());
      const double med = t[t.size() / 2];
      if (med < best[plan_rt[i]]) {
        best[plan_rt[i]] = med;
        best_c[plan_rt[i]] = c;
      }
    }
  }
  opt_.haps_per_warp = saved_hpw;
  std::copy(saved, saved + kTuneBins + 1, tune_);
  staged_ = false;  // the sample was staged with trial shapes
  destroy_graph();
  if (s != BV_OK) return s;
  int32_t n = 0;
  for (int rt = 1; rt <= kTuneBins; ++rt) {
    if (best_c[rt] < 0) continue;
    tune_[rt].haps_per_warp = cands[best_c[rt]].hpw;
    tune_[rt].warps_per_block = cands[best_c[rt]].wpb;
    bv_phmm_tune_entry t{};
    t.rows_per_lane = rt;
    t.haps_per_warp = tune_[rt].haps_per_warp;
    t.warps_per_block = tune_[rt].warps_per_block;
    t.ms = best[rt];
    out[n++] = t;
  }
  *n_out = n;
  ++config_version_;
  return BV_OK;
}

bv_status Engine::set_long_warps(int warps) {
  if (!long_warps_valid(warps)) return fail(BV_ERR_INVALID_ARG, "long-read warps per pair must be 2, 4 or 8");
  if (warps != long_warps_) {
    long_warps_ = warps;
    ++config_version_;
    staged_ = false;  // the FP64 lists and launch plan depend on it: stage again
    destroy_graph();
  }
  return BV_OK;
}

// The long-read kernel's shape: for each candidate warps per pair (and with
// it the long-read edge, 128 x warps bases) the sample is staged in FP64 mode
// -- every pair on the FP64 kernels, long reads on the long-read kernel, the
// rest on the one-warp kernel -- and its FP64 pass timed (repeats runs after
// a warm-up, median); the fastest is installed.
bv_status Engine::autotune_long(const bv_region_batch& sample, int repeats, int32_t* warps_out, double* ms_out) {
  if (!warps_out || !ms_out) return fail(BV_ERR_INVALID_ARG, "null output");
  if (repeats < 1 || repeats > 64) return fail(BV_ERR_INVALID_ARG, "repeats out of range");
  if (band_enabled()) return fail(BV_ERR_INVALID_ARG, "autotune runs the full-DP path: disable the band first");
  const int cands[3] = {2, 4, 8};
  for (int c = 0; c < 3; ++c) ms_out[c] = 0.0;
  const int saved_warps = long_warps_;
  const int32_t saved_precision = opt_.precision;
  opt_.precision = BV_PRECISION_F64;
  int best = saved_warps;
  double best_ms = 1e300;
  bv_status s = BV_OK;
  for (int c = 0; c < 3 && s == BV_OK; ++c) {
    long_warps_ = cands[c];
    s = stage(sample);
    if (s != BV_OK) break;
    if (long_plan_.grid == 0) continue;  // no read this long, or its haplotypes too long for the kernel
    std::vector<float> t;
    for (int k = 0; k <= repeats && s == BV_OK; ++k) {  // the first run warms up
      s = enqueue_kernels(false);
      if (s != BV_OK) break;
      cudaError_t e = cudaStreamSynchronize(stream_);
      if (e != cudaSuccess) {
        s = cuda_fail(e, "tune sync");
        break;
      }
      Counters cc{};
      e = cudaMemcpy(&cc, d_counters_.get(), sizeof(cc), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) {
        s = cuda_fail(e, "tune counters");
        break;
      }
      if (cc.status != 0) {
        s = status_fail(cc.status);
        break;
      }
      float ms = 0;
      cudaEventElapsedTime(&ms, ev_[3], ev_[4]);
      if (k > 0) t.push_back(ms);
    }
    if (s != BV_OK || t.empty()) break;
    std::nth_element(t.begin(), t.begin() + t.size() / 2, t.end());
    ms_out[c] = t[t.size() / 2];
    if (ms_out[c] < best_ms) {
      best_ms = ms_out[c];
      best = cands[c];
    }
  }
  opt_.precision = saved_precision;
  long_warps_ = s == BV_OK ? best : saved_warps;
  staged_ = false;  // the sample was staged in FP64 mode
  destroy_graph();
  ++config_version_;
  *warps_out = long_warps_;
  return s;
}

}  // namespace bvphmm
