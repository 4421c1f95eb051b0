// phmm_engine.h -- host engine behind the C ABI (C++20).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <chrono>
#include <memory>
#include <vector>

#include "bv_pairhmm.h"
#include "phmm_band.h"
#include "phmm_common.h"
#include "phmm_kernels.h"

namespace bvphmm {

// Grow-only device allocation.
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  cudaError_t reserve(size_t bytes);
  void release();
  void* get() const { return p_; }
  template <typename T> T* as() const { return static_cast<T*>(p_); }
  size_t capacity() const { return cap_; }

 private:
  void* p_ = nullptr;
  size_t cap_ = 0;
};

// Launch parameters of one rows-per-lane bin (single-strip FP32 full DP),
// chosen by the autotuner or set by the caller.
struct BinTune {
  int haps_per_warp = 2;    // 1: one haplotype per warp; 2: two (packed FP32x2)
  int warps_per_block = 4;  // 1..4
};
constexpr int kTuneBins = 8;  // rows per lane 1..8

struct LaunchPlan {
  int variant = -1;
  int slot = 0;
  long long unit_base = 0;
  long long n_units = 0;
  int warps_per_block = kThreadsPerBlock / kWarp;
  int hap_bytes = 0;
  int code_row_bytes = 0;
  int warp_smem = 0;
  int grid = 0;
  long long bnd_cols = 0;
  bool multi = false;
  bool f64 = false;
};

// A chunk of regions [g0, g1) of a batch and its result slots [out0, out0 + n_out).
struct ChunkCut {
  int64_t g0, g1, out0, n_out;
};
// Cuts a batch's regions into consecutive chunks of about total / chunks
// pairs each (a chunk ends at the region that reaches the target; the last
// chunk takes the rest).
std::vector<ChunkCut> plan_chunks(const bv_region_batch& b, int chunks);

// A chunk of regions [g0, g1) as a batch of its own: offsets rebased to the
// chunk's first read / haplotype, byte pointers moved to match.  The rebased
// read and haplotype offsets go to `off` (page-locked memory of the context
// that stages the chunk, at least n_off() entries) so that their copies to the
// device do not hold up the host.
struct Chunk {
  int64_t g0 = 0, g1 = 0, out0 = 0, n_out = 0;
  std::vector<int64_t> region_reads, region_haps;
  bv_region_batch view{};

  int64_t n_off(const bv_region_batch& b) const {
    return (b.region_reads[g1] - b.region_reads[g0] + 1) + (b.region_haps[g1] - b.region_haps[g0] + 1);
  }
  void build(const bv_region_batch& b, int64_t* off) {
    const int64_t r0 = b.region_reads[g0], r1 = b.region_reads[g1];
    const int64_t h0 = b.region_haps[g0], h1 = b.region_haps[g1];
    region_reads.resize(g1 - g0 + 1);
    region_haps.resize(g1 - g0 + 1);
    for (int64_t g = g0; g <= g1; ++g) {
      region_reads[g - g0] = b.region_reads[g] - r0;
      region_haps[g - g0] = b.region_haps[g] - h0;
    }
    int64_t* read_off = off;
    int64_t* hap_off = off + (r1 - r0 + 1);
    const int64_t rb0 = r1 > r0 ? b.read_offsets[r0] : 0;
    for (int64_t r = r0; r <= r1 && r1 > r0; ++r) read_off[r - r0] = b.read_offsets[r] - rb0;
    if (r1 == r0) read_off[0] = 0;
    const int64_t hb0 = h1 > h0 ? b.hap_offsets[h0] : 0;
    for (int64_t h = h0; h <= h1 && h1 > h0; ++h) hap_off[h - h0] = b.hap_offsets[h] - hb0;
    if (h1 == h0) hap_off[0] = 0;
    view = b;
    view.num_regions = g1 - g0;
    view.region_reads = region_reads.data();
    view.region_haps = region_haps.data();
    view.num_reads = r1 - r0;
    view.read_offsets = read_off;
    view.num_haps = h1 - h0;
    view.hap_offsets = hap_off;
    auto shift = [](const uint8_t* p, int64_t o) { return p ? p + o : p; };
    view.read_bases = shift(b.read_bases, rb0);
    view.read_q = shift(b.read_q, rb0);
    view.read_i = shift(b.read_i, rb0);
    view.read_d = shift(b.read_d, rb0);
    view.read_c = shift(b.read_c, rb0);
    view.hap_bases = shift(b.hap_bases, hb0);
  }
};

// Adds a call's statistics into a running total (chunks, contexts).
void add_stats(bv_phmm_stats& t, const bv_phmm_stats& s);

// Regions split over n_parts devices: contiguous blocks of about equal DP
// cells (block b = regions [block_start[b], block_start[b+1]), its results at
// block_out0[b]), dealt by greedy LPT on the blocks' cells (block_part[b]).
struct Partition {
  std::vector<int64_t> block_start, block_cells, block_out0, block_pairs, part_cells;
  std::vector<int> block_part;
};
Partition plan_partition(const bv_region_batch& b, int n_parts, int n_blocks);


class Engine {
 public:
  explicit Engine(const bv_phmm_options& opt);
  ~Engine();
  bv_status init();

  bv_status stage(const bv_region_batch& b, bool wait = true);
  bv_status run(bv_phmm_stats* stats);  // launch + finish
  bv_status launch();                    // queue one run of the staged batch; does not wait
  bv_status finish(bv_phmm_stats* stats);  // wait for the queued run, check it, fill stats
  bv_status fetch(double* out, int64_t n);
  bv_status fetch_async(double* out, int64_t n);  // queued behind the run; finish() or a sync waits for it
  const bv_phmm_options& options() const { return opt_; }
  const bv_band_options& band_options() const { return band_opt_; }
  bool mlp_ready() const { return mlp_ready_; }
  uint64_t config_version() const { return config_version_; }
  // Copies band options, MLP weights and launch shapes from `src` (a context
  // with the same options); the chunked compute keeps its second context in step.
  bv_status mirror_config(Engine& src);
  // Constant transitions for every row (the scalar PairHMM model; 7 entries in
  // PairHMM::TrasMatrx order), or the quality-derived ones again (nullptr).
  bv_status set_transitions(const double* trans);
  bool constant_transitions(double* trans) const;
  bv_status genotype_staged(const bv_region_batch& b, const bv_genotype_batch& g, int32_t* kept_count,
                            int32_t* kept_reads, double* allele_lik, double* genotype_lik, double* kernel_ms);
  uint64_t mirrored_version() const { return mirrored_version_; }
  // One batch split into `chunks` region chunks that alternate between this
  // context and `other`: a chunk's copies and the host's planning overlap the
  // previous chunk's kernels.  Results and stats as compute().
  bv_status compute_chunked(Engine& other, const bv_region_batch& b, double* out, bv_phmm_stats* stats, int chunks);
  bv_status compute(const bv_region_batch& b, double* out, bv_phmm_stats* stats);

  const char* last_error() const { return err_.c_str(); }
  bv_status fail(bv_status s, const std::string& msg);
  // BV_ERR_INTERNAL naming the kernel status bits that were set.
  bv_status status_fail(unsigned long long status);
  bv_status cuda_fail(cudaError_t e, const char* what);
  int64_t staged_results() const { return n_results_; }
  cudaStream_t stream() const { return stream_; }
  int device() const { return opt_.device; }
  bv_status set_band_options(const bv_band_options& o);
  bool band_enabled() const { return band_opt_.enabled != 0; }
  bv_status band_train(const bv_region_batch& b, const bv_band_train_options& o, bv_band_train_report* rep);
  bv_status band_labels(const bv_region_batch& b, float tau, int32_t* dstar, int32_t* lo, int32_t* hi, float* feat,
                        int32_t* kmin, int32_t* kmax);
  bv_status band_routes(int64_t n, int32_t* d_lo, int32_t* width, int32_t* route);
  bv_status band_get_weights(float* w, int64_t n);
  bv_status band_set_weights(const float* w, int64_t n);
  bv_status band_save(const char* path);
  bv_status band_load(const char* path);
  bv_status band_mlp_eval(const float* w, const float* x, const float* t, int64_t n, float alpha, float* out,
                          float* loss, float* grad);
  // The inference kernel on [n][80] features (rounded to BF16) with the
  // installed weights: outputs [n][2].
  bv_status band_mlp_infer(const float* x, int64_t n, float* out);
  bv_status autotune(const bv_region_batch& sample, int repeats, bv_phmm_tune_entry* out, int32_t* n_out);
  bv_status set_tuning(const bv_phmm_tune_entry* entries, int32_t n);
  bv_status get_tuning(bv_phmm_tune_entry* out, int32_t* n_out);
  // Warps per pair of the FP64 long-read kernel (2, 4 or 8; reads of at least
  // 128 x warps bases take it), set directly or chosen by timing the FP64 pass
  // of a sample for each (ms[0..2]: 2, 4, 8 warps; 0 where not timed).
  bv_status set_long_warps(int warps);
  int long_warps() const { return long_warps_; }
  bv_status autotune_long(const bv_region_batch& sample, int repeats, int32_t* warps_out, double* ms_out);

 private:
  bv_status validate(const bv_region_batch& b);
  // validate() but for the reads and haplotypes inside the regions' ranges,
  // which the chunked call's chunks validate as they are staged
  bv_status validate_outline(const bv_region_batch& b);
  bv_status validate_ranges(const bv_region_batch& b, bool outline);
  // page-locked room for n rebased offsets of a chunk this context stages
  bv_status reserve_chunk_offsets(int64_t n);
  int64_t* chunk_offsets() const { return h_chunk_off_; }
  bv_status plan(const bv_region_batch& b);
  bv_status upload_inputs(const bv_region_batch& b);
  bv_status upload_plan();
  bv_status enqueue_kernels(bool capturing);
  bv_status band_prepare();
  bv_status enqueue_band(bool capturing, KernelParams& p);
  bv_status band_stats(bv_phmm_stats* stats);
  void destroy_graph();

  bv_phmm_options opt_;
  int sms_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev_[8] = {};
  std::string err_;

  std::unique_ptr<Tables> h_tables_;  // host copy of d_tables_
  DevBuf d_jacobian_, d_gt_regions_, d_gt_offsets_, d_gt_alleles_, d_gt_hap_allele_, d_gt_overlap_;
  DevBuf d_gt_kept_count_, d_gt_kept_reads_, d_gt_allele_lik_, d_gt_geno_lik_;
  bool jacobian_ready_ = false;
  DevBuf d_tables_, d_read_bases_, d_q_, d_i_, d_d_, d_c_, d_quals4_, d_read_off_, d_hap_bases_, d_hap_off_;
  DevBuf d_units_, d_out_, d_rescue_, d_counters_, d_bnd32_, d_bnd64_, d_f64_items_;

  // staged batch
  std::vector<Unit> units_;
  std::vector<PairRef> f64_items_;  // pairs sent straight to FP64 (precision F64)
  std::vector<PairRef> f64_long_items_;  // the long reads among them, ascending cells (the list's far end first)
  std::vector<LaunchPlan> plans_;
  LaunchPlan rescue_plan_;
  LaunchPlan long_plan_;  // FP64 long reads, a block of long_warps_ warps per pair (grid 0: none)
  int long_warps_ = kLongWarps;  // 2, 4 or 8; reads of at least long_rows() bases take the long kernel
  int long_rows() const { return long_warps_ * 128; }
  int long_smem_ = 0;
  int64_t n_results_ = 0;
  int64_t n_cells_ = 0;
  int64_t n_read_bytes_ = 0;
  bool uniform_gaps_ = false;  // the staged batch gave no per-base i, d, c arrays
  uint8_t gap_ins_ = 0, gap_del_ = 0, gap_gcp_ = 0;
  int64_t n_hap_bytes_ = 0;
  int64_t n_reads_ = 0;
  int64_t n_haps_ = 0;
  int max_hap_ = 0;
  bool staged_ = false;
  float ms_h2d_ = 0;
  bool h2d_time_pending_ = false;  // ms_h2d_ is read after the next synchronisation
  Counters* h_counters_ = nullptr;  // page-locked copy of the device counters
  int64_t* h_chunk_off_ = nullptr;  // page-locked rebased offsets of the chunk this context stages
  int64_t chunk_off_cap_ = 0;
  std::chrono::steady_clock::time_point run_t0_{};
  uint64_t config_version_ = 0;     // bumped by every change a second context must mirror
  uint64_t mirrored_version_ = ~0ull;  // the source's config_version_ this context last mirrored

  // learned band
  bv_band_options band_opt_{};
  bool mlp_ready_ = false;
  DevBuf d_pair_read_, d_pair_hap_, d_hap_table_, d_dstar_, d_feat_, d_mlp_out_, d_mlp_, d_bctr_;
  DevBuf d_kmin_, d_kmax_, d_read_kmers_, d_feat_hist_, d_feat_slow_, d_hap_nib_, d_banded_, d_cap_items_;
  DevBuf d_band_items_, d_full_items_, d_audit_pairs_, d_audit_units_, d_audit_out_, d_audit_err_;
  long long item_cap_ = 0, full_cap_ = 0, audit_cap_ = 0;
  LaunchPlan full_plans_[9];
  BandParams band_params() const;
  // training
  bv_status stage_for_labels(const bv_region_batch& b);
  bv_status compute_labels(const bv_region_batch& b, float tau, float* ms);
  bv_status install_weights(const float* w_host);
  std::vector<float> mlp_w_;  // FP32 master weights of the installed MLP
  DevBuf d_lab_lo_, d_lab_hi_, d_lab_fbuf_, d_mlp_w_;

  // per-bin launch parameters; per-launch timing while tuning
  BinTune tune_[kTuneBins + 1];
  bool tune_timing_ = false;
  std::vector<cudaEvent_t> tune_ev_;

  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  int runs_since_stage_ = 0;
};

}  // namespace bvphmm
