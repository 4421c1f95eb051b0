// phmm_engine.cpp -- host engine: validation, work planning, staging,
// launches, FP64 rescue, timing and graph replay.
//
// Work layout.  A result slot is one (read, haplotype) pair of one region,
// numbered region by region in read-major order, which is the layout of the
// [read][hap] matrix that AvxPairHMM::compute_likelihoods returns
// (include/biovoltron/algo/align/inexact_match/pairhmm_avx.hpp:160-171).
// A unit is one read scored against up to `haps_per_unit` consecutive
// haplotypes of its region, so the read's per-row constants and emission table
// are built once per unit.  Units are bucketed by kernel variant (rows per
// lane = ceil((read_len + 1) / 32), multi-strip above 256 rows); each bucket is
// one persistent launch whose warps pull units from a device work-queue head.
// The FP64 launch follows on the same stream and drains the list of pairs the
// FP32 launches flagged.
#include "phmm_engine.h"

#include "phmm_rows.h"

#include <algorithm>
#include <chrono>
#include <memory>
#include <cstring>
#include <string>

namespace bvphmm {

cudaError_t DevBuf::reserve(size_t bytes) {
  if (bytes <= cap_ && p_) return cudaSuccess;
  release();
  size_t want = std::max<size_t>(bytes, 256);
  cudaError_t e = cudaMalloc(&p_, want);
  if (e != cudaSuccess) {
    p_ = nullptr;
    cap_ = 0;
    return e;
  }
  cap_ = want;
  return cudaSuccess;
}

void DevBuf::release() {
  if (p_) cudaFree(p_);
  p_ = nullptr;
  cap_ = 0;
}

namespace {
constexpr int kMaxRowsPerLane = 8;
constexpr int kMaxVariants = 32;
constexpr int kRescaleTarget = 1000;  // FP64 boundary rows are scaled to ~2^1000

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

int hap_bytes_for(int max_hap, int chunk) {
  return (int)round_up((int64_t)max_hap + (kWarp - 1) + chunk + kHapLead + 16, 16);
}
long long bnd_cols_for(int max_hap) { return round_up((int64_t)max_hap + kWarp, 32) + 160; }
}  // namespace

Engine::Engine(const bv_phmm_options& opt) : opt_(opt) {
  // BV_MODE_BAND at creation: the band path with its default options (a fixed
  // band around the seed until MLP weights are trained or loaded).
  band_opt_.struct_size = (int32_t)sizeof(bv_band_options);
  band_opt_.enabled = opt.mode == BV_MODE_BAND;
  band_opt_.use_mlp = 0;
  band_opt_.fixed_half = 8;
  band_opt_.margin = 2;
  band_opt_.audit_period = 0;
  band_opt_.edge_threshold = 1e-3;
}

Engine::~Engine() {
  destroy_graph();
  if (stream_) {
    cudaStreamSynchronize(stream_);
    if (h_counters_) cudaFreeHost(h_counters_);
    if (h_chunk_off_) cudaFreeHost(h_chunk_off_);
    for (auto& e : ev_)
      if (e) cudaEventDestroy(e);
    for (auto& e : tune_ev_)
      if (e) cudaEventDestroy(e);
    cudaStreamDestroy(stream_);
  }
}

bv_status Engine::fail(bv_status s, const std::string& msg) {
  err_ = msg;
  return s;
}

bv_status Engine::status_fail(unsigned long long status) {
  // Kernel status bits: 1 FP64 list overflow, 2 invalid pair, 4 band list
  // overflow, 8 a boundary-row copy or strip hand-over wait gave up, 16 a
  // tensor-core completion wait gave up.
  static const char* const kNames[] = {"FP64 list overflow", "invalid pair", "band list overflow",
                                       "boundary wait gave up", "tensor-core wait gave up"};
  std::string msg = "kernel reported an inconsistent state (";
  bool first = true;
  for (int b = 0; b < 5; ++b) {
    if (!(status >> b & 1ull)) continue;
    msg += first ? "" : ", ";
    msg += kNames[b];
    first = false;
  }
  if (status >> 5) msg += std::string(first ? "" : ", ") + "status " + std::to_string(status);
  return fail(BV_ERR_INTERNAL, msg + ")");
}

bv_status Engine::cuda_fail(cudaError_t e, const char* what) {
  err_ = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return BV_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice) return BV_ERR_NO_DEVICE;
  return BV_ERR_CUDA;
}

#define BV_CUDA(call, what)                         \
  do {                                              \
    cudaError_t e__ = (call);                       \
    if (e__ != cudaSuccess) return cuda_fail(e__, what); \
  } while (0)

bv_status Engine::set_transitions(const double* trans) {
  if (trans) {
    for (int k = 0; k < 7; ++k)
      if (!(trans[k] >= 0.0 && trans[k] <= 1.0)) return fail(BV_ERR_INVALID_ARG, "transition outside [0, 1]");
    if (band_enabled()) return fail(BV_ERR_UNSUPPORTED, "constant transitions run the full-DP path: disable the band");
  }
  BV_CUDA(cudaSetDevice(opt_.device), "cudaSetDevice");
  BV_CUDA(cudaStreamSynchronize(stream_), "sync before table update");
  set_constant_transitions(h_tables_.get(), trans);
  BV_CUDA(cudaMemcpy(d_tables_.get(), h_tables_.get(), sizeof(Tables), cudaMemcpyHostToDevice), "tables copy");
  ++config_version_;
  staged_ = false;
  destroy_graph();
  return BV_OK;
}

bool Engine::constant_transitions(double* trans) const {
  if (!h_tables_ || !h_tables_->const_mode) return false;
  if (trans)
    for (int k = 0; k < 7; ++k) trans[k] = h_tables_->cd[k];
  return true;
}

bv_status Engine::init() {
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(BV_ERR_NO_DEVICE, "no CUDA device available");
  if (opt_.device < 0 || opt_.device >= ndev) return fail(BV_ERR_NO_DEVICE, "device ordinal out of range");
  BV_CUDA(cudaSetDevice(opt_.device), "cudaSetDevice");
  BV_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, opt_.device), "SM count");
  BV_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  for (auto& ev : ev_) BV_CUDA(cudaEventCreate(&ev), "event");
  h_tables_ = std::make_unique<Tables>();
  build_tables(h_tables_.get());
  BV_CUDA(d_tables_.reserve(sizeof(Tables)), "tables alloc");
  BV_CUDA(cudaMemcpyAsync(d_tables_.get(), h_tables_.get(), sizeof(Tables), cudaMemcpyHostToDevice, stream_),
          "tables copy");
  BV_CUDA(d_counters_.reserve(sizeof(Counters)), "counters alloc");
  BV_CUDA(cudaStreamSynchronize(stream_), "init sync");
  return BV_OK;
}

bv_status Engine::reserve_chunk_offsets(int64_t n) {
  if (n <= chunk_off_cap_) return BV_OK;
  if (h_chunk_off_) {
    BV_CUDA(cudaStreamSynchronize(stream_), "chunk offsets sync");
    cudaFreeHost(h_chunk_off_);
    h_chunk_off_ = nullptr;
    chunk_off_cap_ = 0;
  }
  BV_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_chunk_off_), sizeof(int64_t) * (size_t)n), "pinned chunk offsets");
  chunk_off_cap_ = n;
  return BV_OK;
}

bv_status Engine::validate(const bv_region_batch& b) { return validate_ranges(b, false); }
bv_status Engine::validate_outline(const bv_region_batch& b) { return validate_ranges(b, true); }

bv_status Engine::validate_ranges(const bv_region_batch& b, bool outline) {
  if (b.num_regions < 0 || b.num_reads < 0 || b.num_haps < 0) return fail(BV_ERR_INVALID_ARG, "negative count");
  if (b.num_regions > 0 && (!b.region_reads || !b.region_haps))
    return fail(BV_ERR_INVALID_ARG, "region offsets missing");
  if (b.num_reads > 0 && (!b.read_offsets)) return fail(BV_ERR_INVALID_ARG, "read offsets missing");
  if (b.num_haps > 0 && (!b.hap_offsets)) return fail(BV_ERR_INVALID_ARG, "hap offsets missing");
  if (b.num_reads >= INT32_MAX || b.num_haps >= INT32_MAX) return fail(BV_ERR_INVALID_ARG, "too many reads or haps");
  for (int64_t g = 0; g < b.num_regions; ++g) {
    if (b.region_reads[g] > b.region_reads[g + 1] || b.region_haps[g] > b.region_haps[g + 1])
      return fail(BV_ERR_INVALID_ARG, "region offsets decrease");
  }
  if (b.num_regions > 0) {
    if (b.region_reads[0] < 0 || b.region_haps[0] < 0 || b.region_reads[b.num_regions] > b.num_reads ||
        b.region_haps[b.num_regions] > b.num_haps)
      return fail(BV_ERR_INVALID_ARG, "region offsets out of range");
  }
  if (b.num_reads > 0) {
    if (b.read_offsets[0] < 0) return fail(BV_ERR_INVALID_ARG, "read offset negative");
    // outline: only the reads outside [region_reads[0], region_reads[num_regions])
    const int64_t skip0 = outline && b.num_regions > 0 ? b.region_reads[0] : b.num_reads;
    const int64_t skip1 = outline && b.num_regions > 0 ? b.region_reads[b.num_regions] : b.num_reads;
    for (int64_t r = 0; r < b.num_reads; ++r) {
      if (r == skip0 && skip1 > skip0) r = skip1;
      if (r >= b.num_reads) break;
      const int64_t l = b.read_offsets[r + 1] - b.read_offsets[r];
      if (l < 0) return fail(BV_ERR_INVALID_ARG, "read offsets decrease");
      if (l > BV_PHMM_MAX_READ_LEN) return fail(BV_ERR_INVALID_ARG, "read longer than BV_PHMM_MAX_READ_LEN");
    }
    const int n_gap_arrays = (b.read_i != nullptr) + (b.read_d != nullptr) + (b.read_c != nullptr);
    if (b.read_offsets[b.num_reads] > 0 && (!b.read_bases || !b.read_q || (n_gap_arrays != 0 && n_gap_arrays != 3)))
      return fail(BV_ERR_INVALID_ARG, "read arrays missing");
  }
  if (b.num_haps > 0) {
    if (b.hap_offsets[0] < 0) return fail(BV_ERR_INVALID_ARG, "hap offset negative");
    const int64_t skip0 = outline && b.num_regions > 0 ? b.region_haps[0] : b.num_haps;
    const int64_t skip1 = outline && b.num_regions > 0 ? b.region_haps[b.num_regions] : b.num_haps;
    for (int64_t h = 0; h < b.num_haps; ++h) {
      if (h == skip0 && skip1 > skip0) h = skip1;
      if (h >= b.num_haps) break;
      const int64_t l = b.hap_offsets[h + 1] - b.hap_offsets[h];
      if (l < 0) return fail(BV_ERR_INVALID_ARG, "hap offsets decrease");
      if (l > BV_PHMM_MAX_HAP_LEN) return fail(BV_ERR_INVALID_ARG, "haplotype longer than BV_PHMM_MAX_HAP_LEN");
    }
    if (b.hap_offsets[b.num_haps] > 0 && !b.hap_bases) return fail(BV_ERR_INVALID_ARG, "hap bases missing");
  }
  return BV_OK;
}

bv_status Engine::plan(const bv_region_batch& b) {
  units_.clear();
  f64_items_.clear();
  f64_long_items_.clear();
  plans_.clear();
  int64_t max_read = 0;
  n_results_ = 0;
  n_cells_ = 0;
  max_hap_ = 0;
  const int per_unit = std::max(1, opt_.haps_per_unit > 0 ? opt_.haps_per_unit : 8);
  const bool all_f64 = opt_.precision == BV_PRECISION_F64;
  const int v_multi = variant_index(false, 8, true);
  std::vector<int64_t> count(kMaxVariants, 0);
  std::vector<int> var_max_hap(kMaxVariants, 0);
  // pass 1: count units per variant
  std::vector<int> region_max_hap(std::max<int64_t>(b.num_regions, 1), 0);
  for (int64_t g = 0; g < b.num_regions; ++g) {
    int mh = 0;
    for (int64_t h = b.region_haps[g]; h < b.region_haps[g + 1]; ++h)
      mh = std::max<int>(mh, (int)(b.hap_offsets[h + 1] - b.hap_offsets[h]));
    region_max_hap[g] = mh;
    max_hap_ = std::max(max_hap_, mh);
  }
  // two haplotypes per warp (paired variants) unless the options or the bin's tuning ask for one
  auto pair_rows = [&](int64_t rt) {
    if (opt_.haps_per_warp == 1 || per_unit < 2 || rt < 1 || rt > kTuneBins) return false;
    return opt_.haps_per_warp == 2 || tune_[rt].haps_per_warp == 2;
  };
  auto variant_of = [&](int64_t rlen) {
    // rows of the single-strip FP32 kernel: row 0, the read, the summing row
    // and one padding row on top (phmm_device.cuh, rows_needed)
    const int64_t rows = rows_needed((int)std::min<int64_t>(rlen, 1 << 24), true, true);
    const int64_t rt = (rows + kWarp - 1) / kWarp;
    return rt <= kMaxRowsPerLane ? variant_index(false, (int)rt, false, pair_rows(rt)) : v_multi;
  };
  for (int64_t g = 0; g < b.num_regions; ++g) {
    const int64_t nh = b.region_haps[g + 1] - b.region_haps[g];
    const int64_t nr = b.region_reads[g + 1] - b.region_reads[g];
    if (nh == 0 || nr == 0) continue;
    const int64_t chunks = (nh + per_unit - 1) / per_unit;
    for (int64_t r = b.region_reads[g]; r < b.region_reads[g + 1]; ++r) {
      const int v = variant_of(b.read_offsets[r + 1] - b.read_offsets[r]);
      count[v] += chunks;
      var_max_hap[v] = std::max(var_max_hap[v], region_max_hap[g]);
    }
  }
  std::vector<int64_t> start(kMaxVariants + 1, 0);
  for (int v = 0; v < kMaxVariants; ++v) start[v + 1] = start[v] + count[v];
  if (!all_f64) units_.resize(start[kMaxVariants]);
  std::vector<int64_t> fill(start.begin(), start.end() - 1);
  // pass 2: fill units (or FP64 items) in result order within each bucket
  int64_t res = 0;
  for (int64_t g = 0; g < b.num_regions; ++g) {
    const int64_t h0 = b.region_haps[g], nh = b.region_haps[g + 1] - h0;
    const int64_t r0 = b.region_reads[g], nr = b.region_reads[g + 1] - r0;
    const int64_t hap_bases = nh > 0 ? b.hap_offsets[h0 + nh] - b.hap_offsets[h0] : 0;  // haplotypes are contiguous
    for (int64_t r = r0; r < r0 + nr; ++r) {
      const int64_t rl = b.read_offsets[r + 1] - b.read_offsets[r];
      n_cells_ += rl * hap_bases;
      max_read = std::max(max_read, rl);
      if (all_f64) {
        auto& list = rl >= long_rows() ? f64_long_items_ : f64_items_;
        for (int64_t k = 0; k < nh; ++k)
          list.push_back(PairRef{(int32_t)r, (int32_t)(h0 + k), res + (r - r0) * nh + k});
        continue;
      }
      const int v = variant_of(rl);
      for (int64_t k = 0; k < nh; k += per_unit) {
        Unit u{};
        u.read = (int32_t)r;
        u.hap0 = (int32_t)(h0 + k);
        u.nh = (int32_t)std::min<int64_t>(per_unit, nh - k);
        u.out0 = res + (r - r0) * nh + k;
        units_[fill[v]++] = u;
      }
    }
    res += nr * nh;
  }
  n_results_ = res;
  // launch plans
  int slot = 0;
  for (int v = 0; v < kMaxVariants && !all_f64; ++v) {
    if (count[v] == 0) continue;
    LaunchPlan lp;
    lp.variant = v;
    lp.slot = slot++;
    lp.unit_base = start[v];
    lp.n_units = count[v];
    lp.multi = (v == v_multi);
    lp.f64 = false;
    lp.code_row_bytes = hap_bytes_for(var_max_hap[v], lp.multi ? 32 : 8);
    // a paired variant stages one 32-bit entry (both haplotypes' table offsets) per column
    lp.hap_bytes = variant_paired(v) ? 4 * lp.code_row_bytes : lp.code_row_bytes;
    lp.warp_smem = warp_smem_bytes(v, lp.hap_bytes);
    {
      // the bin's block size (rows per lane of a single-strip FP32 variant)
      int rt = 0;
      for (int t = 1; t <= kTuneBins; ++t)
        if (v == variant_index(false, t, false, false) || v == variant_index(false, t, false, true)) rt = t;
      lp.warps_per_block = rt ? tune_[rt].warps_per_block : kThreadsPerBlock / kWarp;
    }
    const int smem_block = lp.warp_smem * lp.warps_per_block;
    if (lp.warp_smem * (kThreadsPerBlock / kWarp) > 227 * 1024)
      return fail(BV_ERR_INVALID_ARG, "haplotype too long for shared-memory staging");
    BV_CUDA(prepare_variant(v, lp.warp_smem * (kThreadsPerBlock / kWarp)), "kernel attribute");
    const int bps = std::max(1, blocks_per_sm(v, smem_block, lp.warps_per_block * kWarp));
    const int64_t need = (count[v] + lp.warps_per_block - 1) / lp.warps_per_block;
    lp.grid = (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)sms_ * bps));
    lp.bnd_cols = lp.multi ? bnd_cols_for(var_max_hap[v]) : 0;
    plans_.push_back(lp);
  }
  // FP64 launch: persistent over the whole device, whatever the FP32 passes flag
  LaunchPlan rp;
  rp.variant = variant_index(true, 4, true);
  rp.slot = 15;
  rp.multi = true;
  rp.f64 = true;
  rp.hap_bytes = hap_bytes_for(std::max(max_hap_, 1), 32);
  rp.warp_smem = warp_smem_bytes(rp.variant, rp.hap_bytes);
  const int smem_block = rp.warp_smem * (kThreadsPerBlock / kWarp);
  if (smem_block > 227 * 1024) return fail(BV_ERR_INVALID_ARG, "haplotype too long for shared-memory staging");
  BV_CUDA(prepare_variant(rp.variant, smem_block), "kernel attribute");
  const int bps = std::max(1, blocks_per_sm(rp.variant, smem_block));
  rp.grid = sms_ * bps;
  rp.bnd_cols = bnd_cols_for(std::max(max_hap_, 1));
  rescue_plan_ = rp;
  // FP64 long reads: one block per pair, longest pairs first (the long list is
  // read from its far end, so the host list is in ascending order of cells)
  long_plan_ = LaunchPlan{};
  if (max_read >= long_rows()) {
    long_smem_ = long_smem_bytes(rp.hap_bytes, long_warps_);
    if (long_smem_ <= 227 * 1024) {
      BV_CUDA(prepare_long(long_smem_, long_warps_), "kernel attribute");
      long_plan_.grid = sms_ * std::max(1, long_blocks_per_sm(long_smem_, long_warps_));
      long_plan_.hap_bytes = rp.hap_bytes;
      long_plan_.bnd_cols = rp.bnd_cols;
      long_plan_.f64 = true;
      long_plan_.multi = true;
    }
  }
  if (long_plan_.grid == 0) {  // no long kernel: the long reads stay on the one-warp FP64 kernel
    f64_items_.insert(f64_items_.end(), f64_long_items_.begin(), f64_long_items_.end());
    f64_long_items_.clear();
  }
  auto cells = [&](const PairRef& x) {
    return (b.read_offsets[x.read + 1] - b.read_offsets[x.read]) * (b.hap_offsets[x.hap + 1] - b.hap_offsets[x.hap]);
  };
  std::sort(f64_long_items_.begin(), f64_long_items_.end(),
            [&](const PairRef& x, const PairRef& y) { return cells(x) < cells(y); });
  return BV_OK;
}

// Inputs: the byte arrays and offsets go to the device as soon as the batch
// is validated, so the copies run while the host plans the launches.
bv_status Engine::upload_inputs(const bv_region_batch& b) {
  n_reads_ = b.num_reads;
  n_haps_ = b.num_haps;
  n_read_bytes_ = b.num_reads > 0 ? b.read_offsets[b.num_reads] : 0;
  n_hap_bytes_ = b.num_haps > 0 ? b.hap_offsets[b.num_haps] : 0;
  const size_t rb = (size_t)std::max<int64_t>(n_read_bytes_, 1);
  BV_CUDA(d_read_bases_.reserve(rb + 16), "alloc reads");  // tail padding for the k-mer kernel's word loads
  // uniform gap penalties: no per-base i, d, c arrays to copy (see bv_region_batch)
  uniform_gaps_ = !b.read_i && !b.read_d && !b.read_c;
  gap_ins_ = b.gap_ins;
  gap_del_ = b.gap_del;
  gap_gcp_ = b.gap_gcp;
  BV_CUDA(d_q_.reserve(rb), "alloc q");
  if (!uniform_gaps_) {
    BV_CUDA(d_i_.reserve(rb), "alloc i");
    BV_CUDA(d_d_.reserve(rb), "alloc d");
    BV_CUDA(d_c_.reserve(rb), "alloc c");
  }
  BV_CUDA(d_quals4_.reserve(rb * 4), "alloc quals");
  BV_CUDA(d_read_off_.reserve(sizeof(int64_t) * (n_reads_ + 1)), "alloc read offsets");
  BV_CUDA(d_hap_bases_.reserve((size_t)std::max<int64_t>(n_hap_bytes_, 1)), "alloc haps");
  BV_CUDA(d_hap_off_.reserve(sizeof(int64_t) * (n_haps_ + 1)), "alloc hap offsets");
  BV_CUDA(cudaEventRecord(ev_[0], stream_), "event");
  // Offsets are copied verbatim; the byte arrays are copied from index 0 so
  // offsets index them directly.
  if (n_read_bytes_ > 0) {
    BV_CUDA(cudaMemcpyAsync(d_read_bases_.get(), b.read_bases, n_read_bytes_, cudaMemcpyHostToDevice, stream_), "H2D");
    BV_CUDA(cudaMemcpyAsync(d_q_.get(), b.read_q, n_read_bytes_, cudaMemcpyHostToDevice, stream_), "H2D");
    if (!uniform_gaps_) {
      BV_CUDA(cudaMemcpyAsync(d_i_.get(), b.read_i, n_read_bytes_, cudaMemcpyHostToDevice, stream_), "H2D");
      BV_CUDA(cudaMemcpyAsync(d_d_.get(), b.read_d, n_read_bytes_, cudaMemcpyHostToDevice, stream_), "H2D");
      BV_CUDA(cudaMemcpyAsync(d_c_.get(), b.read_c, n_read_bytes_, cudaMemcpyHostToDevice, stream_), "H2D");
    }
  }
  if (n_reads_ > 0)
    BV_CUDA(cudaMemcpyAsync(d_read_off_.get(), b.read_offsets, sizeof(int64_t) * (n_reads_ + 1), cudaMemcpyHostToDevice,
                            stream_), "H2D");
  if (n_hap_bytes_ > 0)
    BV_CUDA(cudaMemcpyAsync(d_hap_bases_.get(), b.hap_bases, n_hap_bytes_, cudaMemcpyHostToDevice, stream_), "H2D");
  if (n_haps_ > 0)
    BV_CUDA(cudaMemcpyAsync(d_hap_off_.get(), b.hap_offsets, sizeof(int64_t) * (n_haps_ + 1), cudaMemcpyHostToDevice,
                            stream_), "H2D");
  return BV_OK;
}

// The plan's device side: work units, result and list buffers, and the packed
// qualities.  Nothing here waits for the copies; run() reads the copy time
// once its own synchronisation has passed.
bv_status Engine::upload_plan() {
  BV_CUDA(d_units_.reserve(sizeof(Unit) * std::max<size_t>(units_.size(), 1)), "alloc units");
  BV_CUDA(d_out_.reserve(sizeof(double) * (size_t)std::max<int64_t>(n_results_, 1)), "alloc results");
  BV_CUDA(d_rescue_.reserve(sizeof(PairRef) * (size_t)std::max<int64_t>(n_results_, 1)), "alloc rescue list");
  // strip-boundary buffers for the multi-strip launches
  size_t need32 = 0;
  for (const auto& lp : plans_)
    if (lp.multi) need32 = std::max<size_t>(need32, (size_t)lp.grid * lp.warps_per_block * (size_t)lp.bnd_cols * 4 * sizeof(float));
  if (need32) BV_CUDA(d_bnd32_.reserve(need32), "alloc boundary buffers");
  const size_t need64 = std::max((size_t)rescue_plan_.grid * (kThreadsPerBlock / kWarp) * (size_t)rescue_plan_.bnd_cols,
                                 (size_t)long_plan_.grid * (size_t)long_plan_.bnd_cols) * 4 * sizeof(double);
  BV_CUDA(d_bnd64_.reserve(need64), "alloc FP64 boundary buffers");
  if (!units_.empty())
    BV_CUDA(cudaMemcpyAsync(d_units_.get(), units_.data(), sizeof(Unit) * units_.size(), cudaMemcpyHostToDevice,
                            stream_), "H2D");
  if (!f64_items_.empty())
    BV_CUDA(cudaMemcpyAsync(d_rescue_.get(), f64_items_.data(), sizeof(PairRef) * f64_items_.size(),
                            cudaMemcpyHostToDevice, stream_), "H2D");
  if (!f64_long_items_.empty())  // at the list's far end
    BV_CUDA(cudaMemcpyAsync(d_rescue_.as<PairRef>() + (std::max<int64_t>(n_results_, 1) - (int64_t)f64_long_items_.size()),
                            f64_long_items_.data(), sizeof(PairRef) * f64_long_items_.size(), cudaMemcpyHostToDevice,
                            stream_), "H2D");
  if (uniform_gaps_)
    BV_CUDA(launch_pack_quals_uniform(d_q_.as<uint8_t>(), gap_ins_, gap_del_, gap_gcp_, d_quals4_.as<uchar4>(),
                                      n_read_bytes_, sms_, stream_), "pack quals");
  else
    BV_CUDA(launch_pack_quals(d_q_.as<uint8_t>(), d_i_.as<uint8_t>(), d_d_.as<uint8_t>(), d_c_.as<uint8_t>(),
                              d_quals4_.as<uchar4>(), n_read_bytes_, sms_, stream_), "pack quals");
  BV_CUDA(cudaEventRecord(ev_[1], stream_), "event");
  h2d_time_pending_ = true;
  return BV_OK;
}

// The caller's host arrays are borrowed for the call: unless the caller runs
// the batch before returning (compute, whose run synchronises), stage waits
// for the copies, and every error path after the first copy waits for them too.
bv_status Engine::stage(const bv_region_batch& b, bool wait) {
  staged_ = false;
  destroy_graph();
  BV_CUDA(cudaSetDevice(opt_.device), "cudaSetDevice");
  bv_status s = validate(b);
  if (s != BV_OK) return s;
  s = upload_inputs(b);
  if (s == BV_OK) s = plan(b);
  if (s == BV_OK) s = upload_plan();
  if (s == BV_OK && band_enabled()) s = band_prepare();
  if (s != BV_OK) {
    cudaStreamSynchronize(stream_);
    return s;
  }
  if (wait) BV_CUDA(cudaStreamSynchronize(stream_), "stage sync");
  staged_ = true;
  runs_since_stage_ = 0;
  return BV_OK;
}

bv_status Engine::enqueue_kernels(bool capturing) {
  // Inside stream capture, timing events become event-record nodes of the
  // graph only when recorded as external events.
  auto rec = [&](cudaEvent_t ev) {
    return capturing ? cudaEventRecordWithFlags(ev, stream_, cudaEventRecordExternal) : cudaEventRecord(ev, stream_);
  };
  BV_CUDA(cudaMemsetAsync(d_counters_.get(), 0, sizeof(Counters), stream_), "memset counters");
  if (!f64_items_.empty()) {
    BV_CUDA(launch_set_u64(&d_counters_.as<Counters>()->rescue_count, (unsigned long long)f64_items_.size(), stream_),
            "set FP64 count");
  }
  if (!f64_long_items_.empty()) {
    BV_CUDA(launch_set_u64(&d_counters_.as<Counters>()->rescue_long_count, (unsigned long long)f64_long_items_.size(),
                           stream_), "set FP64 count");
  }
  KernelParams p{};
  p.batch.read_bases = d_read_bases_.as<uint8_t>();
  p.batch.read_quals = d_quals4_.as<uchar4>();
  p.batch.read_off = d_read_off_.as<int64_t>();
  p.batch.hap_bases = d_hap_bases_.as<uint8_t>();
  p.batch.hap_off = d_hap_off_.as<int64_t>();
  p.tables = d_tables_.as<Tables>();
  p.units = d_units_.as<Unit>();
  p.ctr = d_counters_.as<Counters>();
  p.out = d_out_.as<double>();
  p.rescue = d_rescue_.as<PairRef>();
  p.rescue_cap = std::max<int64_t>(n_results_, 1);
  p.long_rows = long_plan_.grid > 0 ? long_rows() : 0;
  p.warps_per_block = kThreadsPerBlock / kWarp;  // band-path fallback and audit launches
  BV_CUDA(rec(ev_[2]), "event");
  if (band_enabled()) {
    bv_status bs = enqueue_band(capturing, p);
    if (bs != BV_OK) return bs;
  }
  if (tune_timing_ && !capturing) {
    while (tune_ev_.size() < 2 * plans_.size()) {
      cudaEvent_t e;
      BV_CUDA(cudaEventCreate(&e), "event");
      tune_ev_.push_back(e);
    }
  }
  for (size_t pi = 0; pi < plans_.size(); ++pi) {
    const LaunchPlan& lp = plans_[pi];
    if (band_enabled()) break;
    const bool timed = tune_timing_ && !capturing;
    if (timed) BV_CUDA(cudaEventRecord(tune_ev_[2 * pi], stream_), "event");
    p.unit_base = lp.unit_base;
    p.n_units = lp.n_units;
    p.slot = lp.slot;
    p.from_rescue = 0;
    p.hap_bytes = lp.hap_bytes;
    p.code_row_bytes = lp.code_row_bytes;
    p.warps_per_block = lp.warps_per_block;
    p.warp_smem_bytes = lp.warp_smem;
    p.bnd = lp.multi ? d_bnd32_.get() : nullptr;
    p.bnd_cols = lp.bnd_cols;
    p.rescale = 0;
    p.rescale_target = 0;
    BV_CUDA(launch_forward(lp.variant, p, lp.grid, stream_), "FP32 forward launch");
    if (timed) BV_CUDA(cudaEventRecord(tune_ev_[2 * pi + 1], stream_), "event");
  }
  BV_CUDA(rec(ev_[3]), "event");
  {
    const LaunchPlan& lp = rescue_plan_;
    p.unit_base = 0;
    p.n_units = 0;
    p.slot = lp.slot;
    p.from_rescue = 1;
    p.hap_bytes = lp.hap_bytes;
    p.code_row_bytes = 0;
    p.warps_per_block = kThreadsPerBlock / kWarp;
    p.warp_smem_bytes = lp.warp_smem;
    p.bnd = d_bnd64_.get();
    p.bnd_cols = lp.bnd_cols;
    p.rescale = 1;
    p.rescale_target = kRescaleTarget;
    p.cells_ctr = &d_counters_.as<Counters>()->rescued_cells;
    if (long_plan_.grid > 0) {  // long reads first: a block per pair, longest first
      KernelParams q = p;
      q.hap_bytes = long_plan_.hap_bytes;
      q.bnd_cols = long_plan_.bnd_cols;
      BV_CUDA(launch_forward_long(q, long_plan_.grid, long_smem_, long_warps_, stream_), "FP64 long-read launch");
    }
    BV_CUDA(launch_forward(lp.variant, p, lp.grid, stream_), "FP64 forward launch");
    p.cells_ctr = nullptr;
  }
  BV_CUDA(rec(ev_[4]), "event");
  if (band_enabled() && band_opt_.audit_period > 0) {
    BV_CUDA(launch_audit_compare(band_params(), d_audit_err_.as<double>(), stream_), "audit compare");
  }
  return BV_OK;
}

void Engine::destroy_graph() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (graph_) cudaGraphDestroy(graph_);
  graph_exec_ = nullptr;
  graph_ = nullptr;
}

bv_status Engine::run(bv_phmm_stats* stats) {
  bv_status s = launch();
  if (s != BV_OK) return s;
  return finish(stats);
}

bv_status Engine::launch() {
  if (!staged_) return fail(BV_ERR_INVALID_ARG, "no staged batch");
  BV_CUDA(cudaSetDevice(opt_.device), "cudaSetDevice");
  run_t0_ = std::chrono::steady_clock::now();
  if (!h_counters_) BV_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_counters_), sizeof(Counters)), "pinned counters");
  // The first run of a staged batch launches directly; later runs replay a
  // captured graph of the same launch sequence.
  if (runs_since_stage_ == 0 || !graph_exec_) {
    if (runs_since_stage_ >= 1 && !graph_exec_) {
      BV_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
      bv_status s = enqueue_kernels(true);
      cudaGraph_t g = nullptr;
      cudaError_t ce = cudaStreamEndCapture(stream_, &g);
      if (s != BV_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
      }
      BV_CUDA(ce, "end capture");
      graph_ = g;
      BV_CUDA(cudaGraphInstantiate(&graph_exec_, graph_, 0), "graph instantiate");
      BV_CUDA(cudaGraphLaunch(graph_exec_, stream_), "graph launch");
    } else {
      bv_status s = enqueue_kernels(false);
      if (s != BV_OK) return s;
    }
  } else {
    BV_CUDA(cudaGraphLaunch(graph_exec_, stream_), "graph launch");
  }
  ++runs_since_stage_;
  // page-locked destination: the copy is queued, the host goes on
  BV_CUDA(cudaMemcpyAsync(h_counters_, d_counters_.get(), sizeof(Counters), cudaMemcpyDeviceToHost, stream_),
          "counters D2H");
  return BV_OK;
}

bv_status Engine::finish(bv_phmm_stats* stats) {
  BV_CUDA(cudaStreamSynchronize(stream_), "run sync");
  if (h2d_time_pending_) {
    BV_CUDA(cudaEventElapsedTime(&ms_h2d_, ev_[0], ev_[1]), "event time");
    h2d_time_pending_ = false;
  }
  const Counters c = *h_counters_;
  if (c.status != 0) return status_fail(c.status);
  if (stats) *stats = bv_phmm_stats{};
  if (stats && band_enabled()) {
    bv_status bs = band_stats(stats);
    if (bs != BV_OK) return bs;
  }
  if (stats) {
    float ms32 = 0, ms64 = 0;
    cudaEventElapsedTime(&ms32, ev_[2], ev_[3]);
    cudaEventElapsedTime(&ms64, ev_[3], ev_[4]);
    stats->pairs = n_results_;
    stats->cells = n_cells_;
    stats->rescued = (int64_t)(c.rescue_count + c.rescue_long_count);
    stats->rescued_cells = (int64_t)c.rescued_cells;
    stats->fp32_skipped_cells = (int64_t)c.fp32_skipped_cells;
    stats->underflow = (int64_t)c.underflow_count;
    // band mode: k-mer tables, nibble image, read k-mers, gap check, two featurisers, MLP, route,
    // scan, route; the banded kernels; the fallback variants; the rescore check and variants;
    // the audit; the FP64 pass
    stats->kernel_launches = band_enabled()
                                 ? 9 + (band_opt_.use_mlp ? 1 : 0) + kBandWidths + 9 + (band_opt_.cap_margin > 0 ? 10 : 0) +
                                       (band_opt_.audit_period > 0 ? 11 : 0) + 1
                                 : (int64_t)plans_.size() + 1;
    stats->ms_fp32 = ms32;
    stats->ms_fp64 = ms64;
    if (band_enabled()) {
      float seed = 0, band = 0, full = 0;
      cudaEventElapsedTime(&seed, ev_[2], ev_[5]);
      cudaEventElapsedTime(&band, ev_[5], ev_[6]);
      cudaEventElapsedTime(&full, ev_[6], ev_[3]);
      stats->ms_seed = seed;
      stats->ms_band = band;
      stats->ms_full = full;
    } else {
      stats->ms_full = ms32;
    }
    stats->ms_h2d = ms_h2d_;
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - run_t0_).count();
  }
  return BV_OK;
}

bv_status Engine::fetch(double* out, int64_t n) {
  if (!staged_) return fail(BV_ERR_INVALID_ARG, "no staged batch");
  if (n < 0 || n > n_results_) return fail(BV_ERR_INVALID_ARG, "fetch size exceeds staged results");
  if (n == 0) return BV_OK;
  if (!out) return fail(BV_ERR_INVALID_ARG, "null output");
  BV_CUDA(cudaMemcpyAsync(out, d_out_.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, stream_), "results D2H");
  BV_CUDA(cudaStreamSynchronize(stream_), "fetch sync");
  return BV_OK;
}

bv_status Engine::fetch_async(double* out, int64_t n) {
  if (!staged_) return fail(BV_ERR_INVALID_ARG, "no staged batch");
  if (n < 0 || n > n_results_) return fail(BV_ERR_INVALID_ARG, "fetch size exceeds staged results");
  if (n == 0) return BV_OK;
  if (!out) return fail(BV_ERR_INVALID_ARG, "null output");
  BV_CUDA(cudaMemcpyAsync(out, d_out_.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, stream_), "results D2H");
  return BV_OK;
}

bv_status Engine::compute(const bv_region_batch& b, double* out, bv_phmm_stats* stats) {
  const auto t0 = std::chrono::steady_clock::now();
  if (!out && b.num_regions > 0) {
    // checked before any copy starts (a batch with results needs an output)
    bv_status v = validate(b);
    if (v != BV_OK) return v;
    int64_t res = 0;
    for (int64_t g = 0; g < b.num_regions; ++g)
      res += (b.region_reads[g + 1] - b.region_reads[g]) * (b.region_haps[g + 1] - b.region_haps[g]);
    if (res > 0) return fail(BV_ERR_INVALID_ARG, "null output");
  }
  bv_status s = stage(b, false);  // run() synchronises before this call returns
  if (s != BV_OK) return s;
  s = run(stats);
  if (s != BV_OK) {
    cudaStreamSynchronize(stream_);  // no copy from the caller's arrays outlives the call
    return s;
  }
  const auto t1 = std::chrono::steady_clock::now();
  s = fetch(out, n_results_);
  if (s != BV_OK) return s;
  if (stats) {
    const auto t2 = std::chrono::steady_clock::now();
    stats->ms_d2h = std::chrono::duration<double, std::milli>(t2 - t1).count();
    stats->ms_total = std::chrono::duration<double, std::milli>(t2 - t0).count();
  }
  return BV_OK;
}

}  // namespace bvphmm
