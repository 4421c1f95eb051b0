// phmm_capi.cpp -- extern "C" entry points declared in include/bv_pairhmm.h.
//
// Nothing crosses the C boundary as an exception: every entry point catches
// and maps failures to a bv_status.
#include <algorithm>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "bv_pairhmm.h"
#include "phmm_engine.h"
#include "phmm_mlp.h"
#include "phmm_genotype.h"

struct bv_phmm_ctx {
  bvphmm::Engine engine;
  std::unique_ptr<bvphmm::Engine> second;  // the chunked compute's other context, made on first use
  explicit bv_phmm_ctx(const bv_phmm_options& o) : engine(o) {}
};

namespace {

// Flattens testcases into one region per run of consecutive testcases that
// share a read, which is how AvxPairHMM::getData lays them out
// ([read][hap], pairhmm_avx.hpp:57-79).
struct Flat {
  std::vector<int64_t> region_reads{0}, region_haps{0}, read_off{0}, hap_off{0};
  std::vector<uint8_t> rb, rq, ri, rd, rc, hb;
  std::vector<int64_t> slot_of;  // testcase k -> result slot
  bv_region_batch view() const {
    bv_region_batch b{};
    b.num_regions = (int64_t)region_reads.size() - 1;
    b.region_reads = region_reads.data();
    b.region_haps = region_haps.data();
    b.num_reads = (int64_t)read_off.size() - 1;
    b.read_offsets = read_off.data();
    b.read_bases = rb.data();
    b.read_q = rq.data();
    b.read_i = ri.data();
    b.read_d = rd.data();
    b.read_c = rc.data();
    b.num_haps = (int64_t)hap_off.size() - 1;
    b.hap_offsets = hap_off.data();
    b.hap_bases = hb.data();
    return b;
  }
  void add_read(int len, const char* s, const char* q, const char* i, const char* d, const char* c) {
    rb.insert(rb.end(), s, s + len);
    rq.insert(rq.end(), q, q + len);
    ri.insert(ri.end(), i, i + len);
    rd.insert(rd.end(), d, d + len);
    rc.insert(rc.end(), c, c + len);
    read_off.push_back((int64_t)rb.size());
  }
  void add_hap(int len, const char* s) {
    hb.insert(hb.end(), s, s + len);
    hap_off.push_back((int64_t)hb.size());
  }
};

bv_status guard(bv_phmm_ctx* ctx, auto&& fn) {
  try {
    return fn();
  } catch (const std::bad_alloc&) {
    if (ctx) ctx->engine.fail(BV_ERR_OOM, "host allocation failed");
    return BV_ERR_OOM;
  } catch (...) {
    if (ctx) ctx->engine.fail(BV_ERR_INTERNAL, "unexpected exception");
    return BV_ERR_INTERNAL;
  }
}

}  // namespace

extern "C" {

void bv_phmm_default_options(bv_phmm_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->struct_size = (int32_t)sizeof(*o);
  o->device = 0;
  o->precision = BV_PRECISION_AUTO;
  o->mode = BV_MODE_FULL;
  o->rescue_threshold = bvphmm::kMinAccepted;
  o->haps_per_unit = 8;
}

int bv_phmm_abi_version(void) { return BV_PHMM_ABI_VERSION; }

const char* bv_phmm_status_string(bv_status s) {
  switch (s) {
    case BV_OK: return "ok";
    case BV_ERR_INVALID_ARG: return "invalid argument";
    case BV_ERR_OOM: return "out of memory";
    case BV_ERR_CUDA: return "CUDA error";
    case BV_ERR_TIMEOUT: return "timeout";
    case BV_ERR_NO_DEVICE: return "no CUDA device";
    case BV_ERR_INTERNAL: return "internal error";
    case BV_ERR_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

bv_status bv_phmm_create(const bv_phmm_options* opts, bv_phmm_ctx** out) {
  if (!out) return BV_ERR_INVALID_ARG;
  *out = nullptr;
  bv_phmm_options o;
  bv_phmm_default_options(&o);
  if (opts) {
    if (opts->struct_size != (int32_t)sizeof(bv_phmm_options)) return BV_ERR_INVALID_ARG;
    o = *opts;
  }
  if (o.precision != BV_PRECISION_AUTO && o.precision != BV_PRECISION_F64) return BV_ERR_INVALID_ARG;
  if (o.mode != BV_MODE_FULL && o.mode != BV_MODE_BAND) return BV_ERR_INVALID_ARG;
  if (o.rescue_threshold != bvphmm::kMinAccepted) return BV_ERR_UNSUPPORTED;
  if (o.haps_per_warp < 0 || o.haps_per_warp > 2) return BV_ERR_INVALID_ARG;
  if (o.pipeline_chunks < 0 || o.pipeline_chunks > 64 || o.pipeline_min_pairs < 0) return BV_ERR_INVALID_ARG;
  bv_phmm_ctx* c = new (std::nothrow) bv_phmm_ctx(o);
  if (!c) return BV_ERR_OOM;
  bv_status s = guard(c, [&] { return c->engine.init(); });
  if (s != BV_OK) {
    delete c;
    return s;
  }
  *out = c;
  return BV_OK;
}

void bv_phmm_destroy(bv_phmm_ctx* ctx) { delete ctx; }

const char* bv_phmm_last_error(const bv_phmm_ctx* ctx) { return ctx ? ctx->engine.last_error() : "null context"; }

int64_t bv_phmm_region_results(const bv_region_batch* b) {
  if (!b || b->num_regions <= 0 || !b->region_reads || !b->region_haps) return 0;
  int64_t n = 0;
  for (int64_t g = 0; g < b->num_regions; ++g)
    n += (b->region_reads[g + 1] - b->region_reads[g]) * (b->region_haps[g + 1] - b->region_haps[g]);
  return n;
}

bv_status bv_phmm_compute_regions(bv_phmm_ctx* ctx, const bv_region_batch* batch, double* out, bv_phmm_stats* stats) {
  if (!ctx || !batch) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    bvphmm::Engine& a = ctx->engine;
    const bv_phmm_options& o = a.options();
    const int64_t min_pairs = o.pipeline_min_pairs > 0 ? o.pipeline_min_pairs : (int64_t)1 << 22;
    const int64_t pairs = bv_phmm_region_results(batch);
    // default: one chunk per min_pairs pairs, 2 to 64 chunks
    const int chunks = o.pipeline_chunks > 0 ? o.pipeline_chunks
                                             : (int)std::min<int64_t>(64, std::max<int64_t>(2, pairs / min_pairs));
    if (chunks < 2 || pairs < min_pairs) return a.compute(*batch, out, stats);
    if (!ctx->second) {
      auto e = std::make_unique<bvphmm::Engine>(o);
      const bv_status s = e->init();
      if (s != BV_OK) return a.fail(s, std::string("second context: ") + e->last_error());
      ctx->second = std::move(e);
    }
    bvphmm::Engine& b = *ctx->second;
    if (b.mirrored_version() != a.config_version()) {
      const bv_status s = b.mirror_config(a);
      if (s != BV_OK) return a.fail(s, std::string("second context: ") + b.last_error());
    }
    return a.compute_chunked(b, *batch, out, stats, chunks);
  });
}

bv_status bv_phmm_stage_regions(bv_phmm_ctx* ctx, const bv_region_batch* batch) {
  if (!ctx || !batch) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.stage(*batch); });
}

bv_status bv_phmm_run_staged(bv_phmm_ctx* ctx, bv_phmm_stats* stats) {
  if (!ctx) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.run(stats); });
}

bv_status bv_phmm_fetch_results(bv_phmm_ctx* ctx, double* out, int64_t n) {
  if (!ctx) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.fetch(out, n); });
}

bv_status bv_phmm_compute_testcases(bv_phmm_ctx* ctx, const bv_testcase* tcs, int64_t n, double* out,
                                    bv_phmm_stats* stats) {
  if (!ctx || n < 0 || (n > 0 && (!tcs || !out))) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&]() -> bv_status {
    Flat f;
    for (int64_t k = 0; k < n; ++k) {
      const bv_testcase& t = tcs[k];
      if (t.rslen < 0 || t.haplen < 0) return ctx->engine.fail(BV_ERR_INVALID_ARG, "negative testcase length");
      if ((t.rslen > 0 && (!t.rs || !t.q || !t.i || !t.d || !t.c)) || (t.haplen > 0 && !t.hap))
        return ctx->engine.fail(BV_ERR_INVALID_ARG, "null testcase array");
      const bool same_read = k > 0 && tcs[k - 1].rs == t.rs && tcs[k - 1].rslen == t.rslen &&
                             tcs[k - 1].q == t.q && tcs[k - 1].i == t.i && tcs[k - 1].d == t.d && tcs[k - 1].c == t.c;
      if (!same_read) {
        if (k > 0) {
          f.region_reads.push_back((int64_t)f.read_off.size() - 1);
          f.region_haps.push_back((int64_t)f.hap_off.size() - 1);
        }
        f.add_read(t.rslen, t.rs, t.q, t.i, t.d, t.c);
      }
      f.add_hap(t.haplen, t.hap);
    }
    if (n > 0) {
      f.region_reads.push_back((int64_t)f.read_off.size() - 1);
      f.region_haps.push_back((int64_t)f.hap_off.size() - 1);
    }
    // Each region holds one read, so result slots follow testcase order.
    const bv_region_batch b = f.view();
    return ctx->engine.compute(b, out, stats);
  });
}

bv_status bv_phmm_shacc_calculate(bv_phmm_ctx* ctx, bv_shacc_batch* batch) {
  if (!ctx || !batch || batch->num_reads < 0 || batch->num_haps < 0) return BV_ERR_INVALID_ARG;
  if ((batch->num_reads > 0 && !batch->reads) || (batch->num_haps > 0 && !batch->haps) ||
      (batch->num_reads > 0 && batch->num_haps > 0 && !batch->results))
    return BV_ERR_INVALID_ARG;
  return guard(ctx, [&]() -> bv_status {
    Flat f;
    for (int r = 0; r < batch->num_reads; ++r) {
      const bv_shacc_read& rd = batch->reads[r];
      if (rd.length < 0 || (rd.length > 0 && (!rd.bases || !rd.q || !rd.i || !rd.d || !rd.c)))
        return ctx->engine.fail(BV_ERR_INVALID_ARG, "bad shacc read");
      f.add_read(rd.length, rd.bases, rd.q, rd.i, rd.d, rd.c);
    }
    for (int h = 0; h < batch->num_haps; ++h) {
      const bv_shacc_hap& hp = batch->haps[h];
      if (hp.length < 0 || (hp.length > 0 && !hp.bases)) return ctx->engine.fail(BV_ERR_INVALID_ARG, "bad shacc hap");
      f.add_hap(hp.length, hp.bases);
    }
    f.region_reads.push_back(batch->num_reads);
    f.region_haps.push_back(batch->num_haps);
    const int64_t n = (int64_t)batch->num_reads * batch->num_haps;
    std::vector<double> tmp((size_t)std::max<int64_t>(n, 1));
    const bv_region_batch b = f.view();
    bv_status s = ctx->engine.compute(b, tmp.data(), nullptr);
    if (s != BV_OK) return s;
    for (int64_t k = 0; k < n; ++k) batch->results[k] = (float)tmp[k];
    return BV_OK;
  });
}

int bv_phmm_debug_tables(float* pf, double* pd, float* mf, double* md, int n) {
  if (n != bvphmm::kMMEntries || !pf || !pd || !mf || !md) return -1;
  auto t = std::make_unique<bvphmm::Tables>();
  bvphmm::build_tables(t.get());
  std::memcpy(pf, t->ph2pr_f, sizeof(t->ph2pr_f));
  std::memcpy(pd, t->ph2pr_d, sizeof(t->ph2pr_d));
  std::memcpy(mf, t->mm_f, sizeof(t->mm_f));
  std::memcpy(md, t->mm_d, sizeof(t->mm_d));
  return 0;
}

void bv_phmm_default_band_options(bv_band_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->struct_size = (int32_t)sizeof(*o);
  o->enabled = 1;
  o->use_mlp = 0;
  o->fixed_half = 8;
  o->margin = 2;
  o->audit_period = 0;
  o->edge_threshold = 1e-3;
  o->cap_margin = 12.f;
}

bv_status bv_phmm_set_band_options(bv_phmm_ctx* ctx, const bv_band_options* o) {
  if (!ctx || !o) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.set_band_options(*o); });
}

void bv_phmm_default_band_train_options(bv_band_train_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->struct_size = (int32_t)sizeof(*o);
  o->epochs = 20;
  o->batch = 1024;
  o->lr = 2e-3f;
  o->alpha = 16.f;
  o->tau = 1e-4f;
  o->clip = 20.f;
  o->margin = 2;
  o->seed = 1234;
}

bv_status bv_phmm_band_train(bv_phmm_ctx* ctx, const bv_region_batch* train, const bv_band_train_options* o,
                             bv_band_train_report* report) {
  if (!ctx || !train || !o) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    bv_band_train_report r{};
    const bv_status s = ctx->engine.band_train(*train, *o, &r);
    if (report) *report = r;
    return s;
  });
}

bv_status bv_phmm_band_labels(bv_phmm_ctx* ctx, const bv_region_batch* batch, float tau, int32_t* dstar, int32_t* lo,
                              int32_t* hi, float* features, int32_t* kmin, int32_t* kmax) {
  if (!ctx || !batch || !dstar || !lo || !hi) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.band_labels(*batch, tau, dstar, lo, hi, features, kmin, kmax); });
}

bv_status bv_phmm_band_routes(bv_phmm_ctx* ctx, int64_t n, int32_t* d_lo, int32_t* width, int32_t* route) {
  if (!ctx || !d_lo || !width || !route || n < 0) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.band_routes(n, d_lo, width, route); });
}

int64_t bv_phmm_band_param_count(void) { return bvphmm::kMlpParamCount; }

bv_status bv_phmm_band_get_weights(bv_phmm_ctx* ctx, float* w, int64_t n) {
  if (!ctx || !w) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.band_get_weights(w, n); });
}

bv_status bv_phmm_band_set_weights(bv_phmm_ctx* ctx, const float* w, int64_t n) {
  if (!ctx || !w) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.band_set_weights(w, n); });
}

bv_status bv_phmm_set_transitions(bv_phmm_ctx* ctx, const double* trans7) {
  if (!ctx) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.set_transitions(trans7); });
}

int bv_phmm_get_transitions(const bv_phmm_ctx* ctx, double* trans7) {
  if (!ctx) return 0;
  return ctx->engine.constant_transitions(trans7) ? 1 : 0;
}

int64_t bv_phmm_debug_chunks(const bv_region_batch* batch, int32_t chunks, int64_t* out, int64_t max) {
  if (!batch || chunks < 1 || batch->num_regions < 0 || (batch->num_regions > 0 && (!batch->region_reads ||
                                                                                  !batch->region_haps)))
    return -1;
  const auto cuts = bvphmm::plan_chunks(*batch, chunks);
  for (int64_t k = 0; out && k < (int64_t)cuts.size() && k < max; ++k) {
    out[4 * k] = cuts[k].g0;
    out[4 * k + 1] = cuts[k].g1;
    out[4 * k + 2] = cuts[k].out0;
    out[4 * k + 3] = cuts[k].n_out;
  }
  return (int64_t)cuts.size();
}

int bv_phmm_debug_jacobian_table(double* out, int n) {
  std::vector<double> t(bvphmm::kJacobianEntries);
  bvphmm::build_jacobian_table(t.data());
  for (int k = 0; out && k < n && k < bvphmm::kJacobianEntries; ++k) out[k] = t[k];
  return bvphmm::kJacobianEntries;
}

bv_status bv_phmm_genotype_staged(bv_phmm_ctx* ctx, const bv_region_batch* staged, const bv_genotype_batch* gt,
                                  int32_t* kept_count, int32_t* kept_reads, double* allele_lik,
                                  double* genotype_lik, double* kernel_ms) {
  if (!ctx || !staged || !gt) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    return ctx->engine.genotype_staged(*staged, *gt, kept_count, kept_reads, allele_lik, genotype_lik, kernel_ms);
  });
}

bv_status bv_phmm_band_save(bv_phmm_ctx* ctx, const char* path) {
  if (!ctx || !path) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.band_save(path); });
}

bv_status bv_phmm_band_load(bv_phmm_ctx* ctx, const char* path) {
  if (!ctx || !path) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.band_load(path); });
}

bv_status bv_phmm_band_mlp_eval(bv_phmm_ctx* ctx, const float* w, const float* x, const float* targets, int64_t n,
                                float alpha, float* out, float* loss, float* grad) {
  if (!ctx || !w || !x || !targets || !out || !loss || n <= 0) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.band_mlp_eval(w, x, targets, n, alpha, out, loss, grad); });
}

bv_status bv_phmm_band_mlp_infer(bv_phmm_ctx* ctx, const float* x, int64_t n, float* out) {
  if (!ctx || !x || !out || n <= 0) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.band_mlp_infer(x, n, out); });
}

bv_status bv_phmm_autotune(bv_phmm_ctx* ctx, const bv_region_batch* sample, int32_t repeats, bv_phmm_tune_entry* out,
                           int32_t* num_out) {
  if (!ctx || !sample || !out || !num_out) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.autotune(*sample, repeats, out, num_out); });
}

bv_status bv_phmm_set_tuning(bv_phmm_ctx* ctx, const bv_phmm_tune_entry* entries, int32_t num) {
  if (!ctx) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.set_tuning(entries, num); });
}

bv_status bv_phmm_get_tuning(bv_phmm_ctx* ctx, bv_phmm_tune_entry* out, int32_t* num_out) {
  if (!ctx || !out || !num_out) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.get_tuning(out, num_out); });
}

bv_status bv_phmm_set_long_warps(bv_phmm_ctx* ctx, int32_t warps) {
  if (!ctx) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.set_long_warps(warps); });
}

int32_t bv_phmm_get_long_warps(const bv_phmm_ctx* ctx) { return ctx ? ctx->engine.long_warps() : 0; }

bv_status bv_phmm_autotune_long(bv_phmm_ctx* ctx, const bv_region_batch* sample, int32_t repeats, int32_t* warps_out,
                                double* ms_out) {
  if (!ctx || !sample || !warps_out || !ms_out) return BV_ERR_INVALID_ARG;
  return guard(ctx, [&] { return ctx->engine.autotune_long(*sample, repeats, warps_out, ms_out); });
}

bv_status bv_phmm_host_register(bv_phmm_ctx* ctx, void* ptr, size_t bytes) {
  if (!ctx || !ptr || bytes == 0) return BV_ERR_INVALID_ARG;
  cudaError_t e = cudaSetDevice(ctx->engine.device());
  if (e == cudaSuccess) e = cudaHostRegister(ptr, bytes, cudaHostRegisterDefault);
  if (e != cudaSuccess) return ctx->engine.cuda_fail(e, "cudaHostRegister");
  return BV_OK;
}

bv_status bv_phmm_host_unregister(bv_phmm_ctx* ctx, void* ptr) {
  if (!ctx || !ptr) return BV_ERR_INVALID_ARG;
  cudaError_t e = cudaHostUnregister(ptr);
  if (e != cudaSuccess) return ctx->engine.cuda_fail(e, "cudaHostUnregister");
  return BV_OK;
}

}  // extern "C"
