// phmm_engine_train.cpp -- band MLP training, labels, weight I/O (see
// phmm_mlp.h for the kernels).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "phmm_engine.h"
#include "phmm_mlp.h"

namespace bvphmm {

#define BV_CUDA(call, what)                                  \
  do {                                                       \
    cudaError_t e__ = (call);                                \
    if (e__ != cudaSuccess) return cuda_fail(e__, what);     \
  } while (0)

namespace {

constexpr char kMagic[8] = {'B', 'V', 'B', 'A', 'N', 'D', 'W', '\0'};
constexpr uint32_t kWeightVersion = 1;
constexpr size_t kLabelBufLimit = size_t(6) << 30;  // forward-row buffers of the label kernel

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Carves the training buffers out of one allocation.
struct TrainArena {
  size_t bytes = 0;
  MlpTrainBuffers b{};
  void layout(char* base, int cap, int loss_slots) {
    size_t off = 0;
    auto take = [&](size_t n) {
      float* p = base ? reinterpret_cast<float*>(base + off) : nullptr;
      off += align256(n * sizeof(float));
      return p;
    };
    b.w = take(kMlpParamCount);
    b.wq = take(kMlpParamCount);
    b.g = take(kMlpParamCount);
    b.m = take(kMlpParamCount);
    b.v = take(kMlpParamCount);
    b.X = take((size_t)cap * kFeat);
    b.T = take((size_t)cap * 2);
    b.mask = take((size_t)cap);
    b.Z1 = take((size_t)cap * kHid);
    b.H1 = take((size_t)cap * kHid);
    b.Z2 = take((size_t)cap * kHid);
    b.H2 = take((size_t)cap * kHid);
    b.O = take((size_t)cap * kOut);
    b.dO = take((size_t)cap * kOut);
    b.dH = take((size_t)cap * kHid);
    b.dH2 = take((size_t)cap * kHid);
    b.loss = take((size_t)std::max(loss_slots, 1));
    b.part = take((size_t)((cap + 127) / 128) * kHid * kHid);
    b.tc_fail = reinterpret_cast<unsigned int*>(take(1));
    b.cap = cap;
    bytes = off;
  }
};

float bf16_to_float(uint16_t h) {
  const uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

}  // namespace

bv_status Engine::stage_for_labels(const bv_region_batch& b) {
  if (constant_transitions(nullptr))
    return fail(BV_ERR_UNSUPPORTED, "band labels take their transitions from the quality bytes");
  staged_ = false;
  destroy_graph();
  BV_CUDA(cudaSetDevice(opt_.device), "cudaSetDevice");
  bv_status s = validate(b);
  if (s != BV_OK) return s;
  s = upload_inputs(b);
  if (s != BV_OK) return s;
  s = plan(b);
  if (s != BV_OK) return s;
  s = upload_plan();
  if (s != BV_OK) return s;
  s = band_prepare();
  if (s != BV_OK) return s;
  BandParams p = band_params();
  BV_CUDA(cudaMemsetAsync(d_bctr_.get(), 0, sizeof(BandCounters), stream_), "memset band counters");
  BV_CUDA(launch_hap_table(p.batch.hap_bases, p.batch.hap_off, n_haps_, n_hap_bytes_, d_hap_table_.as<uint32_t>(),
                           d_hap_nib_.as<uint32_t>(), sms_, stream_),
          "hap tables");
  BV_CUDA(launch_read_kmers(p.batch.read_bases, n_read_bytes_, d_read_kmers_.as<uint32_t>(), sms_, stream_), "kmers");
  BV_CUDA(launch_featurize(p, sms_, stream_), "featurize");
  return BV_OK;
}

bv_status Engine::compute_labels(const bv_region_batch& b, float tau, float* ms) {
  int max_r = 0, max_h = 0;
  for (int64_t r = 0; r < b.num_reads; ++r) max_r = std::max<int>(max_r, (int)(b.read_offsets[r + 1] - b.read_offsets[r]));
  for (int64_t h = 0; h < b.num_haps; ++h) max_h = std::max<int>(max_h, (int)(b.hap_offsets[h + 1] - b.hap_offsets[h]));
  max_r = std::min(max_r, kBandMaxRead);
  max_h = std::min(max_h, kBandMaxHap);
  const long long stride = (long long)(max_r + 1) * 3 * (max_h + 2);
  const size_t per_block = (size_t)stride * sizeof(float) * label_warps_per_block();
  const int blocks = (int)std::max<size_t>(1, std::min<size_t>((size_t)sms_ * 2, kLabelBufLimit / per_block));
  const int64_t n = std::max<int64_t>(n_results_, 1);
  BV_CUDA(d_lab_lo_.reserve(sizeof(int32_t) * n), "alloc labels");
  BV_CUDA(d_lab_hi_.reserve(sizeof(int32_t) * n), "alloc labels");
  BV_CUDA(d_lab_fbuf_.reserve(per_block * blocks), "alloc label rows");
  DeviceBatch db{};
  db.read_bases = d_read_bases_.as<uint8_t>();
  db.read_quals = d_quals4_.as<uchar4>();
  db.read_off = d_read_off_.as<int64_t>();
  db.hap_bases = d_hap_bases_.as<uint8_t>();
  db.hap_off = d_hap_off_.as<int64_t>();
  BV_CUDA(cudaEventRecord(ev_[0], stream_), "event");
  BV_CUDA(launch_posterior_spread(db, d_tables_.as<Tables>(), d_pair_read_.as<int32_t>(), d_pair_hap_.as<int32_t>(),
                                  n_results_, tau, d_lab_fbuf_.as<float>(), stride, d_lab_lo_.as<int32_t>(),
                                  d_lab_hi_.as<int32_t>(), blocks, stream_), "labels");
  BV_CUDA(cudaEventRecord(ev_[1], stream_), "event");
  BV_CUDA(cudaStreamSynchronize(stream_), "labels sync");
  float t = 0;
  BV_CUDA(cudaEventElapsedTime(&t, ev_[0], ev_[1]), "event time");
  if (ms) *ms = t;
  return BV_OK;
}

bv_status Engine::band_labels(const bv_region_batch& b, float tau, int32_t* dstar, int32_t* lo, int32_t* hi,
                              float* feat, int32_t* kmin, int32_t* kmax) {
  bv_status s = stage_for_labels(b);
  if (s != BV_OK) return s;
  s = compute_labels(b, tau, nullptr);
  if (s != BV_OK) return s;
  const size_t n = (size_t)n_results_;
  if (n == 0) return BV_OK;
  BV_CUDA(cudaMemcpy(dstar, d_dstar_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
  BV_CUDA(cudaMemcpy(lo, d_lab_lo_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
  BV_CUDA(cudaMemcpy(hi, d_lab_hi_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
  if (kmin) BV_CUDA(cudaMemcpy(kmin, d_kmin_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
  if (kmax) BV_CUDA(cudaMemcpy(kmax, d_kmax_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
  if (feat) {
    std::vector<uint16_t> f(n * kFeat);
    BV_CUDA(cudaMemcpy(f.data(), d_feat_.get(), f.size() * 2, cudaMemcpyDeviceToHost), "D2H");
    for (size_t x = 0; x < f.size(); ++x) feat[x] = bf16_to_float(f[x]);
  }
  return BV_OK;
}

bv_status Engine::install_weights(const float* w) {
  BV_CUDA(cudaSetDevice(opt_.device), "cudaSetDevice");
  for (int x = 0; x < kMlpParamCount; ++x)
    if (!std::isfinite(w[x])) return fail(BV_ERR_INVALID_ARG, "band MLP weight is not finite");
  BV_CUDA(d_mlp_w_.reserve(sizeof(float) * kMlpParamCount), "alloc weights");
  BV_CUDA(d_mlp_.reserve(sizeof(MlpParams)), "alloc mlp");
  BV_CUDA(cudaMemcpyAsync(d_mlp_w_.get(), w, sizeof(float) * kMlpParamCount, cudaMemcpyHostToDevice, stream_), "H2D");
  BV_CUDA(mlp_export(d_mlp_w_.as<float>(), d_mlp_.as<MlpParams>(), stream_), "export weights");
  BV_CUDA(cudaStreamSynchronize(stream_), "weights sync");
  mlp_w_.assign(w, w + kMlpParamCount);
  mlp_ready_ = true;
  ++config_version_;
  destroy_graph();  // a captured launch sequence may read the old weights only through d_mlp_ (same address)
  return BV_OK;
}

bv_status Engine::band_get_weights(float* w, int64_t n) {
  if (n != kMlpParamCount) return fail(BV_ERR_INVALID_ARG, "weight count");
  if (!mlp_ready_) return fail(BV_ERR_INVALID_ARG, "no band MLP weights (train or load)");
  std::memcpy(w, mlp_w_.data(), sizeof(float) * kMlpParamCount);
  return BV_OK;
}

bv_status Engine::band_set_weights(const float* w, int64_t n) {
  if (n != kMlpParamCount) return fail(BV_ERR_INVALID_ARG, "weight count");
  return install_weights(w);
}

bv_status Engine::band_save(const char* path) {
  if (!mlp_ready_) return fail(BV_ERR_INVALID_ARG, "no band MLP weights (train or load)");
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(BV_ERR_INVALID_ARG, std::string("cannot open ") + path);
  const uint32_t hdr[5] = {kWeightVersion, (uint32_t)kFeat, (uint32_t)kHid, (uint32_t)kOut, (uint32_t)kMlpParamCount};
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(hdr, 4, 5, f) == 5 &&
            std::fwrite(mlp_w_.data(), 4, kMlpParamCount, f) == (size_t)kMlpParamCount;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? BV_OK : fail(BV_ERR_INVALID_ARG, std::string("write failed: ") + path);
}

bv_status Engine::band_load(const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(BV_ERR_INVALID_ARG, std::string("cannot open ") + path);
  char magic[8];
  uint32_t hdr[5];
  std::vector<float> w(kMlpParamCount);
  const bool ok = std::fread(magic, 1, 8, f) == 8 && std::fread(hdr, 4, 5, f) == 5 &&
                  std::memcmp(magic, kMagic, 8) == 0 && hdr[0] == kWeightVersion && hdr[1] == (uint32_t)kFeat &&
                  hdr[2] == (uint32_t)kHid && hdr[3] == (uint32_t)kOut && hdr[4] == (uint32_t)kMlpParamCount &&
                  std::fread(w.data(), 4, kMlpParamCount, f) == (size_t)kMlpParamCount;
  std::fclose(f);
  if (!ok) return fail(BV_ERR_INVALID_ARG, std::string("not a band weight file of this layout: ") + path);
  return install_weights(w.data());
}

bv_status Engine::band_mlp_eval(const float* w, const float* x, const float* t, int64_t n, float alpha, float* out,
                                float* loss, float* grad) {
  BV_CUDA(cudaSetDevice(opt_.device), "cudaSetDevice");
  if (n > (1 << 24)) return fail(BV_ERR_INVALID_ARG, "too many rows");
  TrainArena a;
  a.layout(nullptr, (int)n, 1);
  DevBuf mem;
  BV_CUDA(mem.reserve(a.bytes), "alloc eval");
  a.layout(mem.as<char>(), (int)n, 1);
  MlpTrainBuffers b = a.b;
  b.mask = nullptr;
  BV_CUDA(cudaMemcpyAsync(b.w, w, sizeof(float) * kMlpParamCount, cudaMemcpyHostToDevice, stream_), "H2D");
  BV_CUDA(cudaMemcpyAsync(b.X, x, sizeof(float) * kFeat * n, cudaMemcpyHostToDevice, stream_), "H2D");
  BV_CUDA(cudaMemcpyAsync(b.T, t, sizeof(float) * 2 * n, cudaMemcpyHostToDevice, stream_), "H2D");
  BV_CUDA(cudaMemsetAsync(b.tc_fail, 0, sizeof(unsigned int), stream_), "memset");
  BV_CUDA(mlp_forward_backward(b, (int)n, alpha, grad != nullptr, stream_), "mlp eval");
  BV_CUDA(cudaMemcpyAsync(out, b.O, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost, stream_), "D2H");
  BV_CUDA(cudaMemcpyAsync(loss, b.loss, sizeof(float), cudaMemcpyDeviceToHost, stream_), "D2H");
  if (grad) BV_CUDA(cudaMemcpyAsync(grad, b.g, sizeof(float) * kMlpParamCount, cudaMemcpyDeviceToHost, stream_), "D2H");
  unsigned int tc_fail = 0;
  BV_CUDA(cudaMemcpyAsync(&tc_fail, b.tc_fail, sizeof(tc_fail), cudaMemcpyDeviceToHost, stream_), "D2H");
  BV_CUDA(cudaStreamSynchronize(stream_), "eval sync");
  if (tc_fail) return status_fail(16);
  return BV_OK;
}

bv_status Engine::band_mlp_infer(const float* x, int64_t n, float* out) {
  BV_CUDA(cudaSetDevice(opt_.device), "cudaSetDevice");
  if (!mlp_ready_) return fail(BV_ERR_INVALID_ARG, "no band MLP weights (train or load)");
  if (n < 0 || n > (1 << 24)) return fail(BV_ERR_INVALID_ARG, "row count out of range");
  if (n == 0) return BV_OK;
  // features to BF16, round to nearest even (the featuriser's rounding)
  std::vector<uint16_t> xb((size_t)n * kFeat);
  for (size_t i = 0; i < xb.size(); ++i) {
    uint32_t u;
    std::memcpy(&u, &x[i], 4);
    xb[i] = (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
  }
  DevBuf df, dout, dctr;
  BV_CUDA(df.reserve(xb.size() * 2), "alloc features");
  BV_CUDA(dout.reserve(sizeof(float) * kOut * (size_t)n), "alloc outputs");
  BV_CUDA(dctr.reserve(sizeof(Counters)), "alloc counters");
  BV_CUDA(cudaMemsetAsync(dctr.get(), 0, sizeof(Counters), stream_), "memset");
  BV_CUDA(cudaMemcpyAsync(df.get(), xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, stream_), "H2D");
  BandParams p{};
  p.n_pairs = n;
  p.feat = df.as<__nv_bfloat16>();
  p.mlp_out = dout.as<float>();
  p.mlp = d_mlp_.as<MlpParams>();
  p.ctr = dctr.as<Counters>();
  BV_CUDA(prepare_band_kernels(), "band kernel attributes");
  BV_CUDA(launch_mlp_forward(p, sms_, stream_), "mlp forward");
  Counters c{};
  BV_CUDA(cudaMemcpyAsync(out, dout.get(), sizeof(float) * kOut * (size_t)n, cudaMemcpyDeviceToHost, stream_), "D2H");
  BV_CUDA(cudaMemcpyAsync(&c, dctr.get(), sizeof(Counters), cudaMemcpyDeviceToHost, stream_), "D2H");
  BV_CUDA(cudaStreamSynchronize(stream_), "infer sync");
  if (c.status != 0) return status_fail(c.status);
  return BV_OK;
}

bv_status Engine::band_train(const bv_region_batch& bt, const bv_band_train_options& o, bv_band_train_report* rep) {
  if (o.struct_size != (int32_t)sizeof(bv_band_train_options)) return fail(BV_ERR_INVALID_ARG, "train options size");
  if (o.epochs < 1 || o.batch < 16 || o.batch > (1 << 20) || !(o.lr > 0) || !(o.alpha >= 1) || !(o.tau > 0) ||
      !(o.tau < 1) || !(o.clip >= 1) || o.margin < 0)
    return fail(BV_ERR_INVALID_ARG, "train option out of range");
  *rep = bv_band_train_report{};
  bv_status s = stage_for_labels(bt);
  if (s != BV_OK) return s;
  float ms_lab = 0;
  s = compute_labels(bt, o.tau, &ms_lab);
  if (s != BV_OK) return s;
  const int64_t n = n_results_;
  if (n > INT32_MAX) return fail(BV_ERR_INVALID_ARG, "training batch too large");
  rep->pairs = n;
  rep->ms_labels = ms_lab;
  std::vector<int32_t> ds(n), lo(n), hi(n), km(n), kx(n), pr(n);
  if (n > 0) {
    BV_CUDA(cudaMemcpy(ds.data(), d_dstar_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
    BV_CUDA(cudaMemcpy(lo.data(), d_lab_lo_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
    BV_CUDA(cudaMemcpy(hi.data(), d_lab_hi_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
    BV_CUDA(cudaMemcpy(km.data(), d_kmin_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
    BV_CUDA(cudaMemcpy(kx.data(), d_kmax_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
    BV_CUDA(cudaMemcpy(pr.data(), d_pair_read_.get(), n * 4, cudaMemcpyDeviceToHost), "D2H");
  }
  // training rows: seeded pairs with a label and a read the banded kernel takes
  std::vector<int32_t> rows;
  std::vector<float> targets((size_t)std::max<int64_t>(n, 1) * 2, 0.f);
  double mean_lo = 0, mean_hi = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int R = (int)(bt.read_offsets[pr[i] + 1] - bt.read_offsets[pr[i]]);
    if (ds[i] == INT32_MIN || lo[i] == INT32_MIN || R > kBandMaxRead) continue;
    const float tl = std::clamp((float)(lo[i] - ds[i]), -o.clip, o.clip);
    const float th = std::clamp((float)(hi[i] - ds[i]), -o.clip, o.clip);
    targets[2 * i] = tl;
    targets[2 * i + 1] = th;
    mean_lo += tl;
    mean_hi += th;
    rows.push_back((int32_t)i);
  }
  const int64_t nl = (int64_t)rows.size();
  rep->labelled = nl;
  if (nl == 0) return fail(BV_ERR_INVALID_ARG, "no labelled pairs in the training batch");
  mean_lo /= (double)nl;
  mean_hi /= (double)nl;

  // He-uniform initialisation; the output layer starts small, biased to the mean label
  std::mt19937_64 rng(o.seed);
  std::vector<float> w(kMlpParamCount, 0.f);
  auto fill = [&](size_t off, int fan_out, int fan_in, float scale) {
    std::uniform_real_distribution<float> u(-scale * std::sqrt(6.f / fan_in), scale * std::sqrt(6.f / fan_in));
    for (size_t x = 0; x < (size_t)fan_out * fan_in; ++x) w[off + x] = u(rng);
  };
  const size_t o1 = 0, ob1 = (size_t)kHid * kFeat, o2 = ob1 + kHid, ob2 = o2 + (size_t)kHid * kHid, o3 = ob2 + kHid,
               ob3 = o3 + (size_t)kOut * kHid;
  fill(o1, kHid, kFeat, 1.f);
  fill(o2, kHid, kHid, 1.f);
  fill(o3, kOut, kHid, 0.1f);
  w[ob3] = (float)mean_lo;
  w[ob3 + 1] = (float)mean_hi;

  const int batch = (int)std::min<int64_t>(o.batch, nl);
  const int steps_per_epoch = (int)((nl + batch - 1) / batch);
  const int total_steps = steps_per_epoch * o.epochs;
  TrainArena a;
  a.layout(nullptr, batch, total_steps);
  DevBuf mem, d_targets, d_perm;
  BV_CUDA(mem.reserve(a.bytes), "alloc training");
  a.layout(mem.as<char>(), batch, total_steps);
  MlpTrainBuffers b = a.b;
  BV_CUDA(d_targets.reserve(targets.size() * sizeof(float)), "alloc targets");
  BV_CUDA(d_perm.reserve(sizeof(int32_t) * nl), "alloc permutation");
  BV_CUDA(cudaMemcpyAsync(d_targets.get(), targets.data(), targets.size() * sizeof(float), cudaMemcpyHostToDevice,
                          stream_), "H2D");
  BV_CUDA(cudaMemcpyAsync(b.w, w.data(), sizeof(float) * kMlpParamCount, cudaMemcpyHostToDevice, stream_), "H2D");
  BV_CUDA(cudaMemsetAsync(b.m, 0, sizeof(float) * kMlpParamCount, stream_), "memset");
  BV_CUDA(cudaMemsetAsync(b.v, 0, sizeof(float) * kMlpParamCount, stream_), "memset");
  BV_CUDA(cudaMemsetAsync(b.tc_fail, 0, sizeof(unsigned int), stream_), "memset");
  float* loss_hist = b.loss;
  BV_CUDA(cudaEventRecord(ev_[0], stream_), "event");
  int step = 0;
  const int warm = std::min(50, total_steps / 10 + 1);
  for (int ep = 0; ep < o.epochs; ++ep) {
    std::shuffle(rows.begin(), rows.end(), rng);
    // the copy from `rows` must finish before the next shuffle rewrites it
    BV_CUDA(cudaMemcpyAsync(d_perm.get(), rows.data(), sizeof(int32_t) * nl, cudaMemcpyHostToDevice, stream_), "H2D");
    for (int k = 0; k < steps_per_epoch; ++k, ++step) {
      const int nb = (int)std::min<int64_t>(batch, nl - (int64_t)k * batch);
      b.loss = loss_hist + step;
      BV_CUDA(mlp_gather(d_feat_.as<__nv_bfloat16>(), d_targets.as<float>(), nullptr, d_perm.as<int32_t>() + (size_t)k * batch,
                         nb, b, stream_), "gather");
      BV_CUDA(mlp_forward_backward(b, nb, o.alpha, true, stream_), "forward/backward");
      const float prog = (float)step / (float)std::max(total_steps - 1, 1);
      const float lr = step < warm ? o.lr * (float)(step + 1) / (float)warm
                                   : o.lr * (0.02f + 0.98f * 0.5f * (1.f + std::cos(3.14159265f * prog)));
      BV_CUDA(mlp_adam(b, step + 1, lr, stream_), "adam");
    }
    BV_CUDA(cudaStreamSynchronize(stream_), "epoch sync");
  }
  BV_CUDA(cudaEventRecord(ev_[1], stream_), "event");
  BV_CUDA(cudaStreamSynchronize(stream_), "train sync");
  float ms_train = 0;
  BV_CUDA(cudaEventElapsedTime(&ms_train, ev_[0], ev_[1]), "event time");
  rep->ms_train = ms_train;
  rep->steps = total_steps;
  {
    unsigned int tc_fail = 0;
    BV_CUDA(cudaMemcpy(&tc_fail, b.tc_fail, sizeof(tc_fail), cudaMemcpyDeviceToHost), "D2H");
    if (tc_fail) return status_fail(16);
  }
  std::vector<float> lh(total_steps);
  BV_CUDA(cudaMemcpy(lh.data(), loss_hist, sizeof(float) * total_steps, cudaMemcpyDeviceToHost), "D2H");
  rep->first_loss = (float)(std::accumulate(lh.begin(), lh.begin() + steps_per_epoch, 0.0) / steps_per_epoch);
  rep->last_loss = (float)(std::accumulate(lh.end() - steps_per_epoch, lh.end(), 0.0) / steps_per_epoch);
  BV_CUDA(cudaMemcpy(w.data(), b.w, sizeof(float) * kMlpParamCount, cudaMemcpyDeviceToHost), "D2H");
  s = install_weights(w.data());
  if (s != BV_OK) return s;

  // coverage of the routed band over the labels, with the inference kernel
  BandParams p = band_params();
  p.use_mlp = 1;
  BV_CUDA(launch_mlp_forward(p, sms_, stream_), "mlp forward");
  std::vector<float> mo((size_t)n * kOut);
  BV_CUDA(cudaMemcpyAsync(mo.data(), d_mlp_out_.get(), mo.size() * sizeof(float), cudaMemcpyDeviceToHost, stream_), "D2H");
  BV_CUDA(cudaStreamSynchronize(stream_), "coverage sync");
  int64_t banded = 0, covered = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int R = (int)(bt.read_offsets[pr[i] + 1] - bt.read_offsets[pr[i]]);
    if (ds[i] == INT32_MIN || lo[i] == INT32_MIN || R > kBandMaxRead) continue;
    const float fl = mo[2 * i], fh = mo[2 * i + 1];
    if (!(fl <= fh) || !std::isfinite(fl) || !std::isfinite(fh) || km[i] == INT32_MIN || kx[i] == INT32_MAX) continue;
    const int blo = std::min(ds[i] + (int)std::floor(fl) - o.margin, km[i]);
    const int bhi = std::max(ds[i] + (int)std::ceil(fh) + o.margin, kx[i]);
    if (bhi - blo + 1 > band_width(kBandWidths - 1)) continue;
    ++banded;
    covered += (blo <= lo[i] && bhi >= hi[i]);
  }
  rep->band_frac = (double)banded / (double)nl;
  rep->cover_frac = banded > 0 ? (double)covered / (double)banded : 0.0;
  return BV_OK;
}

}  // namespace bvphmm
