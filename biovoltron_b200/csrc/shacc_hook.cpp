// shacc_hook.cpp -- strong definition of Biovoltron's weak accelerator hook.
//
// lib/intel_native/pairhmm/shacc_pairhmm.h:10-36 declares, with C++ linkage,
//   namespace shacc_pairhmm { struct Read; struct Haplotype; struct Batch;
//                             extern WEAK bool calculate(Batch& batch); }
// A program that includes that header and links this library gets this
// definition.  The struct declarations below repeat the header's member list
// so the mangled name and the layout are the same; they are checked against
// the C ABI's bv_shacc_* structs with static_asserts.
//
// The reference never says what `results` holds; this definition writes
// log10 likelihoods, read-major (results[r * num_haps + h]), the same values
// the C entry point bv_phmm_shacc_calculate writes.  It runs on a
// process-wide context on the device named by BV_PHMM_DEVICE (default 0),
// created on first use, and returns false on any failure.
#include <cstddef>
#include <cstdlib>
#include <mutex>

#include "bv_pairhmm.h"

namespace shacc_pairhmm {

struct Read {
  int length;
  const char* bases;
  const char* q;
  const char* i;
  const char* d;
  const char* c;
};

struct Haplotype {
  int length;
  const char* bases;
};

struct Batch {
  int num_reads;
  int num_haps;
  long num_cells;
  Read* reads;
  Haplotype* haps;
  float* results;
};

bool calculate(Batch& batch);

static_assert(sizeof(Read) == sizeof(bv_shacc_read) && offsetof(Read, c) == offsetof(bv_shacc_read, c));
static_assert(sizeof(Haplotype) == sizeof(bv_shacc_hap));
static_assert(sizeof(Batch) == sizeof(bv_shacc_batch) && offsetof(Batch, results) == offsetof(bv_shacc_batch, results));

namespace {
std::mutex g_mu;
bv_phmm_ctx* g_ctx = nullptr;
bool g_failed = false;
}  // namespace

bool calculate(Batch& batch) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_ctx && !g_failed) {
    bv_phmm_options o;
    bv_phmm_default_options(&o);
    if (const char* dev = std::getenv("BV_PHMM_DEVICE")) o.device = std::atoi(dev);
    if (bv_phmm_create(&o, &g_ctx) != BV_OK) {
      g_ctx = nullptr;
      g_failed = true;
    }
  }
  if (!g_ctx) return false;
  return bv_phmm_shacc_calculate(g_ctx, reinterpret_cast<bv_shacc_batch*>(&batch)) == BV_OK;
}

}  // namespace shacc_pairhmm
