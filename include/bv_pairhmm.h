/*
 * bv_pairhmm.h -- C ABI of the B200 PairHMM forward pass.
 *
 * A drop-in for Biovoltron's PairHMM likelihood call.  Every entry point takes
 * plain pointers and sizes; sequence and quality memory is borrowed for the
 * duration of the call, results go to caller-provided memory, and nothing here
 * throws or aborts: each function returns a bv_status.
 *
 * Input conventions are the reference kernel's (lib/intel_native/pairhmm/
 * pairhmm_common.h:20-44, avx-pairhmm-template.h:3-35, 108-127):
 *   - bases are bytes; A C T G N map to codes 0..4, every other byte reads
 *     as A; a read or haplotype N matches every base;
 *   - q (base), i (insertion), d (deletion) and c (gap continuation) qualities
 *     are raw Phred bytes, used (byte & 127) with no ASCII offset;
 *   - a result is log10 of the pair likelihood: the FP32 forward pass, or the
 *     FP64 pass when the FP32 value scaled by 2^120 is below 1e-28 or not
 *     finite (include/biovoltron/algo/align/inexact_match/pairhmm_avx.hpp:
 *     136-149).  The FP64 pass renormalises long reads, so results stay
 *     finite where the reference's FP64 underflows to -inf.
 *   - a pair with an empty read or an empty haplotype has log10 -inf.
 *
 * Threading: a context owns one CUDA stream and its device buffers; it is not
 * thread-safe.  Use one context per host thread (or per GPU).  Calls are
 * synchronous at the API.
 */
#ifndef BV_PAIRHMM_H
#define BV_PAIRHMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BV_PHMM_ABI_VERSION 1

typedef enum bv_status {
  BV_OK = 0,
  BV_ERR_INVALID_ARG = 1, /* bad pointer, size, offset or length over the limits below */
  BV_ERR_OOM = 2,         /* device or pinned host allocation failed */
  BV_ERR_CUDA = 3,        /* a CUDA call failed; see bv_phmm_last_error */
  BV_ERR_TIMEOUT = 4,     /* a device wait exceeded its bound */
  BV_ERR_NO_DEVICE = 5,   /* no CUDA device, or the ordinal does not exist */
  BV_ERR_INTERNAL = 6,    /* a kernel reported an inconsistent state */
  BV_ERR_UNSUPPORTED = 7  /* option or feature not available in this build */
} bv_status;

/* Longest haplotype one pair may have (bytes).  Reads may be of any length
 * up to BV_PHMM_MAX_READ_LEN. */
#define BV_PHMM_MAX_HAP_LEN 32768
#define BV_PHMM_MAX_READ_LEN (1 << 20)

enum bv_phmm_precision {
  BV_PRECISION_AUTO = 0, /* FP32, FP64 for pairs below the rescue threshold (AvxPairHMM default) */
  BV_PRECISION_F64 = 1   /* FP64 for every pair (AvxPairHMM::initNative(use_double = true)) */
};

enum bv_phmm_mode {
  BV_MODE_FULL = 0, /* full DP matrix for every pair */
  BV_MODE_BAND = 1  /* learned diagonal band, full DP on band-edge fallback */
};

typedef struct bv_phmm_options {
  int32_t struct_size;      /* sizeof(bv_phmm_options) */
  int32_t device;           /* CUDA device ordinal */
  int32_t precision;        /* bv_phmm_precision */
  int32_t mode;             /* bv_phmm_mode */
  double rescue_threshold;  /* FP32 value (scaled by 2^120) below which FP64 runs; default 1e-28 */
  int32_t haps_per_unit;    /* haplotypes one warp scores against a read before taking new work; default 8 */
  int32_t reserved[7];
} bv_phmm_options;

typedef struct bv_phmm_stats {
  int64_t pairs;          /* result slots written */
  int64_t cells;          /* sum of read_len * hap_len over the pairs */
  int64_t rescued;        /* pairs recomputed in FP64 */
  int64_t underflow;      /* FP64 results that were not positive (log10 -inf) */
  int64_t band_pairs;     /* pairs scored by the banded kernel */
  int64_t band_fallback;  /* banded pairs sent back to the full DP */
  int64_t band_cells;     /* cells the banded kernel computed */
  int64_t kernel_launches;
  double ms_h2d;          /* host->device copies (events on the context stream) */
  double ms_fp32;         /* FP32 forward kernels */
  double ms_fp64;         /* FP64 rescue kernel */
  double ms_band;         /* featurise + band MLP + banded DP kernels */
  double ms_d2h;          /* device->host copy of the results */
  double ms_total;        /* whole call, host wall clock */
} bv_phmm_stats;

typedef struct bv_phmm_ctx bv_phmm_ctx;

void bv_phmm_default_options(bv_phmm_options* opts);
int bv_phmm_abi_version(void);
const char* bv_phmm_status_string(bv_status s);

/* Context lifetime.  Creates a CUDA stream on opts->device and uploads the
 * probability tables (Context.h:42-175).  Replaces the per-call set-up of
 * AvxPairHMM::initNative (pairhmm_avx.hpp:83-119). */
bv_status bv_phmm_create(const bv_phmm_options* opts, bv_phmm_ctx** out);
void bv_phmm_destroy(bv_phmm_ctx* ctx);
/* Message describing the last failure on this context ("" if none). */
const char* bv_phmm_last_error(const bv_phmm_ctx* ctx);

/* --- seam 1/2: the per-pair testcase --------------------------------------
 * Layout of `testcase` (lib/intel_native/pairhmm/pairhmm_common.h:20-24).
 * bv_phmm_compute_testcases scores n testcases and writes log10 likelihoods,
 * replacing the loop of AvxPairHMM::computeLikelihoodsNative
 * (pairhmm_avx.hpp:121-157) over the function pointers
 * g_compute_full_prob_float / _double (pairhmm_avx.hpp:33-34, 113-114). */
typedef struct bv_testcase {
  int rslen, haplen;
  const char *q, *i, *d, *c;
  const char *hap, *rs;
} bv_testcase;

bv_status bv_phmm_compute_testcases(bv_phmm_ctx* ctx, const bv_testcase* tcs, int64_t n, double* out_log10,
                                    bv_phmm_stats* stats);

/* --- seam 3: the accelerator batch hook -----------------------------------
 * Layouts of shacc_pairhmm::Read / Haplotype / Batch
 * (lib/intel_native/pairhmm/shacc_pairhmm.h:12-33).  Scores every read
 * against every haplotype and writes batch->results[r * num_haps + h] =
 * log10 likelihood (float), read-major.  Replaces the weak
 * shacc_pairhmm::calculate(Batch&) (shacc_pairhmm.h:35); the library also
 * defines that C++ symbol strongly, on a process-wide context for device 0. */
typedef struct bv_shacc_read {
  int length;
  const char* bases;
  const char* q;
  const char* i;
  const char* d;
  const char* c;
} bv_shacc_read;

typedef struct bv_shacc_hap {
  int length;
  const char* bases;
} bv_shacc_hap;

typedef struct bv_shacc_batch {
  int num_reads;
  int num_haps;
  long num_cells;
  bv_shacc_read* reads;
  bv_shacc_hap* haps;
  float* results;
} bv_shacc_batch;

bv_status bv_phmm_shacc_calculate(bv_phmm_ctx* ctx, bv_shacc_batch* batch);

/* --- many active regions in one call --------------------------------------
 * The batched form of AvxPairHMM::compute_likelihoods(haps, reads)
 * (pairhmm_avx.hpp:160-171) before its normalise/filter step: region g owns
 * reads [region_reads[g], region_reads[g+1]) and haplotypes
 * [region_haps[g], region_haps[g+1]); its results are the read-major
 * [reads x haps] block, blocks concatenated in region order.  Reads and
 * haplotypes are flat byte arrays with prefix-sum offsets (n+1 entries). */
typedef struct bv_region_batch {
  int64_t num_regions;
  const int64_t* region_reads; /* [num_regions + 1] */
  const int64_t* region_haps;  /* [num_regions + 1] */
  int64_t num_reads;
  const int64_t* read_offsets; /* [num_reads + 1] */
  const uint8_t* read_bases;
  const uint8_t* read_q;
  const uint8_t* read_i;
  const uint8_t* read_d;
  const uint8_t* read_c;
  int64_t num_haps;
  const int64_t* hap_offsets; /* [num_haps + 1] */
  const uint8_t* hap_bases;
} bv_region_batch;

/* Number of result slots the batch produces (sum over regions of reads*haps). */
int64_t bv_phmm_region_results(const bv_region_batch* batch);

bv_status bv_phmm_compute_regions(bv_phmm_ctx* ctx, const bv_region_batch* batch, double* out_log10,
                                  bv_phmm_stats* stats);

/* Device-resident form of the same computation, for callers that score one
 * batch repeatedly: stage copies the batch into context-owned device memory;
 * run computes into a context-owned device result array (replayed from a
 * captured CUDA graph after the first run); fetch copies n results back. */
bv_status bv_phmm_stage_regions(bv_phmm_ctx* ctx, const bv_region_batch* batch);
bv_status bv_phmm_run_staged(bv_phmm_ctx* ctx, bv_phmm_stats* stats);
bv_status bv_phmm_fetch_results(bv_phmm_ctx* ctx, double* out_log10, int64_t n);

/* Page-locks caller memory so the context's host->device copies from it run
 * at full bandwidth (cudaHostRegister); unregister before freeing it. */
bv_status bv_phmm_host_register(bv_phmm_ctx* ctx, void* ptr, size_t bytes);
bv_status bv_phmm_host_unregister(bv_phmm_ctx* ctx, void* ptr);

/* --- scoring without any allocation (no counterpart in the reference) ----
 * For callers that cannot call cudaMalloc when they need scores: e.g. a
 * haplotype caller inside a GPU pipeline whose framework's caching allocator
 * already holds nearly all device memory (a new allocation fails or stalls the
 * whole device), or code running under a no-new-allocations policy.  They
 * pass device-resident inputs and a device output array; the library uses
 * only a fixed scratch array compiled into it (about 4.6 MB per GPU that
 * loads the library, held until exit) and allocates nothing, host or device.
 *
 * Computes, for each pair {int32 read; int32 hap; int64 out} (16 bytes each,
 * 8-byte aligned), log10 likelihood into out_log10[out] with the FP64 forward
 * pass -- the values bv_phmm_compute_regions gives with BV_PRECISION_F64.
 * Inputs are device pointers: read_quals holds 4 bytes per read position
 * (q, i, d, c; 4-byte aligned); offsets are prefix sums (n+1 entries).
 * Limits: haplotypes of at most BV_PHMM_NOALLOC_MAX_HAP_LEN bases (the caller
 * states its bound in max_hap_len; larger values are rejected with
 * BV_ERR_INVALID_ARG, and a pair whose haplotype is longer than the maximum
 * or whose indices are out of range gets NaN and makes the call return
 * BV_ERR_INVALID_ARG); reads of any length.
 * The call runs on `stream` (a cudaStream_t, NULL = legacy default stream)
 * and returns after the stream has finished it.  The first call on a device
 * sets that device up (finds the scratch array's device address, copies the
 * probability tables into it, synchronously): make it before any stream
 * capture.  All calls share the one scratch array and it keeps the last
 * call's contents (the call clears what must start at zero); calls that
 * overlap on the GPU -- from two host threads or on two streams -- race. */
#define BV_PHMM_NOALLOC_MAX_HAP_LEN 2048

typedef struct bv_phmm_device_pairs {
  int64_t num_pairs;
  const void* pairs;
  int64_t num_reads;
  const int64_t* read_offsets;
  const uint8_t* read_bases;
  const uint8_t* read_quals;
  int64_t num_haps;
  const int64_t* hap_offsets;
  const uint8_t* hap_bases;
  int32_t max_hap_len;
} bv_phmm_device_pairs;

bv_status bv_phmm_forward_f64_noalloc(int device, const bv_phmm_device_pairs* pairs, double* out_log10,
                                      int64_t num_out, void* stream);

/* Diagnostics: writes the probability tables a context uploads (ph2pr for
 * quals 0..127 and the match-to-match triangle for quals <= 127, both
 * precisions; Context.h:42-175).  Host-only, needs no device.  Returns 0, or
 * -1 if mm_entries is not 127*128/2 + 128. */
int bv_phmm_debug_tables(float* ph2pr_f32, double* ph2pr_f64, float* mm_f32, double* mm_f64, int mm_entries);

/* Diagnostics: measures the device's achievable FP32 FMA throughput (TFLOP/s,
 * 2 flops per FMA), the roofline denominator of the forward kernels, which
 * run on the CUDA-core FP32 pipe.  Returns a bv_status. */
int bv_phmm_measure_fp32_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* BV_PAIRHMM_H */
