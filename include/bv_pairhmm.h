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

#define BV_PHMM_ABI_VERSION 3

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
  int32_t haps_per_warp;    /* 2: a warp scores two haplotypes of a read at once (packed FP32x2), 1: one;
                               0 (default): 2 */
  int32_t pipeline_chunks;  /* bv_phmm_compute_regions on a batch of at least pipeline_min_pairs pairs:
                               region chunks scored by two alternating contexts on the device, one
                               chunk's copies and planning overlapping the previous chunk's kernels;
                               0 (default): one chunk per pipeline_min_pairs pairs, 2 to 64; 1: one pass */
  int32_t pipeline_min_pairs; /* 0 (default): 4,194,304 */
  int32_t reserved[4];
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
  double ms_fp32;         /* all FP32 kernels (band mode: seeding, banded DP and fallback full DP) */
  double ms_fp64;         /* FP64 rescue kernel */
  double ms_band;         /* banded forward-backward kernels */
  double ms_d2h;          /* device->host copy of the results */
  double ms_total;        /* whole call, host wall clock */
  int64_t band_routed_full; /* pairs the router sent to the full DP (no seed, too wide, too long) */
  int64_t audit_pairs;      /* banded pairs also scored by the full DP */
  double audit_max_err;     /* max |log10 band - log10 full| over the audit pairs */
  double audit_p99_err;     /* 99th percentile of the same */
  int64_t band_promoted;    /* banded pairs retried on the next wider band after the edge check */
  double ms_seed;           /* band mode: k-mer tables, featuriser, band MLP and routing kernels */
  double ms_full;           /* full-DP FP32 kernels (band mode: the fallback pairs) */
  int64_t rescued_cells;    /* DP cells the FP64 pass computed (read x haplotype length of its pairs) */
  int64_t band_result_cells; /* band mode: cells of the bands whose likelihood is the result (band plus
                                ring); band_cells adds the inner band the ring test recomputes */
  int64_t fp32_skipped_cells; /* cells of the pairs' remaining strips that the FP32 full DP left to the FP64
                                 pass when a strip proved the FP32 result below the rescue threshold */
  int64_t band_rescored;      /* banded pairs scored again by the full DP, being more than
                                 bv_band_options.cap_margin below their read's best result */
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

/* --- learned band --------------------------------------------------------
 * With `enabled`, every pair is first scored on a diagonal band around its
 * 11-mer seed diagonal: [seed + lo - margin, seed + hi + margin], where lo/hi
 * come from the band MLP (use_mlp, weights from bv_phmm_band_train or
 * bv_phmm_band_load) or are -fixed_half/+fixed_half, widened to hold every
 * diagonal a shared 11-mer votes for and rounded up to a width class of 8,
 * 16, 24 or 32 diagonals.  A banded pair is also scored on its band widened by
 * a ring of 4 (class 8) or 8 diagonals on each side; that wider band's value
 * is the result, and when the ring adds more than edge_threshold of it the
 * pair moves to the next class (after class 32: the full DP).  Pairs without
 * a seed, with a band wider than 32 diagonals or reads longer than 511 bases
 * are scored by the full DP.
 * Every audit_period-th banded pair is also scored by the full DP and the
 * differences are reported in bv_phmm_stats.  No counterpart in the reference
 * (its PairHMM always computes the full matrix). */
typedef struct bv_band_options {
  int32_t struct_size;    /* sizeof(bv_band_options) */
  int32_t enabled;
  int32_t use_mlp;
  int32_t fixed_half;
  int32_t margin;
  int32_t audit_period;
  double edge_threshold;   /* largest share of the likelihood the ring may add (default 1e-3) */
  float cap_margin;        /* a banded pair whose result lies more than this many log10 units below its
                              read's best result is scored again by the full DP (default 12; 0: off) --
                              such a pair's alternatives off the band (a stretch of the read that does not
                              belong to the haplotype, explained by a long insertion) can carry a share of
                              its likelihood the ring test does not see.  A read's results are its
                              pairs in the batch (testcases: a run of consecutive testcases sharing
                              the read); a read scored against one haplotype is never rescored */
  int32_t reserved[5];
} bv_band_options;

void bv_phmm_default_band_options(bv_band_options* opts);
bv_status bv_phmm_set_band_options(bv_phmm_ctx* ctx, const bv_band_options* opts);

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
  /* Uniform gap penalties.  When read_i, read_d and read_c are all NULL,
   * every read base takes these Phred values (insertion open, deletion open,
   * gap continuation), and only bases and base qualities are copied to the
   * device: 2 bytes per read base instead of 5.  Biovoltron's SamRecord fills
   * its insertion/deletion GOP and GCP views from one constant string each
   * (include/biovoltron/file_io/sam.hpp:19-31, 451-475), so a caller holding
   * SamRecords passes those constants here.  Ignored when the per-base arrays
   * are given; giving some of them but not all three is an error. */
  uint8_t gap_ins;
  uint8_t gap_del;
  uint8_t gap_gcp;
  uint8_t reserved_[5];
} bv_region_batch;

/* Number of result slots the batch produces (sum over regions of reads*haps). */
int64_t bv_phmm_region_results(const bv_region_batch* batch);

/* Scores every pair of the batch into out_log10 (bv_phmm_region_results slots,
 * region by region, read-major).  An invalid batch returns BV_ERR_INVALID_ARG;
 * a batch scored in chunks (bv_phmm_options.pipeline_chunks) has each chunk's
 * reads and haplotypes validated as the chunk is staged, so out_log10 may then
 * hold the results of the chunks before the invalid one. */
bv_status bv_phmm_compute_regions(bv_phmm_ctx* ctx, const bv_region_batch* batch, double* out_log10,
                                  bv_phmm_stats* stats);

/* --- one batch over several GPUs (no counterpart in the reference, whose
 * AvxPairHMM parallelises over reads with OpenMP, pairhmm_avx.hpp:133-135) --
 * Regions are independent, so the batch is split with no exchange between
 * devices: its regions are cut into contiguous blocks of about equal DP cells
 * (sum over a block's regions of read bases x haplotype bases, at most 16
 * blocks per context) and the blocks are dealt to the contexts by greedy LPT
 * -- the largest block first, each to the context with the fewest cells so
 * far (lower index on ties).  Each context scores its blocks with
 * bv_phmm_compute_regions on views of the caller's arrays, one host thread
 * per context; results land in region order, as one context writes them.
 * The contexts must be distinct (one per GPU, or several on one GPU) and are
 * used with their own options: give them the same band options and weights.
 * Returns the first failing context's status. */
bv_status bv_phmm_compute_regions_multi(bv_phmm_ctx* const* ctxs, int32_t num_ctx, const bv_region_batch* batch,
                                        double* out_log10, bv_phmm_stats* stats);
/* The partition bv_phmm_compute_regions_multi uses, for num_parts devices and
 * at most num_blocks blocks (host only, no device): block b holds regions
 * [block_start[b], block_start[b+1]) (num_blocks+1 entries at most) and goes
 * to part block_part[b]; part_cells[p] is the cells part p gets.  Returns the
 * number of blocks, or -1 for an invalid batch or count.  Any output may be
 * NULL. */
int64_t bv_phmm_plan_partition(const bv_region_batch* batch, int32_t num_parts, int32_t num_blocks,
                               int64_t* block_start, int32_t* block_part, int64_t* part_cells);

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

/* --- learned band: training and weights ---------------------------------- */
/* Band MLP training, on this context's GPU.  Labels: for every pair of
 * `train` the full-DP forward-backward gives the posterior of each cell,
 * normalised per read row; the label is the lowest and highest diagonal
 * whose largest per-row posterior reaches `tau`, relative to the pair's
 * 11-mer seed diagonal.  Pairs without a seed or with reads longer than 511
 * bases are not used.  The MLP (80-128-128-2, ReLU, BF16 weights as the
 * inference kernel uses them) is trained with Adam on an asymmetric squared
 * loss that weights a band narrower than the label by `alpha`.  On success
 * the weights are installed (use_mlp may be set).  Replaces the previous
 * staged batch (stage again before bv_phmm_run).  No counterpart in the
 * reference. */
typedef struct bv_band_train_options {
  int32_t struct_size;  /* sizeof(bv_band_train_options) */
  int32_t epochs;
  int32_t batch;        /* pairs per Adam step */
  float lr;             /* peak learning rate (cosine decay to 0) */
  float alpha;          /* loss weight of under-covering errors */
  float tau;            /* posterior threshold of the label spread */
  float clip;           /* labels are clipped to [-clip, clip] diagonals */
  int32_t margin;       /* margin used for the coverage figures of the report */
  uint64_t seed;        /* weight initialisation and shuffling */
  int32_t reserved[4];
} bv_band_train_options;

typedef struct bv_band_train_report {
  int64_t pairs;          /* pairs in the training batch */
  int64_t labelled;       /* pairs with a seed and a label */
  int32_t steps;          /* Adam steps taken */
  float first_loss;       /* loss of the first and of the last epoch (mean over steps) */
  float last_loss;
  double cover_frac;      /* labelled pairs whose routed band (margin, 11-mer extent) covers the label */
  double band_frac;       /* labelled pairs whose routed band fits the banded kernel (<= 32 diagonals) */
  double ms_labels;       /* label kernel time */
  double ms_train;        /* training loop time */
} bv_band_train_report;

void bv_phmm_default_band_train_options(bv_band_train_options* opts);
bv_status bv_phmm_band_train(bv_phmm_ctx* ctx, const bv_region_batch* train, const bv_band_train_options* opts,
                             bv_band_train_report* report);
/* Labels and features of a batch, as training sees them (testing and
 * analysis): per result slot the seed diagonal (INT32_MIN: none), the label
 * spread lo/hi in absolute diagonals (INT32_MIN: none) and, for the pointers
 * that are not NULL, the 80 MLP inputs and the lowest / highest diagonal of a
 * shared 11-mer.  Replaces the staged batch. */
bv_status bv_phmm_band_labels(bv_phmm_ctx* ctx, const bv_region_batch* batch, float tau, int32_t* dstar, int32_t* lo,
                              int32_t* hi, float* features, int32_t* kmin, int32_t* kmax);
/* After bv_phmm_run_staged in band mode: per result slot the route taken
 * (0 banded, 1 full DP from the router, 2 banded then sent to the full DP by
 * the edge check, 3 banded then recomputed in FP64, 4 banded then scored
 * again by the full DP for lying far below its read's best) and, for routes
 * 0, 2, 3 and 4, the band's first diagonal and width.  For testing and
 * analysis. */
bv_status bv_phmm_band_routes(bv_phmm_ctx* ctx, int64_t n, int32_t* d_lo, int32_t* width, int32_t* route);
/* Number of FP32 MLP parameters: W1[128][80], b1[128], W2[128][128], b2[128],
 * W3[2][128], b3[2], weights as [output][input], in that order. */
int64_t bv_phmm_band_param_count(void);
bv_status bv_phmm_band_get_weights(bv_phmm_ctx* ctx, float* w, int64_t n);
bv_status bv_phmm_band_set_weights(bv_phmm_ctx* ctx, const float* w, int64_t n);
/* Weight file: 8-byte magic "BVBANDW\0", u32 version (1), u32 80, u32 128,
 * u32 2, u32 parameter count, FP32 parameters (little endian). */
bv_status bv_phmm_band_save(bv_phmm_ctx* ctx, const char* path);
bv_status bv_phmm_band_load(bv_phmm_ctx* ctx, const char* path);
/* One evaluation of the training objective on the GPU with the given FP32
 * weights (rounded to BF16 as in training): outputs [n][2], the loss and, if
 * `grad` is not NULL, its gradient (bv_phmm_band_param_count floats).  x is
 * [n][80], targets [n][2].  For gradient checks. */
bv_status bv_phmm_band_mlp_eval(bv_phmm_ctx* ctx, const float* w, const float* x, const float* targets, int64_t n,
                                float alpha, float* out, float* loss, float* grad);
/* The band pipeline's MLP inference kernel (tcgen05 tensor cores) on x
 * ([n][80], rounded to BF16 as the featuriser stores them) with the installed
 * weights: out [n][2].  For checks against the objective's forward pass. */
bv_status bv_phmm_band_mlp_infer(bv_phmm_ctx* ctx, const float* x, int64_t n, float* out);

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
 * and returns after the stream has finished it, so it cannot be captured into
 * a CUDA graph: a call on a capturing stream returns BV_ERR_UNSUPPORTED
 * before enqueuing anything (the capture stays valid).  The first call on a device
 * sets that device up (finds the scratch array's device address, copies the
 * probability tables into it, synchronously): make it before any stream
 * capture.  Under lazy module loading (the CUDA default since 12.2) that
 * first call is also when the driver loads this library's device code on the
 * device and reserves the 4.6 MB array: make it at start-up, before the
 * framework's allocator reserves its memory, or set CUDA_MODULE_LOADING=EAGER.
 * Later calls reserve no device memory.  All calls share the one scratch array and it keeps the last
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

/* --- autotuning ------------------------------------------------------------
 * The full-DP kernels run one launch per bin of reads with the same rows per
 * lane (ceil((read_len + 3) / 32), 1..8; longer reads use the multi-strip
 * kernel).  Per bin a warp scores one or two haplotypes of a read at a time
 * (haps_per_warp) and a block holds 1..4 warps (warps_per_block).
 * bv_phmm_autotune times every combination on `sample` (repeats timed runs
 * each, device time per bin launch), installs the fastest per bin in the
 * context and writes one entry per bin the sample exercises (at most 8).
 * No counterpart in the reference (its AVX kernels have no launch shape). */
typedef struct bv_phmm_tune_entry {
  int32_t rows_per_lane;    /* bin: 1..8 */
  int32_t haps_per_warp;    /* 1 or 2 */
  int32_t warps_per_block;  /* 1..4 */
  int32_t reserved;
  double ms;                /* the bin's best time on the sample (autotune output) */
} bv_phmm_tune_entry;

bv_status bv_phmm_autotune(bv_phmm_ctx* ctx, const bv_region_batch* sample, int32_t repeats, bv_phmm_tune_entry* out,
                           int32_t* num_out);
/* Installs (set) or reads (get) per-bin launch parameters; entries for bins
 * not listed keep their values (defaults: two haplotypes per warp, 4 warps). */
bv_status bv_phmm_set_tuning(bv_phmm_ctx* ctx, const bv_phmm_tune_entry* entries, int32_t num);
bv_status bv_phmm_get_tuning(bv_phmm_ctx* ctx, bv_phmm_tune_entry* out, int32_t* num_out);
/* The FP64 long-read kernel: a block of `warps` warps per pair (2, 4 or 8;
 * default 4) runs reads of at least 128 x warps bases, strip w of every
 * group of `warps` strips on warp w.  bv_phmm_autotune_long stages `sample`
 * in FP64 mode for each choice (the long-read edge moves with it), times the
 * FP64 pass (`repeats` runs, median), installs the fastest and writes it to
 * *warps_out and the times to ms_out[0..2] (2, 4, 8 warps; 0 where the
 * sample has no read that long).  No counterpart in the reference. */
bv_status bv_phmm_set_long_warps(bv_phmm_ctx* ctx, int32_t warps);
int32_t bv_phmm_get_long_warps(const bv_phmm_ctx* ctx);
bv_status bv_phmm_autotune_long(bv_phmm_ctx* ctx, const bv_region_batch* sample, int32_t repeats, int32_t* warps_out,
                                double* ms_out);

/* --- the scalar PairHMM model ----------------------------------------------
 * Replaces PairHMM::compute_likelihoods(haplotypes, reads, trans)
 * (include/biovoltron/algo/align/inexact_match/pairhmm.hpp:116-141; the model
 * :56-80): every row uses the same seven transition probabilities, in
 * PairHMM::TrasMatrx order {M->M, M->I, M->D, I->M, I->I, D->M, D->D}
 * (ORIGINAL_DEFAULT = {0.9998, 1e-4, 1e-4, 0.9, 0.1, 0.9, 0.1}, :32-33), and the
 * emission prior comes from the base quality byte (& 127) alone: the insertion,
 * deletion and gap-continuation arrays of a batch are not read (they must still
 * be valid pointers).  Bases compare as A/C/G/T with N matching everything (the
 * scalar model compares raw bytes: equal for upper-case ACGTN input).  NULL
 * goes back to the quality-derived transitions.  The band path needs the
 * quality-derived ones (BV_ERR_UNSUPPORTED while the band is on).  Values
 * outside [0, 1]: BV_ERR_INVALID_ARG. */
bv_status bv_phmm_set_transitions(bv_phmm_ctx* ctx, const double* trans7);
/* 1 and the seven values when constant transitions are set, else 0. */
int bv_phmm_get_transitions(const bv_phmm_ctx* ctx, double* trans7);

/* --- genotyping on the device -------------------------------------------
 * After bv_phmm_run_staged, runs on the staged batch's [read][hap] log10
 * matrix (it stays on the device) what HaplotypeCaller does with each
 * region's matrix next: PairHMM::normalize_likelihoods and
 * filter_poorly_modeled_reads (pairhmm.hpp:83-114), the genotyper's read
 * selection by site overlap, Genotyper::marginal_likelihoods and the diploid
 * genotype likelihoods with MathUtils::approximate_log10_sum_log10
 * (genotyper.hpp:223-240, 254-326; math_utils.hpp:112-139).  Results equal
 * the reference's bit for bit.  `staged` is the batch that was staged (its
 * region and read structure is read again).  Outputs, per region g with nr_g
 * reads, nh_g haplotypes and A_g alleles, in region order:
 *   kept_count[g]                     reads kept (filter and overlap);
 *   kept_reads[first read of g + k]   their batch read indices, k < kept;
 *   allele_lik[sum of nr * A before g + k * A_g + a]  max over the region's
 *                                     haplotypes of allele a (normalised);
 *   genotype_lik[sum of A (A + 1) / 2 before g + i]  genotype i = (a1, a2),
 *                                     a1 <= a2, in the reference's order.
 * Slots beyond kept_count are left unwritten. */
typedef struct bv_genotype_batch {
  const int32_t* allele_count;  /* [num_regions]: alleles at the region's site, 1..64 */
  const int32_t* hap_allele;    /* [num_haps]: allele (0..A-1) each haplotype carries; others are ignored */
  const uint8_t* read_overlaps; /* [num_reads]: nonzero when the read overlaps its region's site */
} bv_genotype_batch;

bv_status bv_phmm_genotype_staged(bv_phmm_ctx* ctx, const bv_region_batch* staged, const bv_genotype_batch* gt,
                                  int32_t* kept_count, int32_t* kept_reads, double* allele_lik,
                                  double* genotype_lik, double* kernel_ms);

/* Diagnostics: writes the probability tables a context uploads (ph2pr for
 * quals 0..127 and the match-to-match triangle for quals <= 127, both
 * precisions; Context.h:42-175).  Host-only, needs no device.  Returns 0, or
 * -1 if mm_entries is not 127*128/2 + 128. */
int bv_phmm_debug_tables(float* ph2pr_f32, double* ph2pr_f64, float* mm_f32, double* mm_f64, int mm_entries);

/* Diagnostics: the region chunks bv_phmm_compute_regions would use for
 * `chunks` chunks: writes up to `max` (first region, end region, first result,
 * results) quadruples and returns the number of chunks.  Host-only. */
int64_t bv_phmm_debug_chunks(const bv_region_batch* batch, int32_t chunks, int64_t* out, int64_t max);

/* Diagnostics: writes up to n entries of the genotyper's Jacobian log table
 * (math_utils.hpp:122-139) as this library builds it; returns the table size.
 * Host-only. */
int bv_phmm_debug_jacobian_table(double* out, int n);

/* Diagnostics: measures the device's achievable FP32 FMA throughput (TFLOP/s,
 * 2 flops per FMA), the roofline denominator of the forward kernels, which
 * run on the CUDA-core FP32 pipe.  Returns a bv_status. */
int bv_phmm_measure_fp32_peak(int device, double* tflops);
/* The same for FP64 FMAs: the roofline denominator of the FP64 rescue kernel. */
int bv_phmm_measure_fp64_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* BV_PAIRHMM_H */
