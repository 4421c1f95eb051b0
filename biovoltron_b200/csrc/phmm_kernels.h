// phmm_kernels.h -- launch interface between the host engine and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "phmm_common.h"

namespace bvphmm {

constexpr int kThreadsPerBlock = 128;

struct KernelParams {
  DeviceBatch batch;
  const Tables* tables;
  const Unit* units;
  long long unit_base;
  long long n_units;
  const unsigned long long* n_units_dev;  // if set, the unit count is read from device memory
  int slot;               // work-queue head used by this launch
  int from_rescue;        // 1: items come from the FP64 list
  Counters* ctr;
  double* out;            // log10 likelihoods, one per result slot
  PairRef* rescue;        // null: pairs below the FP32 threshold get NaN (audit runs)
  long long rescue_cap;
  int warps_per_block;    // block size of the launch / 32 (1..4)
  int hap_bytes;          // per-warp bytes for staged haplotype codes
  int code_row_bytes;     // entries of a staged code row (paired variants stage 4-byte entries)
  int warp_smem_bytes;    // per-warp dynamic shared memory
  void* bnd;              // per-warp strip-boundary buffers (multi-strip variants)
  long long bnd_cols;     // rows of 4 values per warp buffer
  int rescale;            // renormalise between strips (FP64 variants)
  int rescale_target;     // binary exponent the boundary maximum is scaled to
  unsigned long long* cells_ctr;  // if set, FP64 launches add read x haplotype length per pair here
  int long_rows;          // > 0: FP32 results of reads this long or longer go to the FP64 list's long part
};

// Long reads in FP64: a block of `warps` warps per pair (phmm_long.cu; 2, 4
// or 8, kLongWarps by default, chosen per context by the long-read tuner);
// reads of at least warps x 128 bases (as many strips of 128 rows as the
// block has warps) take it.
constexpr int kLongWarps = 4;
constexpr int kLongRows = kLongWarps * 128;
bool long_warps_valid(int warps);
int long_smem_bytes(int hap_bytes, int warps);
cudaError_t prepare_long(int smem, int warps);
int long_blocks_per_sm(int smem, int warps);
cudaError_t launch_forward_long(const KernelParams& p, int grid, int smem, int warps, cudaStream_t st);

// Variant table: (precision, rows per lane, multi-strip, two haplotypes per
// warp).  Paired variants exist for FP32 single strip only.
int variant_index(bool f64, int rows_per_lane, bool multi, bool paired = false);
bool variant_paired(int variant);
int warp_smem_bytes(int variant, int hap_bytes);
int blocks_per_sm(int variant, int smem_per_block, int threads = kThreadsPerBlock);
// Raises (never lowers) a kernel's dynamic shared-memory limit on the current
// device to at least `bytes`; safe to call from several host threads.
cudaError_t raise_dynamic_smem(const void* func, int bytes);
// Sets the variant's dynamic shared-memory limit; call before launching or capturing it.
cudaError_t prepare_variant(int variant, int smem_per_block);
cudaError_t launch_forward(int variant, const KernelParams& p, int grid, cudaStream_t st);
cudaError_t launch_pack_quals(const uint8_t* q, const uint8_t* i, const uint8_t* d, const uint8_t* c, uchar4* out,
                              long long n, int sms, cudaStream_t st);
// The same with the insertion, deletion and continuation qualities constant.
cudaError_t launch_pack_quals_uniform(const uint8_t* q, uint8_t gi, uint8_t gd, uint8_t gc, uchar4* out, long long n,
                                      int sms, cudaStream_t st);

// Writes one 64-bit value on the device (graph-capturable).
cudaError_t launch_set_u64(unsigned long long* dst, unsigned long long v, cudaStream_t st);

// Host-side construction of the reference's probability tables (Context.h).
void build_tables(Tables* t);
// Constant transitions for every row (7 entries, PairHMM::TrasMatrx order), or
// back to the quality-derived ones (nullptr).
void set_constant_transitions(Tables* t, const double* trans);

}  // namespace bvphmm
