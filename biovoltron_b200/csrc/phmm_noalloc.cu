// phmm_noalloc.cu -- an FP64 forward-pass entry point that allocates nothing.
//
// Why it exists.  Some callers cannot call cudaMalloc at the moment they
// need likelihoods: a haplotype caller embedded in a GPU pipeline whose
// device memory is owned by the host framework's caching allocator (the
// framework holds nearly all of HBM, so a stray cudaMalloc fails or forces a
// device-wide synchronisation), or code running under a policy that forbids
// new device allocations after start-up.  Such callers already hold their
// reads, haplotypes and output in device memory and want the scores written
// into that memory without the library reserving anything.
//
// How.  bv_phmm_forward_f64_noalloc runs a variant of the FP64 multi-strip
// forward kernel (k_forward<double, 4, multi-strip>, phmm_forward.cu): the
// scratch that kernel normally takes from context-owned allocations -- the
// work-queue counters, the probability tables and one strip-boundary buffer
// per resident warp -- lives here in one file-scope __device__ array of fixed
// size (kScratchBytes, about 4.6 MB).  Every GPU that loads this library holds
// that array until the process exits.  Consequences, all documented in
// include/bv_pairhmm.h:
//   * haplotypes are limited to BV_PHMM_NOALLOC_MAX_HAP_LEN bases (the
//     boundary buffers are sized for it); reads may be of any length;
//   * the kernel runs on a fixed grid of kWarps warps, so it is slower than
//     the allocating path;
//   * every call shares the array and it keeps the last call's contents:
//     the counters are cleared by a small kernel at the start of each call,
//     each warp clears its boundary buffer before each pair, and calls that
//     overlap on the GPU (two host threads, or two streams) race on it;
//   * the first call on a device sets that device up (looks up the array's
//     device address with cudaGetSymbolAddress and copies the tables into
//     it, synchronously); make that first call before any stream capture.
//     With lazy module loading (the CUDA default since 12.2) that first call
//     is also when the driver loads this library's device code on the device
//     and reserves the array, so a caller whose framework will later take
//     nearly all of HBM makes its first call at start-up, before the
//     framework's allocator reserves memory (or runs with
//     CUDA_MODULE_LOADING=EAGER, which loads every module when the context is
//     created).  After that first call, calls reserve no device memory.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "bv_pairhmm.h"
#include "phmm_common.h"
#include "phmm_device.cuh"
#include "phmm_kernels.h"

namespace bvphmm {
namespace {

constexpr int kWarps = 64;
constexpr int kBlocks = kWarps / (kThreadsPerBlock / kWarp);
constexpr int kRT = 4;
constexpr int kMaxHap = BV_PHMM_NOALLOC_MAX_HAP_LEN;
// boundary columns per warp: the haplotype rounded up to the warp, plus 128 of
// headroom; the kernel's largest index is nsteps + 96 (2,176 at 2,048 bases),
// below these 2,208 (the allocating path keeps 160 columns of headroom)
constexpr long long kBndCols = ((kMaxHap + kWarp - 1 + 31) / 32) * 32 + 128;
constexpr int kHapBytes = ((kMaxHap + (kWarp - 1) + 32 + kHapLead + 16 + 15) / 16) * 16;
constexpr size_t kCountersBytes = 512;
constexpr size_t kTablesBytes = (sizeof(Tables) + 255) / 256 * 256;
constexpr size_t kBndBytes = (size_t)kWarps * kBndCols * 4 * sizeof(double);
constexpr size_t kScratchBytes = kCountersBytes + kTablesBytes + kBndBytes;
static_assert(sizeof(Counters) <= kCountersBytes, "counters do not fit");
// The launch sets no dynamic shared-memory attribute, so a block must stay
// within the 48 KB every kernel may use without one.
static_assert((size_t)(kHapBytes + WarpSmem<double, kRT>::kEtabBytes + WarpSmem<double, kRT>::kRingBytes) *
                      (kThreadsPerBlock / kWarp) <= 48 * 1024,
              "no-allocation kernel needs more than 48 KB of shared memory per block");
constexpr int kMaxDevices = 64;

// The scratch.  Host code only ever uses the address cudaGetSymbolAddress
// returns for the current device; the name itself is a host-side stand-in.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct DeviceSetup {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_scratch on that device
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mu;
Tables g_host_tables;  // static storage: building it allocates nothing
unsigned long long g_status_host[kMaxDevices];

__global__ void k_noalloc_reset(Counters* c) {
  if (threadIdx.x == 0) {
    for (int k = 0; k < (int)(sizeof(c->unit_next) / sizeof(c->unit_next[0])); ++k) c->unit_next[k] = 0;
    c->rescue_count = 0;
    c->rescue_next = 0;
    c->underflow_count = 0;
    c->status = 0;
  }
}

// Each warp takes pairs from the list; a pair whose indices or haplotype
// length fall outside the bounds the scratch was sized for is skipped, its
// output (when addressable) set to NaN and the status flagged.
__global__ void __launch_bounds__(kThreadsPerBlock) k_forward_f64_noalloc(KernelParams p, long long n_pairs,
                                                                          long long n_reads, long long n_haps,
                                                                          long long n_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & (kWarp - 1);
  const int wib = threadIdx.x >> 5;
  const int warp_global = blockIdx.x * (kThreadsPerBlock / kWarp) + wib;
  unsigned char* wsm = smem + (size_t)wib * p.warp_smem_bytes;
  double* bnd = reinterpret_cast<double*>(p.bnd) + (size_t)warp_global * p.bnd_cols * 4;
  for (;;) {
    unsigned long long w = 0;
    if (lane == 0) w = atomicAdd(&p.ctr->rescue_next, 1ull);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= (unsigned long long)n_pairs) break;
    const PairRef pr = p.rescue[w];
    bool ok = pr.read >= 0 && pr.read < n_reads && pr.hap >= 0 && pr.hap < n_haps && pr.out >= 0 && pr.out < n_out;
    if (ok) {
      const long long H = p.batch.hap_off[pr.hap + 1] - p.batch.hap_off[pr.hap];
      const long long R = p.batch.read_off[pr.read + 1] - p.batch.read_off[pr.read];
      ok = H >= 0 && H <= kMaxHap && R >= 0;
    }
    if (!ok) {
      if (lane == 0) {
        atomicOr(&p.ctr->status, 2ull);
        if (pr.out >= 0 && pr.out < n_out) p.out[pr.out] = __longlong_as_double(0x7ff8000000000000ll);
      }
      continue;
    }
    Item it;
    it.read = pr.read;
    it.hap0 = pr.hap;
    it.nh = 1;
    it.out0 = pr.out;
    process_item<double, kRT, true>(p, it, wsm, lane, bnd);
  }
}

bv_status setup_device(int device, unsigned char** scratch) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  DeviceSetup& d = g_setup[device];
  if (!d.ready) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_scratch) != cudaSuccess || !ptr) return BV_ERR_CUDA;
    build_tables(&g_host_tables);
    if (cudaMemcpy(static_cast<unsigned char*>(ptr) + kCountersBytes, &g_host_tables, sizeof(Tables),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return BV_ERR_CUDA;
    d.scratch = static_cast<unsigned char*>(ptr);
    d.ready = true;
  }
  *scratch = d.scratch;
  return BV_OK;
}

}  // namespace
}  // namespace bvphmm

extern "C" bv_status bv_phmm_forward_f64_noalloc(int device, const bv_phmm_device_pairs* in, double* out_log10,
                                                 int64_t num_out, void* stream) {
  using namespace bvphmm;
  if (!in || device < 0 || device >= kMaxDevices || num_out < 0) return BV_ERR_INVALID_ARG;
  if (in->num_pairs < 0 || in->num_reads < 0 || in->num_haps < 0) return BV_ERR_INVALID_ARG;
  if (in->max_hap_len < 0 || in->max_hap_len > BV_PHMM_NOALLOC_MAX_HAP_LEN) return BV_ERR_INVALID_ARG;
  if (in->num_pairs == 0) return BV_OK;
  if (!in->pairs || !out_log10 || !in->read_offsets || !in->hap_offsets || !in->read_bases || !in->read_quals ||
      !in->hap_bases)
    return BV_ERR_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(in->pairs) & 7) || (reinterpret_cast<uintptr_t>(in->read_quals) & 3) ||
      (reinterpret_cast<uintptr_t>(in->read_offsets) & 7) || (reinterpret_cast<uintptr_t>(in->hap_offsets) & 7) ||
      (reinterpret_cast<uintptr_t>(out_log10) & 7))
    return BV_ERR_INVALID_ARG;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return BV_ERR_NO_DEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return BV_ERR_NO_DEVICE;
  // every call reads its status back and waits for the stream, which a stream
  // capture forbids: a capturing stream is refused before anything is enqueued
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cs) != cudaSuccess) {
    cudaGetLastError();
    cudaSetDevice(prev);
    return BV_ERR_UNSUPPORTED;
  }
  if (cs != cudaStreamCaptureStatusNone) {
    cudaSetDevice(prev);
    return BV_ERR_UNSUPPORTED;
  }
  unsigned char* scratch = nullptr;
  bv_status s = setup_device(device, &scratch);
  if (s == BV_OK) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    KernelParams p{};
    p.batch.read_bases = in->read_bases;
    p.batch.read_quals = reinterpret_cast<const uchar4*>(in->read_quals);
    p.batch.read_off = in->read_offsets;
    p.batch.hap_bases = in->hap_bases;
    p.batch.hap_off = in->hap_offsets;
    p.tables = reinterpret_cast<const Tables*>(scratch + kCountersBytes);
    p.ctr = reinterpret_cast<Counters*>(scratch);
    p.out = out_log10;
    p.rescue = const_cast<PairRef*>(static_cast<const PairRef*>(in->pairs));
    p.rescue_cap = in->num_pairs;
    p.from_rescue = 1;
    p.hap_bytes = kHapBytes;
    p.warp_smem_bytes = kHapBytes + WarpSmem<double, kRT>::kEtabBytes + WarpSmem<double, kRT>::kRingBytes;
    p.bnd = scratch + kCountersBytes + kTablesBytes;
    p.bnd_cols = kBndCols;
    p.rescale = 1;
    p.rescale_target = 1000;
    const int smem_block = p.warp_smem_bytes * (kThreadsPerBlock / kWarp);
    k_noalloc_reset<<<1, 32, 0, st>>>(p.ctr);
    k_forward_f64_noalloc<<<kBlocks, kThreadsPerBlock, smem_block, st>>>(p, in->num_pairs, in->num_reads,
                                                                         in->num_haps, num_out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&g_status_host[device], &p.ctr->status, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) s = BV_ERR_CUDA;
    else if (g_status_host[device] != 0) s = BV_ERR_INVALID_ARG;
  }
  cudaSetDevice(prev);
  return s;
}
