// phmm_labels.cu -- training labels for the band MLP: the posterior spread of
// each pair's alignment over diagonals, from the full-DP forward-backward.
//
// For row r the posterior of cell (r, c) is p_r(c) ~ sum_s F_s(r,c) B_s(r,c)
// (s = M, X, Y), normalised to 1 over the row; pstar(d) = max_r p_r(d + r).
// The label is the lowest and highest diagonal d with pstar(d) >= tau.
// Recurrences are the reference's (avx-pairhmm-template.h:183-198) and their
// adjoint:
//   B_M(r,c) = mm(r+1) e(r+1,c+1) B_M(r+1,c+1) + mx(r+1) B_X(r+1,c) + my(r) B_Y(r,c+1) + [r==R]
//   B_X(r,c) = gp(r+1) e(r+1,c+1) B_M(r+1,c+1) + g(r+1) B_X(r+1,c) + [r==R]
//   B_Y(r,c) = gp(r+1) e(r+1,c+1) B_M(r+1,c+1) + g(r) B_Y(r,c+1)
//
// One warp per pair; lane l owns columns [l*C + 1, (l+1)*C] of a row.  M and X
// of a row depend only on the previous row (kept in shared memory); the
// in-row Y recurrence is affine with a per-row constant (Y(c) = g Y(c-1) +
// t(c)), solved by a warp scan over the lanes' chunks.  Every row is
// renormalised by a power of two; the per-row normalisation of p_r makes the
// scales cancel.  Forward rows go to a per-warp global buffer that the
// backward reads back.
#include <cuda_runtime.h>

#include <cstdint>

#include "phmm_band.h"
#include "phmm_common.h"
#include "phmm_kernels.h"

namespace bvphmm {
namespace {

constexpr int kLabelMaxH = kBandMaxHap;   // columns per pair
constexpr int kLabelWarps = 4;
constexpr int kLabelCols = kLabelMaxH + 2;

__device__ __forceinline__ uint32_t code_of(uint8_t b) {
  return b == 'C' ? 1u : b == 'T' ? 2u : b == 'G' ? 3u : b == 'N' ? 4u : 0u;
}

struct RowC {
  float mm, gp, mx, my, g, em, ex;
  uint32_t rc;
};

__device__ __forceinline__ RowC row_consts(const Tables* tb, const uchar4* quals, const uint8_t* bases, int r) {
  RowC k;
  const uchar4 q = quals[r - 1];
  const int qi = q.y & kQualMask, qd = q.z & kQualMask;
  const int mx = max(qi, qd), mn = min(qi, qd);
  k.mm = tb->mm_f[((mx * (mx + 1)) >> 1) + mn];
  k.g = tb->ph2pr_f[q.w & kQualMask];
  k.gp = 1.f - k.g;
  k.mx = tb->ph2pr_f[qi];
  k.my = tb->ph2pr_f[qd];
  const float eps = tb->ph2pr_f[q.x & kQualMask];
  k.em = 1.f - eps;
  k.ex = eps / 3.f;
  k.rc = code_of(bases[r - 1]);
  return k;
}

__device__ __forceinline__ float emis(const RowC& k, uint32_t hc) {
  return (k.rc == hc || k.rc == 4u || hc == 4u) ? k.em : k.ex;
}

// Inclusive warp scan of affine maps y -> a*y + b (lane order = left to right
// when `forward`, right to left otherwise).  Returns the map composed over
// the lanes before this one applied to 0, i.e. the carry-in.
__device__ __forceinline__ float affine_carry(float a, float b, int lane, bool forward) {
  for (int o = 1; o < 32; o <<= 1) {
    const float ao = forward ? __shfl_up_sync(0xffffffffu, a, o) : __shfl_down_sync(0xffffffffu, a, o);
    const float bo = forward ? __shfl_up_sync(0xffffffffu, b, o) : __shfl_down_sync(0xffffffffu, b, o);
    const bool has = forward ? lane >= o : lane + o < 32;
    if (has) { b = a * bo + b; a = a * ao; }
  }
  const float prev = forward ? __shfl_up_sync(0xffffffffu, b, 1) : __shfl_down_sync(0xffffffffu, b, 1);
  return (forward ? lane == 0 : lane == 31) ? 0.f : prev;
}

__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kLabelWarps * 32) k_posterior_spread(DeviceBatch b, const Tables* tb,
                                                                      const int32_t* pair_read, const int32_t* pair_hap,
                                                                      long long n_pairs, float tau, float* fbuf,
                                                                      long long fbuf_stride, int32_t* lo_out,
                                                                      int32_t* hi_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float* prevM = reinterpret_cast<float*>(smem) + (size_t)wib * (6 * kLabelCols + kBandMaxSpan);
  float* prevX = prevM + kLabelCols;
  float* prevY = prevX + kLabelCols;
  float* curM = prevY + kLabelCols;
  float* curX = curM + kLabelCols;
  float* curY = curX + kLabelCols;
  float* pstar = curY + kLabelCols;
  uint8_t* hcode = reinterpret_cast<uint8_t*>(reinterpret_cast<float*>(smem) + (size_t)kLabelWarps * (6 * kLabelCols + kBandMaxSpan)) +
                   (size_t)wib * kLabelCols;
  const long long warp = blockIdx.x * (long long)kLabelWarps + wib;
  float* F = fbuf + warp * fbuf_stride;
  for (long long pi = warp; pi < n_pairs; pi += (long long)gridDim.x * kLabelWarps) {
    const int r_idx = pair_read[pi], h_idx = pair_hap[pi];
    const int64_t ro = b.read_off[r_idx], ho = b.hap_off[h_idx];
    const int R = (int)(b.read_off[r_idx + 1] - ro), H = (int)(b.hap_off[h_idx + 1] - ho);
    if (R < 1 || H < 1 || H > kLabelMaxH || R + H >= kBandMaxSpan ||
        (long long)(R + 1) * 3 * (H + 2) > fbuf_stride) {
      if (lane == 0) { lo_out[pi] = INT32_MIN; hi_out[pi] = INT32_MIN; }
      continue;
    }
    const uchar4* quals = b.read_quals + ro;
    const uint8_t* bases = b.read_bases + ro;
    const int C = (H + 31) / 32;
    const int c0 = lane * C + 1, c1 = min(c0 + C - 1, H);  // this lane's columns (may be empty)
    __syncwarp();
    for (int c = lane; c < H; c += 32) hcode[c + 1] = (uint8_t)code_of(b.hap_bases[ho + c]);
    for (int x = lane; x < R + H; x += 32) pstar[x] = 0.f;
    for (int c = lane; c <= H + 1; c += 32) { prevM[c] = 0.f; prevX[c] = 0.f; prevY[c] = 1.f; curM[c] = 0.f; curX[c] = 0.f; curY[c] = 0.f; }
    __syncwarp();
    // ---- forward, rows 1..R; row r stored at F[r * 3 * (H+2) + {0, H+2, 2(H+2)} + c]
    const int stride = H + 2;
    for (int r = 1; r <= R; ++r) {
      const RowC k = row_consts(tb, quals, bases, r);
      // M, X from the previous row; the Y pass with its carry-in follows
      for (int c = c0; c <= c1; ++c) {
        const float e = emis(k, hcode[c]);
        curM[c] = e * (k.mm * prevM[c - 1] + k.gp * (prevX[c - 1] + prevY[c - 1]));
        curX[c] = k.mx * prevM[c] + k.g * prevX[c];
      }
      __syncwarp();
      // Y(c) = g Y(c-1) + my M(c-1): affine along the row
      const float mleft = (c0 <= H && c0 > 1) ? curM[c0 - 1] : 0.f;
      float a = 1.f, bb = 0.f;
      {
        float y = 0.f, m = mleft;
        for (int c = c0; c <= c1; ++c) { y = k.g * y + k.my * m; m = curM[c]; a *= k.g; }
        bb = y;
      }
      if (c0 > c1) { a = 1.f; bb = 0.f; }
      const float carry = affine_carry(a, bb, lane, true);
      {
        float y = carry, m = mleft;
        for (int c = c0; c <= c1; ++c) { y = k.g * y + k.my * m; curY[c] = y; m = curM[c]; }
      }
      __syncwarp();
      float mx = 0.f;
      for (int c = c0; c <= c1; ++c) mx = fmaxf(mx, fmaxf(curM[c], fmaxf(curX[c], curY[c])));
      mx = warp_max(mx);
      const float sc = mx > 0.f ? ldexpf(1.f, -ilogbf(mx)) : 1.f;
      float* Fr = F + (size_t)r * 3 * stride;
      for (int c = lane; c <= H; c += 32) {
        const float m = c == 0 ? 0.f : curM[c] * sc, x = c == 0 ? 0.f : curX[c] * sc, y = c == 0 ? 0.f : curY[c] * sc;
        prevM[c] = m; prevX[c] = x; prevY[c] = y;
        Fr[c] = m; Fr[stride + c] = x; Fr[2 * stride + c] = y;
      }
      __syncwarp();
    }
    // ---- backward, rows R..1, B of row r+1 in prev*, posterior per row
    for (int c = lane; c <= H + 1; c += 32) { prevM[c] = 0.f; prevX[c] = 0.f; prevY[c] = 0.f; }
    __syncwarp();
    RowC k1{};  // constants of row r+1
    for (int r = R; r >= 1; --r) {
      const RowC k0 = row_consts(tb, quals, bases, r);
      // B_Y(c) = g(r) B_Y(c+1) + t(c), right to left, t(c) = gp(r+1) e(r+1,c+1) B_M(r+1,c+1)
      float a = 1.f, bb = 0.f;
      auto tval = [&](int c) -> float {
        if (r == R || c + 1 > H) return 0.f;
        return k1.gp * emis(k1, hcode[c + 1]) * prevM[c + 1];
      };
      {
        float y = 0.f;
        for (int c = c1; c >= c0; --c) { y = k0.g * y + tval(c); a *= k0.g; }
        bb = y;
      }
      if (c0 > c1) { a = 1.f; bb = 0.f; }
      const float carry = affine_carry(a, bb, lane, false);
      {
        float y = carry;  // B_Y(r, c+1)
        for (int c = c1; c >= c0; --c) {
          const float byr = y;
          y = k0.g * y + tval(c);
          curY[c] = y;
          if (r == R) {
            curM[c] = 1.f;
            curX[c] = 1.f;
          } else {
            const float nm = (c + 1 <= H) ? emis(k1, hcode[c + 1]) * prevM[c + 1] : 0.f;
            curM[c] = k1.mm * nm + k1.mx * prevX[c] + k0.my * byr;
            curX[c] = k1.gp * nm + k1.g * prevX[c];
          }
        }
      }
      __syncwarp();
      // posterior of row r
      const float* Fr = F + (size_t)r * 3 * stride;
      float tot = 0.f;
      for (int c = c0; c <= c1; ++c) tot += Fr[c] * curM[c] + Fr[stride + c] * curX[c] + Fr[2 * stride + c] * curY[c];
      tot = warp_sum(tot);
      if (tot > 0.f) {
        const float inv = 1.f / tot;
        for (int c = c0; c <= c1; ++c) {
          const float pr = (Fr[c] * curM[c] + Fr[stride + c] * curX[c] + Fr[2 * stride + c] * curY[c]) * inv;
          const int d = c - r + (R - 1);  // index into pstar, d in [1-R, H-1]
          pstar[d] = fmaxf(pstar[d], pr);   // each (r, c) is owned by one lane: no race within a row
        }
      }
      float mx = 0.f;
      for (int c = c0; c <= c1; ++c) mx = fmaxf(mx, fmaxf(curM[c], fmaxf(curX[c], curY[c])));
      mx = warp_max(mx);
      const float sc = mx > 0.f ? ldexpf(1.f, -ilogbf(mx)) : 1.f;
      __syncwarp();
      for (int c = lane; c <= H + 1; c += 32) {
        prevM[c] = (c >= 1 && c <= H) ? curM[c] * sc : 0.f;
        prevX[c] = (c >= 1 && c <= H) ? curX[c] * sc : 0.f;
        prevY[c] = (c >= 1 && c <= H) ? curY[c] * sc : 0.f;
      }
      k1 = k0;
      __syncwarp();
    }
    // spread: lowest and highest diagonal with pstar >= tau
    int lo = INT32_MAX, hi = INT32_MIN;
    for (int x = lane; x < R + H - 1; x += 32)
      if (pstar[x] >= tau) { lo = min(lo, x - (R - 1)); hi = max(hi, x - (R - 1)); }
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) { lo_out[pi] = lo == INT32_MAX ? INT32_MIN : lo; hi_out[pi] = hi; }
    __syncwarp();
  }
}

}  // namespace

int label_smem_bytes() {
  return kLabelWarps * ((6 * kLabelCols + kBandMaxSpan) * 4 + kLabelCols);
}

int label_warps_per_block() { return kLabelWarps; }

cudaError_t launch_posterior_spread(const DeviceBatch& b, const Tables* tb, const int32_t* pair_read,
                                    const int32_t* pair_hap, long long n_pairs, float tau, float* fbuf,
                                    long long fbuf_stride, int32_t* lo, int32_t* hi, int blocks, cudaStream_t st) {
  if (n_pairs <= 0) return cudaSuccess;
  const int smem = label_smem_bytes();
  cudaError_t e = raise_dynamic_smem(reinterpret_cast<const void*>(&k_posterior_spread), smem);
  if (e != cudaSuccess) return e;
  k_posterior_spread<<<blocks, kLabelWarps * 32, smem, st>>>(b, tb, pair_read, pair_hap, n_pairs, tau, fbuf,
                                                             fbuf_stride, lo, hi);
  return cudaGetLastError();
}

}  // namespace bvphmm
