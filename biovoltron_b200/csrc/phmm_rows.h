// phmm_rows.h -- the padded row space of one pair, shared by host and device.
#pragma once

namespace bvphmm {

// Rows a pair occupies in the wavefront: row 0 (the initial row), the read's
// rows, for FP32 the summing row below the last read row, and for the
// single-strip FP32 kernel one padding row on top (see phmm_device.cuh).
#if defined(__CUDACC__)
__host__ __device__
#endif
constexpr int rows_needed(int read_len, bool f32, bool single_strip) {
  return read_len + 1 + (f32 ? 1 : 0) + ((f32 && single_strip) ? 1 : 0);
}

}  // namespace bvphmm
