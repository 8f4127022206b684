// Block-cooperative staging of per-Gaussian rows through shared memory.
//
// Kernels that give each thread one Gaussian read and write short rows
// (5..80 values) per Gaussian.  Accessed thread-per-row, a warp's loads and
// stores hit 32 different sectors per instruction; staged here, the block
// moves its rows [row0, row0 + nrows) as one contiguous, coalesced span, and
// each thread then reads its row from shared memory with an odd row stride
// (bank-conflict free).  Every thread of the block must call these (they
// synchronise), including threads past the end of the array.
#pragma once

#include "gsb_common.cuh"

namespace gsb {

__host__ __device__ constexpr int odd_stride(int n) { return n | 1; }

// Rows of ROWLEN values, row r of the block at s[r * odd_stride(ROWLEN)].
// Loads are issued in batches of 8 independent requests per thread so that
// the copy is not serialised on global-memory latency.
template <int ROWLEN, typename T>
__device__ __forceinline__ void stage_in(const T* __restrict__ g, int64_t row0, int64_t nrows_total,
                                         float* s) {
  constexpr int S = odd_stride(ROWLEN);
  constexpr int U = 8;
  const int64_t rows = min((int64_t)blockDim.x, nrows_total - row0);
  const int total = rows > 0 ? (int)rows * ROWLEN : 0;
  const T* base = g + row0 * ROWLEN;
  const int nt = blockDim.x;
  for (int j0 = threadIdx.x; j0 < total; j0 += nt * U) {
    float v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * nt;
      v[u] = j < total ? ld(base, j) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * nt;
      if (j < total) {
        const int r = j / ROWLEN, c = j - r * ROWLEN;
        s[r * S + c] = v[u];
      }
    }
  }
}

template <int ROWLEN>
__device__ __forceinline__ void stage_out(float* __restrict__ g, int64_t row0, int64_t nrows_total,
                                          const float* s) {
  constexpr int S = odd_stride(ROWLEN);
  const int64_t rows = min((int64_t)blockDim.x, nrows_total - row0);
  const int total = rows > 0 ? (int)rows * ROWLEN : 0;
  float* base = g + row0 * ROWLEN;
  for (int j = threadIdx.x; j < total; j += blockDim.x) {
    const int r = j / ROWLEN, c = j - r * ROWLEN;
    base[j] = s[r * S + c];
  }
}

// Same copies with the rows packed back to back (row stride = ROWLEN), the
// layout a 1-D bulk copy produces.
template <int ROWLEN, typename T>
__device__ __forceinline__ void stage_in_plain(const T* __restrict__ g, int64_t row0,
                                               int64_t nrows_total, float* s) {
  constexpr int U = 8;
  const int64_t rows = min((int64_t)blockDim.x, nrows_total - row0);
  const int total = rows > 0 ? (int)rows * ROWLEN : 0;
  const T* base = g + row0 * ROWLEN;
  const int nt = blockDim.x;
  for (int j0 = threadIdx.x; j0 < total; j0 += nt * U) {
    float v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * nt;
      v[u] = j < total ? ld(base, j) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * nt;
      if (j < total) s[j] = v[u];
    }
  }
}

template <int ROWLEN>
__device__ __forceinline__ void stage_out_plain(float* __restrict__ g, int64_t row0,
                                                int64_t nrows_total, const float* s) {
  const int64_t rows = min((int64_t)blockDim.x, nrows_total - row0);
  const int total = rows > 0 ? (int)rows * ROWLEN : 0;
  float* base = g + row0 * ROWLEN;
  for (int j = threadIdx.x; j < total; j += blockDim.x) base[j] = s[j];
}

}  // namespace gsb
