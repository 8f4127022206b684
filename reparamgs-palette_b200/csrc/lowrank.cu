// Low-rank view-dependent palette weights: sh2Weight_fast and
// sh2Weight_fast_B (gsplatcu/kernel.cu:884-1032), generalised from rank 1 to
// rank r.  The L*K higher-order coefficients of a Gaussian, flattened
// band-major (g = l*K + k), are the P x Q matrix C = A B with A [P,r],
// B [r,Q]:  w_k = C0 dc_k + sum_l C[g/Q][g%Q] Y_l.
//
// Shapes used by the benchmark configurations (K = P = 5, Q = 15, rank 1..4,
// and K = P in 3..8 with Q = 15 -- the reference's default reshape) are
// compiled with every index known, so factors and gradient accumulators live
// in registers; any other valid shape runs a generic kernel that keeps each
// thread's accumulators in shared memory.  Both visit (k, l) in the
// reference's order (k outer, l inner) and add one rounded product at a time,
// so rank-1 gradients are bit-identical to the reference's sequential
// atomicAdd sums.
#include <algorithm>

#include "gsb_geometry.cuh"
#include "gsb_internal.h"
#include "gsb_stage.cuh"
#include "gsb_tma.cuh"

namespace gsb {

constexpr int kLrThreads = 128;

// ------------------------------------------------------------- forward
// Status word of this file's kernels (bit kStatusBulkTimeout: a bulk-copy wait
// gave up).  Read and cleared through gsb_device_status.
static __device__ uint32_t g_lowrank_status;

// Shared-memory layout of the fixed-shape kernels: one region per array, the
// rows of the block's Gaussians back to back (row stride = row length), so a
// full block's span of every array moves as one 1-D bulk copy.  BF16 factors
// stay raw (their spans are multiples of 256 bytes), packed at the start of
// the factor regions they replace, and are widened when read.
template <int K, int P, int Q, int R>
struct LrSmem {
  static constexpr int L = P * Q / K;
  static constexpr int LL = L > 0 ? L : 1;
  // forward: dc, A, B, pws in; w, ylm out
  static constexpr int fwd_floats = K + P * R + R * Q + 3 + K + LL;
  // backward: A, B, ylm, dw in; dA, dB out
  static constexpr int bwd_floats = P * R + R * Q + LL + K + P * R + R * Q;
};

// The block's rows of a BF16 array, copied raw (no bulk copy: the last block
// or an unaligned base); 8 loads in flight per thread.
template <int ROWLEN>
__device__ __forceinline__ void stage_raw_plain(const __nv_bfloat16* __restrict__ g, int64_t row0,
                                                int64_t nrows_total, __nv_bfloat16* s) {
  constexpr int U = 8;
  const int64_t rows = min((int64_t)blockDim.x, nrows_total - row0);
  const int total = rows > 0 ? (int)rows * ROWLEN : 0;
  const __nv_bfloat16* base = g + row0 * ROWLEN;
  const int nt = blockDim.x;
  for (int j0 = threadIdx.x; j0 < total; j0 += nt * U) {
    __nv_bfloat16 v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * nt;
      v[u] = j < total ? base[j] : __nv_bfloat16();
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * nt;
      if (j < total) s[j] = v[u];
    }
  }
}

template <int K, int P, int Q, int R, typename T>
__global__ void __launch_bounds__(kLrThreads)
    k_lowrank_fixed(int64_t n, const T* __restrict__ dc, const T* __restrict__ A,
                    const T* __restrict__ B, const float* __restrict__ pws,
                    const float* __restrict__ twc, float* __restrict__ w, float* __restrict__ ddc,
                    float* __restrict__ ylm) {
  using S = LrSmem<K, P, Q, R>;
  constexpr int L = S::L, PR = P * R, RQ = R * Q;
  extern __shared__ __align__(16) float sm[];
  __shared__ __align__(8) uint64_t bar;
  const int nt = blockDim.x;
  float* s_dc = sm;
  float* s_a = s_dc + nt * K;
  float* s_b = s_a + nt * PR;
  float* s_p = s_b + nt * RQ;
  float* s_w = s_p + nt * 3;
  float* s_y = s_w + nt * K;
  constexpr bool kBf = sizeof(T) == 2;
  T* r_dc = reinterpret_cast<T*>(sm);  // BF16: raw rows inside the dc, A, B regions
  T* r_a = r_dc + nt * K;
  T* r_b = r_a + nt * PR;
  const int64_t row0 = (int64_t)blockIdx.x * nt;
  const bool full = row0 + nt <= n;
  const bool bulk = full && aligned16(dc + row0 * K) && aligned16(A + row0 * PR) &&
                    aligned16(B + row0 * RQ) && aligned16(pws + row0 * 3);
  if (bulk && threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_arrive_expect_tx(&bar, (uint32_t)(nt * ((K + PR + RQ) * sizeof(T) + 3 * 4)));
  }
  if constexpr (kBf) {
    if (bulk) {
      if (threadIdx.x == 0) {
        bulk_load(r_dc, dc + row0 * K, (uint32_t)(nt * K * 2), &bar);
        bulk_load(r_a, A + row0 * PR, (uint32_t)(nt * PR * 2), &bar);
        bulk_load(r_b, B + row0 * RQ, (uint32_t)(nt * RQ * 2), &bar);
      }
    } else {
      stage_raw_plain<K>(dc, row0, n, r_dc);
      stage_raw_plain<PR>(A, row0, n, r_a);
      stage_raw_plain<RQ>(B, row0, n, r_b);
    }
  } else {
    stage_rows<K>(dc, row0, n, s_dc, bulk, &bar);
    stage_rows<PR>(A, row0, n, s_a, bulk, &bar);
    stage_rows<RQ>(B, row0, n, s_b, bulk, &bar);
  }
  stage_rows<3>(pws, row0, n, s_p, bulk, &bar);
  __syncthreads();
  if (bulk && !mbar_wait(&bar, 0)) {
    if (threadIdx.x == 0) atomicOr(&g_lowrank_status, kStatusBulkTimeout);
    mbar_wait(&bar, 0);  // bounded second wait for copies still in flight
    return;
  }
  const int t = threadIdx.x;
  if (row0 + t < n) {
    float wk[K], Y[16];
    Y[0] = SH_C0;
    if (L > 0) {
      float dir[3];
      const float3 pw = make_float3(s_p[t * 3], s_p[t * 3 + 1], s_p[t * 3 + 2]);
      const float3 cam = make_float3(__ldg(twc), __ldg(twc + 1), __ldg(twc + 2));
      view_direction(pw, cam, dir, nullptr, nullptr);
      sh_basis(dir, L + 1, Y);
#pragma unroll
      for (int l = 0; l < L; ++l) s_y[t * S::LL + l] = Y[l + 1];
    }
    if constexpr (kBf)
      lowrank_weights<K, P, Q, R>(r_dc + t * K, r_a + t * PR, r_b + t * RQ, Y, wk);
    else
      lowrank_weights<K, P, Q, R>(s_dc + t * K, s_a + t * PR, s_b + t * RQ, Y, wk);
#pragma unroll
    for (int k = 0; k < K; ++k) s_w[t * K + k] = wk[k];
  }
  if (ddc) {
    const int64_t rows = min((int64_t)nt, n - row0);
    for (int64_t j = t; j < rows * K; j += nt) ddc[row0 * K + j] = SH_C0;
  }
  const bool bulk_out = full && aligned16(w + row0 * K) && (L == 0 || !ylm || aligned16(ylm + row0 * L));
  if (bulk_out) {
    fence_proxy_async_shared();
    __syncthreads();
    if (t == 0) {
      bulk_store(w + row0 * K, s_w, (uint32_t)(nt * K * 4));
      if (L > 0 && ylm) bulk_store(ylm + row0 * L, s_y, (uint32_t)(nt * L * 4));
      bulk_store_drain();
    }
  } else {
    __syncthreads();
    stage_out_plain<K>(w, row0, n, s_w);
    if (L > 0 && ylm) stage_out_plain<S::LL>(ylm, row0, n, s_y);
  }
}

template <int K, typename T>
__global__ void __launch_bounds__(kLrThreads)
    k_lowrank_generic(int64_t n, const T* __restrict__ dc, const T* __restrict__ A,
                      const T* __restrict__ B, int P, int Q, int rank, int L,
                      const float* __restrict__ pws, const float* __restrict__ twc,
                      float* __restrict__ w, float* __restrict__ ddc, float* __restrict__ ylm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float wk[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    wk[k] = SH_C0 * ld(dc, i * K + k);
    if (ddc) ddc[i * K + k] = SH_C0;
  }
  if (L > 0) {
    float dir[3], Y[16];
    const float3 pw = make_float3(pws[3 * i], pws[3 * i + 1], pws[3 * i + 2]);
    const float3 cam = make_float3(__ldg(twc), __ldg(twc + 1), __ldg(twc + 2));
    view_direction(pw, cam, dir, nullptr, nullptr);
    sh_basis(dir, L + 1, Y);
    if (ylm)
      for (int l = 0; l < L; ++l) ylm[i * L + l] = Y[l + 1];
    const T* a = A + i * (int64_t)P * rank;
    const T* b = B + i * (int64_t)rank * Q;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float acc = 0.f;
      for (int l = 0; l < L; ++l) {
        const int g = l * K + k, row = g / Q, col = g % Q;
        float coef = ld(a, row * rank) * ld(b, col);
        for (int r = 1; r < rank; ++r) coef += ld(a, row * rank + r) * ld(b, r * Q + col);
        acc += coef * Y[l + 1];
      }
      wk[k] += acc;
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) w[i * K + k] = wk[k];
}

// ------------------------------------------------------------ backward
// dA[row][r] += (dw_k B[r][col]) Y_l ;  dB[r][col] += (dw_k A[row][r]) Y_l
// Rank 1 accumulates in the reference's (k outer, l inner) order.  Higher
// ranks (no reference counterpart) use dC[p][q] = dw_k Y_l with g = p*Q + q
// and two register-light sweeps: dA = dC B^T row by row, then dB = A^T dC
// column by column.
template <int K, int P, int Q, int R, typename T>
__global__ void __launch_bounds__(kLrThreads)
    k_lowrank_b_fixed(int64_t n, const T* __restrict__ A, const T* __restrict__ B,
                      const float* __restrict__ ylm, const float* __restrict__ dw,
                      float* __restrict__ dA, float* __restrict__ dB) {
  using S = LrSmem<K, P, Q, R>;
  constexpr int L = S::L, LL = S::LL, PR = P * R, RQ = R * Q;
  extern __shared__ __align__(16) float sm[];
  __shared__ __align__(8) uint64_t bar;
  const int nt = blockDim.x;
  float* s_a = sm;
  float* s_b = s_a + nt * PR;
  float* s_y = s_b + nt * RQ;
  float* s_g = s_y + nt * LL;
  float* s_da = s_g + nt * K;
  float* s_db = s_da + nt * PR;
  constexpr bool kBf = sizeof(T) == 2;
  T* r_a = reinterpret_cast<T*>(sm);  // BF16: raw rows inside the A, B regions
  T* r_b = r_a + nt * PR;
  const int64_t row0 = (int64_t)blockIdx.x * nt;
  const bool full = row0 + nt <= n;
  const bool bulk = full && L > 0 && aligned16(A + row0 * PR) && aligned16(B + row0 * RQ) &&
                    aligned16(ylm + row0 * L) && aligned16(dw + row0 * K);
  if (bulk && threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_arrive_expect_tx(&bar, (uint32_t)(nt * ((PR + RQ) * sizeof(T) + (L + K) * 4)));
  }
  if constexpr (kBf) {
    if (bulk) {
      if (threadIdx.x == 0) {
        bulk_load(r_a, A + row0 * PR, (uint32_t)(nt * PR * 2), &bar);
        bulk_load(r_b, B + row0 * RQ, (uint32_t)(nt * RQ * 2), &bar);
      }
    } else {
      stage_raw_plain<PR>(A, row0, n, r_a);
      stage_raw_plain<RQ>(B, row0, n, r_b);
    }
  } else {
    stage_rows<PR>(A, row0, n, s_a, bulk, &bar);
    stage_rows<RQ>(B, row0, n, s_b, bulk, &bar);
  }
  if (L > 0) stage_rows<LL>(ylm, row0, n, s_y, bulk, &bar);
  stage_rows<K>(dw, row0, n, s_g, bulk, &bar);
  __syncthreads();
  if (bulk && !mbar_wait(&bar, 0)) {
    if (threadIdx.x == 0) atomicOr(&g_lowrank_status, kStatusBulkTimeout);
    mbar_wait(&bar, 0);  // bounded second wait for copies still in flight
    return;
  }
  const int t = threadIdx.x;
  // this thread's factor rows, FP32 or raw BF16 widened on read
  const auto fa = [&](int j) -> float {
    if constexpr (kBf) return __bfloat162float(r_a[t * PR + j]);
    else return s_a[t * PR + j];
  };
  const auto fb = [&](int j) -> float {
    if constexpr (kBf) return __bfloat162float(r_b[t * RQ + j]);
    else return s_b[t * RQ + j];
  };
  if (row0 + t < n) {
    float y[LL], g0[K];
#pragma unroll
    for (int l = 0; l < L; ++l) y[l] = s_y[t * LL + l];
#pragma unroll
    for (int k = 0; k < K; ++k) g0[k] = s_g[t * K + k];
    if constexpr (R == 1) {
      float a[P], b[Q], da[P], db[Q];
#pragma unroll
      for (int j = 0; j < P; ++j) {
        a[j] = fa(j);
        da[j] = 0.f;
      }
#pragma unroll
      for (int j = 0; j < Q; ++j) {
        b[j] = fb(j);
        db[j] = 0.f;
      }
#pragma unroll
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int l = 0; l < L; ++l) {
          const int g = l * K + k, row = g / Q, col = g % Q;
          da[row] = __fadd_rn(da[row], (g0[k] * b[col]) * y[l]);
          db[col] = __fadd_rn(db[col], (g0[k] * a[row]) * y[l]);
        }
#pragma unroll
      for (int j = 0; j < P; ++j) s_da[t * P + j] = da[j];
#pragma unroll
      for (int j = 0; j < Q; ++j) s_db[t * Q + j] = db[j];
    } else {
#pragma unroll
      for (int p = 0; p < P; ++p) {  // dA[p][r] = sum_q dC[p][q] B[r][q]
        float acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0.f;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const int g = p * Q + q;
          const float c = g0[g % K] * y[g / K];
#pragma unroll
          for (int r = 0; r < R; ++r) acc[r] += c * fb(r * Q + q);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) s_da[t * PR + p * R + r] = acc[r];
      }
#pragma unroll
      for (int q = 0; q < Q; ++q) {  // dB[r][q] = sum_p dC[p][q] A[p][r]
        float acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0.f;
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const int g = p * Q + q;
          const float c = g0[g % K] * y[g / K];
#pragma unroll
          for (int r = 0; r < R; ++r) acc[r] += c * fa(p * R + r);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) s_db[t * RQ + r * Q + q] = acc[r];
      }
    }
  }
  const bool bulk_out = full && aligned16(dA + row0 * PR) && aligned16(dB + row0 * RQ);
  if (bulk_out) {
    fence_proxy_async_shared();
    __syncthreads();
    if (t == 0) {
      bulk_store(dA + row0 * PR, s_da, (uint32_t)(nt * PR * 4));
      bulk_store(dB + row0 * RQ, s_db, (uint32_t)(nt * RQ * 4));
      bulk_store_drain();
    }
  } else {
    __syncthreads();
    stage_out_plain<PR>(dA, row0, n, s_da);
    stage_out_plain<RQ>(dB, row0, n, s_db);
  }
}

const uint32_t* lowrank_status_word() {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_lowrank_status) != cudaSuccess) {
    (void)cudaGetLastError();
    return nullptr;
  }
  return (const uint32_t*)p;
}

int lowrank_status(uint32_t* out, bool clear, cudaStream_t st) {
  if (cudaMemcpyFromSymbolAsync(out, g_lowrank_status, sizeof(uint32_t), 0,
                                cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return check_launch("device_status", 0);
  if (clear) {
    const uint32_t zero = 0;
    if (cudaMemcpyToSymbolAsync(g_lowrank_status, &zero, sizeof(uint32_t), 0,
                                cudaMemcpyHostToDevice, st) != cudaSuccess)
      return check_launch("device_status", 0);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return check_launch("device_status", 0);
  return GSB_OK;
}

// Any valid shape: each thread's dA/dB accumulators in dynamic shared memory.
template <typename T>
__global__ void k_lowrank_b_generic(int64_t n, const T* __restrict__ A, const T* __restrict__ B,
                                    const float* __restrict__ ylm, const float* __restrict__ dw,
                                    int K, int P, int Q, int rank, int L, float* __restrict__ dA,
                                    float* __restrict__ dB) {
  extern __shared__ float sacc[];
  const int per = (P + Q) * rank;
  float* da = sacc + threadIdx.x * per;
  float* db = da + P * rank;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T* a = A + i * (int64_t)P * rank;
  const T* b = B + i * (int64_t)rank * Q;
  for (int j = 0; j < per; ++j) da[j] = 0.f;
  for (int k = 0; k < K; ++k) {
    const float g0 = dw[i * K + k];
    for (int l = 0; l < L; ++l) {
      const int g = l * K + k, row = g / Q, col = g % Q;
      const float y = ylm[i * L + l];
      for (int r = 0; r < rank; ++r) {
        da[row * rank + r] = __fadd_rn(da[row * rank + r], (g0 * ld(b, r * Q + col)) * y);
        db[r * Q + col] = __fadd_rn(db[r * Q + col], (g0 * ld(a, row * rank + r)) * y);
      }
    }
  }
  for (int j = 0; j < P * rank; ++j) dA[i * (int64_t)P * rank + j] = da[j];
  for (int j = 0; j < rank * Q; ++j) dB[i * (int64_t)rank * Q + j] = db[j];
}

// ------------------------------------------------------------ dispatch
static int grid_lr(int64_t n, int threads) { return div_up(n > 0 ? n : 1, threads); }

template <typename T>
static bool lowrank_fixed(int64_t n, const void* dc, const void* A, const void* B, int K, int P,
                          int Q, int rank, const float* pws, const float* twc, float* w, float* ddc,
                          float* ylm, cudaStream_t st) {
  const int g = grid_lr(n, kLrThreads);
  const T *d = (const T*)dc, *a = (const T*)A, *b = (const T*)B;
#define GSB_LR(KK, PP, QQ, RR)                                                              \
  if (K == KK && P == PP && Q == QQ && rank == RR) {                                        \
    const int sm = LrSmem<KK, PP, QQ, RR>::fwd_floats * kLrThreads * 4;                     \
    auto kern = k_lowrank_fixed<KK, PP, QQ, RR, T>;                                         \
    static bool attr_set = false; /* once per process; set before first launch */          \
    if (sm > 48 * 1024 && !attr_set)                                                        \
      attr_set = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                      sm) == cudaSuccess;                                   \
    kern<<<g, kLrThreads, sm, st>>>(n, d, a, b, pws, twc, w, ddc, ylm);                     \
    return true;                                                                            \
  }
  GSB_LR(5, 5, 15, 1) GSB_LR(5, 5, 15, 2) GSB_LR(5, 5, 15, 3) GSB_LR(5, 5, 15, 4)
  GSB_LR(3, 3, 15, 1) GSB_LR(4, 4, 15, 1) GSB_LR(6, 6, 15, 1) GSB_LR(7, 7, 15, 1)
  GSB_LR(8, 8, 15, 1) GSB_LR(6, 6, 15, 3)
#undef GSB_LR
  return false;
}

template <typename T>
static int lowrank_t(int64_t n, const void* dc, const void* A, const void* B, int K, int P, int Q,
                     int rank, int L, const float* pws, const float* twc, float* w, float* ddc,
                     float* ylm, cudaStream_t st) {
  if (lowrank_fixed<T>(n, dc, A, B, K, P, Q, rank, pws, twc, w, ddc, ylm, st))
    return check_launch("sh2Weight_fast");
  const int g = grid_lr(n, kLrThreads);
  const T *d = (const T*)dc, *a = (const T*)A, *b = (const T*)B;
  switch (K) {
#define GSB_K(KK)                                                                              \
  case KK:                                                                                     \
    k_lowrank_generic<KK, T><<<g, kLrThreads, 0, st>>>(n, d, a, b, P, Q, rank, L, pws, twc, w, \
                                                       ddc, ylm);                              \
    break;
    GSB_K(1) GSB_K(2) GSB_K(3) GSB_K(4) GSB_K(5) GSB_K(6) GSB_K(7) GSB_K(8)
#undef GSB_K
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
  return check_launch("sh2Weight_fast");
}

int launch_sh2weight_lowrank(int64_t n, const void* dc, const void* A, const void* B, int dtype,
                             int K, int P, int Q, int rank, int L, const float* pws,
                             const float* twc, float* w, float* ddc, float* ylm, cudaStream_t st) {
  if (n == 0) return GSB_OK;
  return dtype == GSB_DTYPE_BF16
             ? lowrank_t<__nv_bfloat16>(n, dc, A, B, K, P, Q, rank, L, pws, twc, w, ddc, ylm, st)
             : lowrank_t<float>(n, dc, A, B, K, P, Q, rank, L, pws, twc, w, ddc, ylm, st);
}

template <typename T>
static int lowrank_b_t(int64_t n, const void* A, const void* B, const float* ylm, const float* dw,
                       int K, int P, int Q, int rank, int L, float* dA, float* dB,
                       cudaStream_t st) {
  const T *a = (const T*)A, *b = (const T*)B;
  const int g = grid_lr(n, kLrThreads);
#define GSB_LRB(KK, PP, QQ, RR)                                                              \
  if (K == KK && P == PP && Q == QQ && rank == RR) {                                         \
    const int sm = LrSmem<KK, PP, QQ, RR>::bwd_floats * kLrThreads * 4;                      \
    auto kern = k_lowrank_b_fixed<KK, PP, QQ, RR, T>;                                        \
    static bool attr_set = false; /* once per process; set before first launch */           \
    if (sm > 48 * 1024 && !attr_set)                                                         \
      attr_set = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                      sm) == cudaSuccess;                                    \
    kern<<<g, kLrThreads, sm, st>>>(n, a, b, ylm, dw, dA, dB);                               \
    return check_launch("sh2Weight_fast_B");                                                 \
  }
  GSB_LRB(5, 5, 15, 1) GSB_LRB(5, 5, 15, 2) GSB_LRB(5, 5, 15, 3) GSB_LRB(5, 5, 15, 4)
  GSB_LRB(3, 3, 15, 1) GSB_LRB(4, 4, 15, 1) GSB_LRB(6, 6, 15, 1) GSB_LRB(7, 7, 15, 1)
  GSB_LRB(8, 8, 15, 1) GSB_LRB(6, 6, 15, 3)
#undef GSB_LRB
  // generic: pick the block size so that the accumulators fit in 96 KB
  const size_t per = (size_t)(P + Q) * rank * sizeof(float);
  int threads = (int)std::min<size_t>(kLrThreads, (96 * 1024) / per) / 32 * 32;
  if (threads < 32) {
    set_error("sh2Weight_fast_B: factor shape P=%d Q=%d rank=%d too large", P, Q, rank);
    return GSB_ERR_UNSUPPORTED;
  }
  const size_t smem = per * threads;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(k_lowrank_b_generic<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return check_launch("sh2Weight_fast_B (smem attribute)", 0);
  k_lowrank_b_generic<T><<<grid_lr(n, threads), threads, smem, st>>>(n, a, b, ylm, dw, K, P, Q,
                                                                     rank, L, dA, dB);
  return check_launch("sh2Weight_fast_B");
}

int launch_sh2weight_lowrank_b(int64_t n, const void* A, const void* B, int dtype,
                               const float* ylm, const float* dw, int K, int P, int Q, int rank,
                               int L, float* dA, float* dB, cudaStream_t st) {
  if (n == 0) return GSB_OK;
  return dtype == GSB_DTYPE_BF16
             ? lowrank_b_t<__nv_bfloat16>(n, A, B, ylm, dw, K, P, Q, rank, L, dA, dB, st)
             : lowrank_b_t<float>(n, A, B, ylm, dw, K, P, Q, rank, L, dA, dB, st);
}

}  // namespace gsb
