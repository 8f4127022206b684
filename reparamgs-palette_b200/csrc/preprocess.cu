// Per-Gaussian preprocess kernels behind the reference's geometry and SH
// operators (project, computeCov3D, computeCov2D, inverseCov2D, sh2Weight,
// sh2Weight_fast(_B), sh2Color).  One thread per Gaussian; every output
// element is written (culled Gaussians get the reference's zero values), so
// callers need not pre-clear outputs.
#include "gsb_geometry.cuh"
#include "gsb_internal.h"

namespace gsb {

constexpr int kThreads = 256;

// project -- gsplatcu/kernel.cu:618-663.
__global__ void __launch_bounds__(kThreads)
    k_project(int64_t n, const float* __restrict__ pws, const float* __restrict__ Rcw,
              const float* __restrict__ tcw, float fx, float fy, float cx, float cy,
              float* __restrict__ us, float* __restrict__ pcs, float* __restrict__ depths,
              float* __restrict__ du) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float R[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) R[k] = __ldg(Rcw + k);
  const float3 t = make_float3(__ldg(tcw), __ldg(tcw + 1), __ldg(tcw + 2));
  const float3 pw = make_float3(pws[3 * i], pws[3 * i + 1], pws[3 * i + 2]);
  const Projected p = project_point(pw, R, t, fx, fy, cx, cy);
  if (!p.valid) {
    depths[i] = kBadDepth;
    us[2 * i] = us[2 * i + 1] = 0.f;
    pcs[3 * i] = pcs[3 * i + 1] = pcs[3 * i + 2] = 0.f;
    if (du)
#pragma unroll
      for (int k = 0; k < 6; ++k) du[6 * i + k] = 0.f;
    return;
  }
  us[2 * i] = p.ux;
  us[2 * i + 1] = p.uy;
  pcs[3 * i] = p.x;
  pcs[3 * i + 1] = p.y;
  pcs[3 * i + 2] = p.z;
  depths[i] = p.z;
  if (du) {
    const float z_inv = 1.f / p.z;
    const float z2_inv = z_inv * z_inv;
    du[6 * i + 0] = fx * z_inv;
    du[6 * i + 1] = 0.f;
    du[6 * i + 2] = -(p.x * fx) * z2_inv;
    du[6 * i + 3] = 0.f;
    du[6 * i + 4] = fy * z_inv;
    du[6 * i + 5] = -(p.y * fy) * z2_inv;
  }
}

// computeCov3D -- gsplatcu/kernel.cu:422-501.
__global__ void __launch_bounds__(kThreads)
    k_cov3d(int64_t n, const float4* __restrict__ rots, const float* __restrict__ scales,
            const float* __restrict__ depths, float* __restrict__ cov3ds,
            float* __restrict__ dq, float* __restrict__ ds) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (depths[i] < kMinDepth) {
#pragma unroll
    for (int k = 0; k < 6; ++k) cov3ds[6 * i + k] = 0.f;
    if (dq) {
      for (int k = 0; k < 24; ++k) dq[24 * i + k] = 0.f;
      for (int k = 0; k < 18; ++k) ds[18 * i + k] = 0.f;
    }
    return;
  }
  const float4 q = rots[i];
  const float3 s = make_float3(scales[3 * i], scales[3 * i + 1], scales[3 * i + 2]);
  float cov[6], M[9], R[9];
  covariance_3d(q, s, cov, M, R);
#pragma unroll
  for (int k = 0; k < 6; ++k) cov3ds[6 * i + k] = cov[k];
  if (dq) {
    float jq[24], js[18];
    cov3d_jacobians(q, s, M, R, jq, js);
#pragma unroll
    for (int k = 0; k < 24; ++k) dq[24 * i + k] = jq[k];
#pragma unroll
    for (int k = 0; k < 18; ++k) ds[18 * i + k] = js[k];
  }
}

// computeCov2D -- gsplatcu/kernel.cu:508-611.
__global__ void __launch_bounds__(kThreads)
    k_cov2d(int64_t n, const float* __restrict__ cov3ds, const float* __restrict__ pcs,
            const float* __restrict__ Rcw, const float* __restrict__ depths, float fx, float fy,
            float tanx, float tany, float* __restrict__ cov2ds, float* __restrict__ d3,
            float* __restrict__ dp) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (depths[i] < kMinDepth) {
    cov2ds[3 * i] = cov2ds[3 * i + 1] = cov2ds[3 * i + 2] = 0.f;
    if (d3) {
      for (int k = 0; k < 18; ++k) d3[18 * i + k] = 0.f;
      for (int k = 0; k < 9; ++k) dp[9 * i + k] = 0.f;
    }
    return;
  }
  float R[9], c3[6], c2[3], M[6], xy[2];
#pragma unroll
  for (int k = 0; k < 9; ++k) R[k] = __ldg(Rcw + k);
#pragma unroll
  for (int k = 0; k < 6; ++k) c3[k] = cov3ds[6 * i + k];
  const float z = pcs[3 * i + 2];
  covariance_2d(c3, pcs[3 * i], pcs[3 * i + 1], z, R, fx, fy, tanx, tany, c2, M, xy);
  cov2ds[3 * i] = c2[0];
  cov2ds[3 * i + 1] = c2[1];
  cov2ds[3 * i + 2] = c2[2];
  if (d3) {
    float j3[18], jp[9];
    cov2d_jacobians(c3, M, R, xy[0], xy[1], z, fx, fy, j3, jp);
#pragma unroll
    for (int k = 0; k < 18; ++k) d3[18 * i + k] = j3[k];
#pragma unroll
    for (int k = 0; k < 9; ++k) dp[9 * i + k] = jp[k];
  }
}

// inverseCov2D -- gsplatcu/kernel.cu:379-415.  Updates depths in place.
__global__ void __launch_bounds__(kThreads)
    k_inverse_cov2d(int64_t n, const float* __restrict__ cov2ds, float* __restrict__ depths,
                    float* __restrict__ cinv, int* __restrict__ areas, float* __restrict__ dcinv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float conic[3] = {0.f, 0.f, 0.f};
  int ext[2] = {0, 0};
  float det_inv = 0.f;
  bool ok = false;
  const float a = cov2ds[3 * i], b = cov2ds[3 * i + 1], c = cov2ds[3 * i + 2];
  if (!(depths[i] < kMinDepth)) {
    ok = conic_and_extent(a, b, c, conic, ext, &det_inv);
    if (!ok) depths[i] = kBadDepth;
  }
  cinv[3 * i] = conic[0];
  cinv[3 * i + 1] = conic[1];
  cinv[3 * i + 2] = conic[2];
  areas[2 * i] = ext[0];
  areas[2 * i + 1] = ext[1];
  if (dcinv) {
    float J[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (ok) {
      const float d2 = det_inv * det_inv;
      J[0] = -c * c * d2;
      J[1] = 2 * b * c * d2;
      J[2] = -a * c * d2 + det_inv;
      J[3] = b * c * d2;
      J[4] = -2 * b * b * d2 - det_inv;
      J[5] = a * b * d2;
      J[6] = -a * c * d2 + det_inv;
      J[7] = 2 * a * b * d2;
      J[8] = -a * a * d2;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) dcinv[9 * i + k] = J[k];
  }
}

// sh2Weight / sh2Color -- gsplatcu/kernel.cu:670-870, 1040-1169.  Both are the
// same map feat_k = sum_l Y_l(dir) c[l*K + k] (band-major); colours are K = 3.
// All Gaussians are evaluated (no depth test), as in the reference.
// A Gaussian's coefficient row is NB*K values (up to 128); read one row per
// thread straight from global memory, a warp's loads would be strided by the
// row length and thrash L1.  The block's rows, one contiguous span, are
// therefore copied first into shared memory, where each thread reads its own
// row without bank conflicts, by asynchronous copies (cp.async), so the whole
// span is in flight at once without holding registers.  The staging mode is a
// template parameter (kShInPlace, kShStage4, kShStage16; see below), so the
// coefficient reads carry no runtime choice.  The band count NB is a template
// parameter too, so the basis, its gradient and the Jacobian sums stay in
// registers.  The outputs (K weights, and with the Jacobians NB basis
// values and 3K direction derivatives per Gaussian) are gathered in shared
// memory at odd row strides and written back as contiguous spans of the
// block's rows.
constexpr int kShThreads = 64;  // 64 rows of at most 129 floats: 33 KB of shared memory

// Staging modes of k_sh2feat:
// - kShInPlace: rows read from global memory (BF16 rows of odd length or from
//   a base that is not 4-byte aligned);
// - kShStage4: one 4-byte copy per FP32 element or BF16 element pair, rows at
//   an odd stride of 32-bit words;
// - kShStage16: FP32 rows whose length is a multiple of 4, from a 16-byte
//   aligned base: one 16-byte copy per 4 elements, rows at an odd stride of
//   16-byte words, read as float4 (a quarter-warp's 8 lanes hit 8 distinct
//   4-bank groups).
constexpr int kShInPlace = 0, kShStage4 = 1, kShStage16 = 2;

template <int K, int NB>
struct ShOut {
  static constexpr int SK = K | 1, SNB = NB | 1, S3K = (3 * K) | 1;  // odd row strides
};

// Copies `rows` rows of `w` floats from shared memory (row stride `ws`) to
// the contiguous global span `dst`, one float per thread per step.
template <int w, int ws>
__device__ __forceinline__ void rows_out(const float* src, int rows, float* __restrict__ dst) {
  for (int e = threadIdx.x; e < rows * w; e += kShThreads) {
    const int r = e / w;
    dst[e] = src[r * ws + (e - r * w)];
  }
}

template <int K, int NB, typename T, int MODE>
__global__ void __launch_bounds__(kShThreads)
    k_sh2feat(int64_t n, const T* __restrict__ shs, const float* __restrict__ pws,
              const float* __restrict__ twc, float* __restrict__ feat,
              float* __restrict__ dshs, float* __restrict__ dpws) {
  extern __shared__ __align__(16) float srows[];
  constexpr int rl = NB * K, stride = rl | 1;
  // kShStage16: 16-byte words per row and the row stride in floats
  constexpr int kV4 = rl / 4 > 0 ? rl / 4 : 1, kV4Stride = 4 * (kV4 | 1);
  static_assert(MODE != kShStage16 || (sizeof(T) == 4 && rl % 4 == 0), "16-byte staging");
  // staged BF16 rows: 32-bit words per row and the row stride in words
  // (odd BF16 rows are never staged)
  constexpr int kBfWords = rl / 2 > 0 ? rl / 2 : 1, kBfStride = kBfWords | 1;
  using O = ShOut<K, NB>;
  const int64_t row0 = (int64_t)blockIdx.x * kShThreads;
  const int rows = (int)min((int64_t)kShThreads, n - row0);
  // BF16 rows of even length from a 4-byte aligned base are copied as element
  // pairs (2-byte copies cost more than the strided reads they replace); other
  // BF16 rows are read in place.  The host picks the mode and sizes the
  // shared memory by it.
  constexpr bool kF32 = sizeof(T) == 4;
  if constexpr (MODE == kShStage16) {
    const float4* src = reinterpret_cast<const float4*>(shs + row0 * rl);
    const int total = rows * kV4;
    int r = threadIdx.x / kV4, q = threadIdx.x - r * kV4;
    constexpr int dr = kShThreads / kV4, dq = kShThreads - dr * kV4;
    for (int e = threadIdx.x; e < total; e += kShThreads) {
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                       (uint32_t)__cvta_generic_to_shared(srows + r * kV4Stride + 4 * q)),
                   "l"(src + e)
                   : "memory");
      q += dq;
      r += dr;
      if (q >= kV4) {
        q -= kV4;
        ++r;
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if constexpr (MODE == kShStage4 && kF32) {
    // FP32: every element of the block's span is one 4-byte asynchronous
    // copy (cp.async), so the whole span is in flight at once without
    // holding registers; (row, column) of element e advanced by kShThreads
    // elements per step
    const float* src = reinterpret_cast<const float*>(shs) + row0 * rl;
    const int total = rows * rl;
    int r = threadIdx.x / rl, q = threadIdx.x - r * rl;
    constexpr int dr = kShThreads / rl, dq = kShThreads - dr * rl;
    for (int e = threadIdx.x; e < total; e += kShThreads) {
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                       (uint32_t)__cvta_generic_to_shared(srows + r * stride + q)),
                   "l"(src + e)
                   : "memory");
      q += dq;
      r += dr;
      if (q >= rl) {
        q -= rl;
        ++r;
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if constexpr (MODE == kShStage4) {
    // BF16 rows of even length from a 4-byte aligned base: each element pair
    // is one 4-byte asynchronous copy, kept raw at an odd row stride of
    // 32-bit words and converted when read
    uint32_t* dst = reinterpret_cast<uint32_t*>(srows);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(shs + row0 * rl);
    const int total = rows * kBfWords;
    int r = threadIdx.x / kBfWords, q = threadIdx.x - r * kBfWords;
    constexpr int dr = kShThreads / kBfWords, dq = kShThreads - dr * kBfWords;
    for (int e = threadIdx.x; e < total; e += kShThreads) {
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                       (uint32_t)__cvta_generic_to_shared(dst + r * kBfStride + q)),
                   "l"(src + e)
                   : "memory");
      q += dq;
      r += dr;
      if (q >= kBfWords) {
        q -= kBfWords;
        ++r;
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  }
  __syncthreads();
  const int64_t i = row0 + threadIdx.x;
  const bool live = i < n;
  const bool jac = dshs != nullptr;
  float acc[K], Y[16], dp[3 * K];
  if (live) {
    const float* srow = srows + threadIdx.x * stride;
    const float4* srow4 = reinterpret_cast<const float4*>(srows + threadIdx.x * kV4Stride);
    const __nv_bfloat16* sraw = reinterpret_cast<const __nv_bfloat16*>(
        reinterpret_cast<const uint32_t*>(srows) + threadIdx.x * kBfStride);
    const T* grow = shs + i * (int64_t)rl;
    const auto c = [&](int idx) -> float {
      if constexpr (MODE == kShStage16) {
        const float4 v = srow4[idx >> 2];
        return (idx & 3) == 0 ? v.x : (idx & 3) == 1 ? v.y : (idx & 3) == 2 ? v.z : v.w;
      } else if constexpr (MODE == kShStage4) {
        if constexpr (kF32)
          return srow[idx];
        else
          return __bfloat162float(sraw[idx]);
      } else {
        return ld(grow, idx);
      }
    };
    float dir[3] = {0.f, 0.f, 0.f}, nd[3] = {0.f, 0.f, 0.f}, ninv = 0.f;
    if (NB > 1) {
      const float3 pw = make_float3(pws[3 * i], pws[3 * i + 1], pws[3 * i + 2]);
      const float3 cam = make_float3(__ldg(twc), __ldg(twc + 1), __ldg(twc + 2));
      view_direction(pw, cam, dir, nd, &ninv);
    }
    sh_basis(dir, NB, Y);
    sh_weights_full<K>(c, NB, Y, acc);
    if (jac) {
      float Gd[48], J[9];
      sh_basis_grad(dir, NB, /*ref_quirk=*/true, Gd);
      if (NB > 1) dir_jacobian(nd, ninv, J);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        float dd[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int l = 1; l < NB; ++l) {
          const float cv = c(l * K + k);
          dd[0] += Gd[3 * l] * cv;
          dd[1] += Gd[3 * l + 1] * cv;
          dd[2] += Gd[3 * l + 2] * cv;
        }
#pragma unroll
        for (int j = 0; j < 3; ++j)
          dp[3 * k + j] = NB > 1 ? dd[0] * J[j] + dd[1] * J[3 + j] + dd[2] * J[6 + j] : 0.f;
      }
    }
  }
  __syncthreads();  // the staged rows are no longer read
  float* s_feat = srows;
  float* s_y = s_feat + kShThreads * O::SK;
  float* s_dp = s_y + kShThreads * O::SNB;
  if (live) {
#pragma unroll
    for (int k = 0; k < K; ++k) s_feat[threadIdx.x * O::SK + k] = acc[k];
    if (jac) {
#pragma unroll
      for (int l = 0; l < NB; ++l) s_y[threadIdx.x * O::SNB + l] = Y[l];
#pragma unroll
      for (int m = 0; m < 3 * K; ++m) s_dp[threadIdx.x * O::S3K + m] = dp[m];
    }
  }
  __syncthreads();
  rows_out<K, O::SK>(s_feat, rows, feat + row0 * K);
  if (jac) {
    rows_out<NB, O::SNB>(s_y, rows, dshs + row0 * NB);
    rows_out<3 * K, O::S3K>(s_dp, rows, dpws + row0 * 3 * K);
  }
}

// ------------------------------------------------------------ launchers
static int grid_for(int64_t n) { return div_up(n > 0 ? n : 1, kThreads); }

int launch_project(int64_t n, const float* pws, const float* Rcw, const float* tcw, float fx,
                   float fy, float cx, float cy, float* us, float* pcs, float* depths, float* du,
                   cudaStream_t st) {
  if (n == 0) return GSB_OK;
  k_project<<<grid_for(n), kThreads, 0, st>>>(n, pws, Rcw, tcw, fx, fy, cx, cy, us, pcs, depths, du);
  return check_launch("project");
}

int launch_cov3d(int64_t n, const float* rots, const float* scales, const float* depths,
                 float* cov3ds, float* dq, float* ds, cudaStream_t st) {
  if (n == 0) return GSB_OK;
  k_cov3d<<<grid_for(n), kThreads, 0, st>>>(n, (const float4*)rots, scales, depths, cov3ds, dq, ds);
  return check_launch("computeCov3D");
}

int launch_cov2d(int64_t n, const float* cov3ds, const float* pcs, const float* Rcw,
                 const float* depths, float fx, float fy, float tanx, float tany, float* cov2ds,
                 float* d3, float* dp, cudaStream_t st) {
  if (n == 0) return GSB_OK;
  k_cov2d<<<grid_for(n), kThreads, 0, st>>>(n, cov3ds, pcs, Rcw, depths, fx, fy, tanx, tany, cov2ds, d3, dp);
  return check_launch("computeCov2D");
}

int launch_inverse_cov2d(int64_t n, const float* cov2ds, float* depths, float* cinv, int* areas,
                         float* dcinv, cudaStream_t st) {
  if (n == 0) return GSB_OK;
  k_inverse_cov2d<<<grid_for(n), kThreads, 0, st>>>(n, cov2ds, depths, cinv, areas, dcinv);
  return check_launch("inverseCov2D");
}

template <int K, int NB, typename T>
static void sh2feat_launch(int64_t n, const T* s, int mode, size_t smem, int g, const float* pws,
                           const float* twc, float* feat, float* dshs, float* dpws,
                           cudaStream_t st) {
  if constexpr (sizeof(T) == 4 && (NB * K) % 4 == 0) {
    if (mode == kShStage16) {
      k_sh2feat<K, NB, T, kShStage16><<<g, kShThreads, smem, st>>>(n, s, pws, twc, feat, dshs,
                                                                   dpws);
      return;
    }
  }
  if (mode == kShStage4)
    k_sh2feat<K, NB, T, kShStage4><<<g, kShThreads, smem, st>>>(n, s, pws, twc, feat, dshs, dpws);
  else
    k_sh2feat<K, NB, T, kShInPlace><<<g, kShThreads, smem, st>>>(n, s, pws, twc, feat, dshs,
                                                                 dpws);
}

template <int K, typename T>
static int sh2feat_kn(int64_t n, const T* s, int nb, int mode, size_t smem, int g,
                      const float* pws, const float* twc, float* feat, float* dshs, float* dpws,
                      cudaStream_t st) {
  switch (nb) {
    case 1: sh2feat_launch<K, 1, T>(n, s, mode, smem, g, pws, twc, feat, dshs, dpws, st); break;
    case 4: sh2feat_launch<K, 4, T>(n, s, mode, smem, g, pws, twc, feat, dshs, dpws, st); break;
    case 9: sh2feat_launch<K, 9, T>(n, s, mode, smem, g, pws, twc, feat, dshs, dpws, st); break;
    case 16: sh2feat_launch<K, 16, T>(n, s, mode, smem, g, pws, twc, feat, dshs, dpws, st); break;
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
  return GSB_OK;
}

template <typename T>
static int sh2feat_t(int64_t n, const void* shs, int nb, int K, const float* pws, const float* twc,
                     float* feat, float* dshs, float* dpws, cudaStream_t st) {
  const T* s = (const T*)shs;
  const int g = div_up(n > 0 ? n : 1, kShThreads);
  // FP32 rows by 16-byte copies when their length is a multiple of 4 and the
  // base 16-byte aligned, else by 4-byte copies; BF16 rows as 32-bit element
  // pairs when of even length from a 4-byte aligned base, else in place
  const int rl = nb * K;
  const uintptr_t base = reinterpret_cast<uintptr_t>(shs);
  const int mode = sizeof(T) == 4 ? (rl % 4 == 0 && (base & 15) == 0 ? kShStage16 : kShStage4)
                                  : (rl % 2 == 0 && (base & 3) == 0 ? kShStage4 : kShInPlace);
  const size_t row_words = mode == kShStage16 ? (size_t)(4 * ((rl / 4) | 1))
                           : sizeof(T) == 4   ? (size_t)(rl | 1)
                                              : (size_t)((rl / 2) | 1);  // raw BF16 pairs
  const size_t stage_bytes = mode != kShInPlace ? (size_t)kShThreads * row_words * 4 : 0;
  // output gathering: K weights, NB basis values and 3K derivatives per row
  // at odd strides (the NB + 3K part only with the Jacobians, but always
  // reserved: it is small)
  const size_t out_bytes =
      (size_t)kShThreads * ((K | 1) + (nb | 1) + ((3 * K) | 1)) * sizeof(float);
  const size_t smem = stage_bytes > out_bytes ? stage_bytes : out_bytes;
  int rc;
  switch (K) {
#define GSB_K(KK)                                                                          \
  case KK:                                                                                 \
    rc = sh2feat_kn<KK, T>(n, s, nb, mode, smem, g, pws, twc, feat, dshs, dpws, st);       \
    break;
    GSB_K(1) GSB_K(2) GSB_K(3) GSB_K(4) GSB_K(5) GSB_K(6) GSB_K(7) GSB_K(8)
#undef GSB_K
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
  if (rc) return rc;
  return check_launch("sh2Weight");
}

int launch_sh2feat(int64_t n, const void* shs, int dtype, int nb, int K, const float* pws,
                   const float* twc, float* feat, float* dshs, float* dpws, cudaStream_t st) {
  if (n == 0) return GSB_OK;
  return dtype == GSB_DTYPE_BF16
             ? sh2feat_t<__nv_bfloat16>(n, shs, nb, K, pws, twc, feat, dshs, dpws, st)
             : sh2feat_t<float>(n, shs, nb, K, pws, twc, feat, dshs, dpws, st);
}

}  // namespace gsb
