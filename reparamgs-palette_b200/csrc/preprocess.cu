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
// A Gaussian's coefficient row is nb*K values (up to 128); read one row per
// thread straight from global memory, a warp's loads would be strided by the
// row length and thrash L1.  The block's rows, one contiguous span, are
// therefore copied first (coalesced, kShCopy loads in flight per thread) into
// shared memory at an odd row stride, where each thread reads its own row
// without bank conflicts.
constexpr int kShThreads = 64;  // 64 rows of at most 129 floats: 33 KB of shared memory
constexpr int kShCopy = 8;

template <int K, typename T>
__global__ void __launch_bounds__(kShThreads)
    k_sh2feat(int64_t n, const T* __restrict__ shs, int nb, bool staged,
              const float* __restrict__ pws, const float* __restrict__ twc,
              float* __restrict__ feat, float* __restrict__ dshs, float* __restrict__ dpws) {
  extern __shared__ float srows[];
  const int rl = nb * K, stride = rl | 1;
  const int64_t row0 = (int64_t)blockIdx.x * kShThreads;
  const int rows = (int)min((int64_t)kShThreads, n - row0);
  // FP32 rows are copied element by element; BF16 rows of even length from a
  // 4-byte aligned base as element pairs, one 32-bit load each (2-byte
  // element loads cost more than the strided reads they replace); other BF16
  // rows are read in place.  The host makes that decision (`staged`) and
  // sizes the shared memory by it.
  constexpr bool kF32 = sizeof(T) == 4;
  if (staged) {
    // G elements per load; (row, column) of load e advanced by kShThreads
    // loads per step
    const int G = kF32 ? 1 : 2;
    const int rlg = rl / G, total = rows * rlg;
    int r = threadIdx.x / rlg, q = threadIdx.x - r * rlg;
    const int dr = kShThreads / rlg, dq = kShThreads - dr * rlg;
    for (int e0 = threadIdx.x; e0 < total; e0 += kShCopy * kShThreads) {
      float2 v[kShCopy];
      int at[kShCopy];
#pragma unroll
      for (int u = 0; u < kShCopy; ++u) {
        const int e = e0 + u * kShThreads;
        if constexpr (kF32) {
          v[u].x = e < total ? ld(shs + row0 * rl, e) : 0.f;
        } else {
          const __nv_bfloat162* src = reinterpret_cast<const __nv_bfloat162*>(shs + row0 * rl);
          v[u] = e < total ? __bfloat1622float2(src[e]) : make_float2(0.f, 0.f);
        }
        at[u] = r * stride + q * G;
        q += dq;
        r += dr;
        if (q >= rlg) {
          q -= rlg;
          ++r;
        }
      }
#pragma unroll
      for (int u = 0; u < kShCopy; ++u) {
        if (e0 + u * kShThreads < total) {
          srows[at[u]] = v[u].x;
          if constexpr (!kF32) srows[at[u] + 1] = v[u].y;
        }
      }
    }
  }
  __syncthreads();
  const int64_t i = row0 + threadIdx.x;
  if (i >= n) return;
  const float* srow = srows + threadIdx.x * stride;
  const T* grow = shs + i * (int64_t)rl;
  const auto c = [&](int idx) { return staged ? srow[idx] : ld(grow, idx); };
  float dir[3] = {0.f, 0.f, 0.f}, nd[3] = {0.f, 0.f, 0.f}, ninv = 0.f;
  float Y[16];
  if (nb > 1) {
    const float3 pw = make_float3(pws[3 * i], pws[3 * i + 1], pws[3 * i + 2]);
    const float3 cam = make_float3(__ldg(twc), __ldg(twc + 1), __ldg(twc + 2));
    view_direction(pw, cam, dir, nd, &ninv);
  }
  sh_basis(dir, nb, Y);
  float acc[K];
  sh_weights_full<K>(c, nb, Y, acc);
#pragma unroll
  for (int k = 0; k < K; ++k) feat[i * K + k] = acc[k];
  if (dshs) {
    for (int l = 0; l < nb; ++l) dshs[i * nb + l] = Y[l];
    float G[48], J[9];
    sh_basis_grad(dir, nb, /*ref_quirk=*/true, G);
    if (nb > 1) dir_jacobian(nd, ninv, J);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float dd[3] = {0.f, 0.f, 0.f};
      for (int l = 1; l < nb; ++l) {
        const float cv = c(l * K + k);
        dd[0] += G[3 * l] * cv;
        dd[1] += G[3 * l + 1] * cv;
        dd[2] += G[3 * l + 2] * cv;
      }
#pragma unroll
      for (int j = 0; j < 3; ++j)
        dpws[(i * K + k) * 3 + j] =
            nb > 1 ? dd[0] * J[j] + dd[1] * J[3 + j] + dd[2] * J[6 + j] : 0.f;
    }
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

template <typename T>
static int sh2feat_t(int64_t n, const void* shs, int nb, int K, const float* pws, const float* twc,
                     float* feat, float* dshs, float* dpws, cudaStream_t st) {
  const T* s = (const T*)shs;
  const int g = div_up(n > 0 ? n : 1, kShThreads);
  // BF16 rows are staged as 32-bit element pairs: only rows of even length
  // from a 4-byte aligned base
  const bool staged = sizeof(T) == 4 ||
                      ((nb * K) % 2 == 0 && (reinterpret_cast<uintptr_t>(shs) & 3) == 0);
  const size_t smem = staged ? (size_t)kShThreads * ((nb * K) | 1) * sizeof(float) : 0;
  switch (K) {
#define GSB_K(KK)                                                                              \
  case KK:                                                                                     \
    k_sh2feat<KK, T><<<g, kShThreads, smem, st>>>(n, s, nb, staged, pws, twc, feat, dshs, dpws); \
    break;
    GSB_K(1) GSB_K(2) GSB_K(3) GSB_K(4) GSB_K(5) GSB_K(6) GSB_K(7) GSB_K(8)
#undef GSB_K
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
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
