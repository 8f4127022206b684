// Per-Gaussian geometry and spherical-harmonic evaluation (device functions).
//
// Every value the rasterizer's decisions depend on (projected centre, depth,
// 3D/2D covariance, conic, 3-sigma extents) is computed with explicit
// round-to-nearest intrinsics (__fmul_rn, __fadd_rn, __fmaf_rn, __fdiv_rn)
// in the operation order the reference build's FP32 results follow
// (gsplatcu/kernel.cu:379-663): which product of each sum is fused into a
// multiply-add and which is rounded on its own was pinned by reproducing the
// reference build's outputs bit for bit from its inputs (exact FP32
// emulation, 1M and 3M Gaussians, two cameras).  The intrinsics are never
// contracted or reordered by the compiler, so the results do not depend on
// the kernel these functions are inlined into (separate operator kernels,
// the fused preprocess, the adjoint's recomputation): tile rectangles, sort
// keys and the per-pixel skip/stop decisions downstream agree with the
// reference exactly everywhere.  Jacobians are written in closed form.
#pragma once

#include "gsb_common.cuh"

namespace gsb {

__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }

// a0 b0 + a1 b1 + a2 b2 accumulated from zero in index order, each product
// fused into the running sum (the first rounded on its own).
__device__ __forceinline__ float dot3_fused(float a0, float a1, float a2, float b0, float b1,
                                            float b2) {
  return rfma(a2, b2, rfma(a1, b1, rmul(a0, b0)));
}
// The same sum with every product rounded before it is added.
__device__ __forceinline__ float dot3_plain(float a0, float a1, float a2, float b0, float b1,
                                            float b2) {
  return radd(radd(rmul(a0, b0), rmul(a1, b1)), rmul(a2, b2));
}

// ---------------------------------------------------------------- project
struct Projected {
  float x, y, z;  // camera-space centre
  float ux, uy;   // pixel centre
  bool valid;     // z >= 0.2
};

// pc = Rcw pw + t; u = (x fx) / z + c written as (x fx) * (1/z) + c.
__device__ __forceinline__ Projected project_point(float3 pw, const float* Rcw, float3 t, float fx,
                                                   float fy, float cx, float cy) {
  Projected r;
  r.x = radd(dot3_fused(Rcw[0], Rcw[1], Rcw[2], pw.x, pw.y, pw.z), t.x);
  r.y = radd(dot3_fused(Rcw[3], Rcw[4], Rcw[5], pw.x, pw.y, pw.z), t.y);
  r.z = radd(dot3_fused(Rcw[6], Rcw[7], Rcw[8], pw.x, pw.y, pw.z), t.z);
  r.valid = !(r.z < kMinDepth);
  if (r.valid) {
    const float z_inv = rdiv(1.f, r.z);
    r.ux = rfma(rmul(r.x, fx), z_inv, cx);
    r.uy = rfma(rmul(r.y, fy), z_inv, cy);
  } else {
    r.ux = r.uy = 0.f;
  }
  return r;
}

// ------------------------------------------------------------ covariance
// Rotation of an unnormalised quaternion (w, x, y, z), row-major:
// diagonal 1 - 2(.. + ..), off-diagonal 2(.. +- ..), each sum of two
// products with the fused product the reference's results show.
__device__ __forceinline__ void quat_rotation(float4 q, float* R) {
  const float w = q.x, x = q.y, y = q.z, z = q.w;
  const float xx = rmul(x, x), yy = rmul(y, y), zz = rmul(z, z);
  const float xz = rmul(x, z), zw = rmul(z, w), xw = rmul(x, w);
  R[0] = rsub(1.f, rmul(2.f, radd(yy, zz)));
  R[1] = rmul(2.f, rfma(x, y, -zw));
  R[2] = rmul(2.f, rfma(y, w, xz));
  R[3] = rmul(2.f, rfma(x, y, zw));
  R[4] = rsub(1.f, rmul(2.f, rfma(x, x, zz)));
  R[5] = rmul(2.f, rfma(y, z, -xw));
  R[6] = rmul(2.f, rfma(-y, w, xz));
  R[7] = rmul(2.f, rfma(y, z, xw));
  R[8] = rsub(1.f, rmul(2.f, rfma(x, x, yy)));
}

// Sigma = M M^T, M = R(q) diag(s); out = 6 upper entries (00,01,02,11,12,22).
// Also returns M (row-major) and R for the Jacobians.
__device__ __forceinline__ void covariance_3d(float4 q, float3 s, float* cov, float* Mout,
                                              float* Rout) {
  float R[9], M[9];
  quat_rotation(q, R);
  const float sv[3] = {s.x, s.y, s.z};
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) M[3 * r + c] = rmul(R[3 * r + c], sv[c]);
  const int sym[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
#pragma unroll
  for (int u = 0; u < 6; ++u) {
    const float* a = M + 3 * sym[u][0];
    const float* b = M + 3 * sym[u][1];
    cov[u] = dot3_fused(a[0], a[1], a[2], b[0], b[1], b[2]);
  }
  if (Mout)
#pragma unroll
    for (int k = 0; k < 9; ++k) Mout[k] = M[k];
  if (Rout)
#pragma unroll
    for (int k = 0; k < 9; ++k) Rout[k] = R[k];
}

// 2D screen covariance of a camera-space Gaussian.  The point is clamped to
// 1.3x the half field of view before forming the perspective Jacobian J;
// Sigma' = (J Rcw) Sigma (J Rcw)^T; +0.3 dilation on the diagonal.
// Mout receives J Rcw (row-major 2x3), xy the clamped x, y.
__device__ __forceinline__ void covariance_2d(const float* cov3, float px, float py, float pz,
                                              const float* Rcw, float fx, float fy, float tanx,
                                              float tany, float* cov2, float* Mout, float* xy) {
  const float z = pz;
  const float limx = rmul(1.3f, tanx);
  const float limy = rmul(1.3f, tany);
  const float x = rmul(fminf(limx, fmaxf(-limx, rdiv(px, z))), z);
  const float y = rmul(fminf(limy, fmaxf(-limy, rdiv(py, z))), z);
  const float z2 = rmul(z, z);
  // J = [[fx/z, 0, -(fx x)/z^2], [0, fy/z, -(fy y)/z^2]]
  const float J0[3] = {rdiv(fx, z), 0.0f, -rdiv(rmul(fx, x), z2)};
  const float J1[3] = {0.0f, rdiv(fy, z), -rdiv(rmul(fy, y), z2)};
  float M[6];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    M[j] = dot3_fused(J0[0], J0[1], J0[2], Rcw[j], Rcw[3 + j], Rcw[6 + j]);
    M[3 + j] = dot3_fused(J1[0], J1[1], J1[2], Rcw[j], Rcw[3 + j], Rcw[6 + j]);
  }
  const float a = cov3[0], b = cov3[1], c = cov3[2], d = cov3[3], e = cov3[4], f = cov3[5];
  // (M Sigma): row 0 fuses only the last product of its first entry; the
  // other entries round every product
  const float m00 = rfma(M[2], c, radd(rmul(M[0], a), rmul(M[1], b)));
  const float m01 = dot3_plain(M[0], M[1], M[2], b, d, e);
  const float m02 = dot3_plain(M[0], M[1], M[2], c, e, f);
  const float m10 = dot3_plain(M[3], M[4], M[5], a, b, c);
  const float m11 = dot3_plain(M[3], M[4], M[5], b, d, e);
  const float m12 = dot3_plain(M[3], M[4], M[5], c, e, f);
  // (M Sigma) M^T
  cov2[0] = radd(dot3_fused(m00, m01, m02, M[0], M[1], M[2]), 0.3f);
  cov2[1] = dot3_fused(m00, m01, m02, M[3], M[4], M[5]);
  cov2[2] = radd(dot3_fused(m10, m11, m12, M[3], M[4], M[5]), 0.3f);
  if (Mout)
#pragma unroll
    for (int k = 0; k < 6; ++k) Mout[k] = M[k];
  if (xy) {
    xy[0] = x;
    xy[1] = y;
  }
}

// Conic (inverse 2D covariance) and integer 3-sigma extents.  Returns false
// when 1/det is NaN (the Gaussian is then dropped).
__device__ __forceinline__ bool conic_and_extent(float a, float b, float c, float* conic,
                                                 int* ext, float* det_inv_out) {
  const float det_inv = rdiv(1.f, rfma(a, c, -rmul(b, b)));
  if (isnan(det_inv)) return false;
  conic[0] = rmul(det_inv, c);
  conic[1] = rmul(-det_inv, b);
  conic[2] = rmul(det_inv, a);
  ext[0] = (int)ceilf(rmul(3.f, sqrtf(fabsf(a))));
  ext[1] = (int)ceilf(rmul(3.f, sqrtf(fabsf(c))));
  if (det_inv_out) *det_inv_out = det_inv;
  return true;
}

// ------------------------------------------------------------ tile rects
// Tile rectangle [x0,x1) x [y0,y1) covered by centre u and extents (xs, ys),
// clamped to the tile grid; integer conversions truncate toward zero.  The
// upper bound rounds up as ((v + 16) - 1) / 16 in FP32.
struct TileRect {
  uint32_t x0, y0, x1, y1;
};

__device__ __forceinline__ TileRect tile_rect(float ux, float uy, float xs, float ys,
                                              uint32_t gx, uint32_t gy) {
  TileRect r;
  r.x0 = min(gx, (uint32_t)max(0, (int)((ux - xs) / kTile)));
  r.y0 = min(gy, (uint32_t)max(0, (int)((uy - ys) / kTile)));
  r.x1 = min(gx, (uint32_t)max(0, (int)(((ux + xs) + kTile - 1) / kTile)));
  r.y1 = min(gy, (uint32_t)max(0, (int)(((uy + ys) + kTile - 1) / kTile)));
  return r;
}

// ------------------------------------------------------ spherical harmonics
// Unit view direction and (optionally) its Jacobian w.r.t. the centre.
__device__ __forceinline__ void view_direction(float3 pw, float3 cam, float* dir, float* nd,
                                               float* inv_norm) {
  const float d0 = pw.x - cam.x, d1 = pw.y - cam.y, d2 = pw.z - cam.z;
  const float ninv = 1.f / sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
  dir[0] = d0 * ninv;
  dir[1] = d1 * ninv;
  dir[2] = d2 * ninv;
  if (nd) {
    nd[0] = d0;
    nd[1] = d1;
    nd[2] = d2;
  }
  if (inv_norm) *inv_norm = ninv;
}

// Real SH basis Y_0 .. Y_{nb-1} (nb in {1,4,9,16}) in band-major order.
__device__ __forceinline__ void sh_basis(const float* dir, int nb, float* Y) {
  const float x = dir[0], y = dir[1], z = dir[2];
  Y[0] = SH_C0;
  if (nb > 1) {
    Y[1] = -SH_C1 * y;
    Y[2] = SH_C1 * z;
    Y[3] = -SH_C1 * x;
    if (nb > 4) {
      const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
      Y[4] = SH_C2_0 * xy;
      Y[5] = -SH_C2_0 * yz;
      Y[6] = SH_C2_2 * (2.f * zz - xx - yy);
      Y[7] = -SH_C2_0 * xz;
      Y[8] = SH_C2_4 * (xx - yy);
      if (nb > 9) {
        Y[9] = -SH_C3_0 * y * (3.f * xx - yy);
        Y[10] = SH_C3_1 * xy * z;
        Y[11] = -SH_C3_2 * y * (4.f * zz - xx - yy);
        Y[12] = SH_C3_3 * z * (2.f * zz - 3.f * xx - 3.f * yy);
        Y[13] = -SH_C3_2 * x * (4.f * zz - xx - yy);
        Y[14] = SH_C3_5 * z * (xx - yy);
        Y[15] = -SH_C3_0 * x * (xx - 3.f * yy);
      }
    }
  }
}

// dY_l / d dir for l in [1, nb): G[3*l + r].  `ref_quirk` reproduces the
// reference's d Y_9 / d y = C (3x^2 - 2y^2) (gsplatcu/kernel.cu:840) that the
// compatibility Jacobian outputs return; the adjoint uses the true
// derivative C (3x^2 - 3y^2).
__device__ __forceinline__ void sh_basis_grad(const float* dir, int nb, bool ref_quirk, float* G) {
  const float x = dir[0], y = dir[1], z = dir[2];
#pragma unroll
  for (int k = 0; k < 48; ++k) G[k] = 0.f;
  if (nb <= 1) return;
  G[3 * 1 + 1] = -SH_C1;
  G[3 * 2 + 2] = SH_C1;
  G[3 * 3 + 0] = -SH_C1;
  if (nb <= 4) return;
  const float xx = x * x, yy = y * y, zz = z * z;
  G[3 * 4 + 0] = SH_C2_0 * y;
  G[3 * 4 + 1] = SH_C2_0 * x;
  G[3 * 5 + 1] = -SH_C2_0 * z;
  G[3 * 5 + 2] = -SH_C2_0 * y;
  G[3 * 6 + 0] = -2.f * SH_C2_2 * x;
  G[3 * 6 + 1] = -2.f * SH_C2_2 * y;
  G[3 * 6 + 2] = 4.f * SH_C2_2 * z;
  G[3 * 7 + 0] = -SH_C2_0 * z;
  G[3 * 7 + 2] = -SH_C2_0 * x;
  G[3 * 8 + 0] = 2.f * SH_C2_4 * x;
  G[3 * 8 + 1] = -2.f * SH_C2_4 * y;
  if (nb <= 9) return;
  G[3 * 9 + 0] = -6.f * SH_C3_0 * x * y;
  G[3 * 9 + 1] = -SH_C3_0 * (3.f * xx - (ref_quirk ? 2.f : 3.f) * yy);
  G[3 * 10 + 0] = SH_C3_1 * y * z;
  G[3 * 10 + 1] = SH_C3_1 * x * z;
  G[3 * 10 + 2] = SH_C3_1 * x * y;
  G[3 * 11 + 0] = 2.f * SH_C3_2 * x * y;
  G[3 * 11 + 1] = -SH_C3_2 * (4.f * zz - xx - 3.f * yy);
  G[3 * 11 + 2] = -8.f * SH_C3_2 * y * z;
  G[3 * 12 + 0] = -6.f * SH_C3_3 * x * z;
  G[3 * 12 + 1] = -6.f * SH_C3_3 * y * z;
  G[3 * 12 + 2] = SH_C3_3 * (6.f * zz - 3.f * xx - 3.f * yy);
  G[3 * 13 + 0] = -SH_C3_2 * (4.f * zz - 3.f * xx - yy);
  G[3 * 13 + 1] = 2.f * SH_C3_2 * x * y;
  G[3 * 13 + 2] = -8.f * SH_C3_2 * x * z;
  G[3 * 14 + 0] = 2.f * SH_C3_5 * x * z;
  G[3 * 14 + 1] = -2.f * SH_C3_5 * y * z;
  G[3 * 14 + 2] = SH_C3_5 * (xx - yy);
  G[3 * 15 + 0] = -SH_C3_0 * (3.f * xx - 3.f * yy);
  G[3 * 15 + 1] = 6.f * SH_C3_0 * x * y;
}

// Palette weights from full SH coefficients c[l*K + k] (band-major; nb
// bands in {1,4,9,16}): acc_k = sum_l Y_l c[l*K + k], summed band by band as
// the reference groups its sums (gsplatcu/kernel.cu:694-710).  `load(idx)`
// returns coefficient idx as float.
template <int K, typename Loader>
__device__ __forceinline__ void sh_weights_full(Loader load, int nb, const float* Y, float* acc) {
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = Y[0] * load(k);
  // band-by-band accumulation, as the reference groups its sums
  if (nb > 1) {
#pragma unroll
    for (int k = 0; k < K; ++k)
      acc[k] += Y[1] * load(K + k) + Y[2] * load(2 * K + k) + Y[3] * load(3 * K + k);
    if (nb > 4) {
#pragma unroll
      for (int k = 0; k < K; ++k)
        acc[k] += Y[4] * load(4 * K + k) + Y[5] * load(5 * K + k) + Y[6] * load(6 * K + k) +
                  Y[7] * load(7 * K + k) + Y[8] * load(8 * K + k);
      if (nb > 9) {
#pragma unroll
        for (int k = 0; k < K; ++k)
          acc[k] += Y[9] * load(9 * K + k) + Y[10] * load(10 * K + k) +
                    Y[11] * load(11 * K + k) + Y[12] * load(12 * K + k) +
                    Y[13] * load(13 * K + k) + Y[14] * load(14 * K + k) +
                    Y[15] * load(15 * K + k);
      }
    }
  }
}

// Rank-R low-rank weights (sh2Weight_fast generalised, gsplatcu/kernel.cu:884-987):
// w_k = C0 dc_k + sum_l C[g/Q][g%Q] Y_{l+1}, g = l*K + k, C = A B with
// a = A [P,R] and b = B [R,Q] row-major.  Summation order fixed: each
// coefficient over r, then over l, then added to the DC term.
// The factors may be FP32 or BF16 (shared memory or registers); the
// arithmetic is FP32 either way.
__device__ __forceinline__ float as_f32(float v) { return v; }
__device__ __forceinline__ float as_f32(__nv_bfloat16 v) { return __bfloat162float(v); }

template <int K, int P, int Q, int R, typename S>
__device__ __forceinline__ void lowrank_weights(const S* dc, const S* a, const S* b,
                                                const float* Y, float* wk) {
  constexpr int L = P * Q / K;
#pragma unroll
  for (int k = 0; k < K; ++k) wk[k] = SH_C0 * as_f32(dc[k]);
  if (L > 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      float acc = 0.f;
#pragma unroll
      for (int l = 0; l < L; ++l) {
        const int g = l * K + k, row = g / Q, col = g % Q;
        float coef = as_f32(a[row * R]) * as_f32(b[col]);
#pragma unroll
        for (int r = 1; r < R; ++r) coef += as_f32(a[row * R + r]) * as_f32(b[r * Q + col]);
        acc += coef * Y[l + 1];
      }
      wk[k] += acc;
    }
  }
}

// ------------------------------------------------------------ Jacobians
// Computed in the scalar type T: float for the operators' Jacobian outputs,
// double in the adjoint's geometry chain (in FP32 that chain's rotation and
// scale gradients lost up to 3e-4 relative to rounding).
// d Sigma_(rc) / d q_j and / d s_j for Sigma = M M^T, M = R(q) diag(s).
template <typename T>
__device__ __forceinline__ void cov3d_jacobians(float4 q, float3 s, const T* M, const T* R,
                                                T* dq /*6x4*/, T* ds /*6x3*/) {
  const T w = q.x, x = q.y, y = q.z, z = q.w;
  // dR_ab / dq_j (rows a*3+b)
  const T dR[9][4] = {{T(0), T(0), -T(4) * y, -T(4) * z},
                      {-T(2) * z, T(2) * y, T(2) * x, -T(2) * w},
                      {T(2) * y, T(2) * z, T(2) * w, T(2) * x},
                      {T(2) * z, T(2) * y, T(2) * x, T(2) * w},
                      {T(0), -T(4) * x, T(0), -T(4) * z},
                      {-T(2) * x, -T(2) * w, T(2) * z, T(2) * y},
                      {-T(2) * y, T(2) * z, -T(2) * w, T(2) * x},
                      {T(2) * x, T(2) * w, T(2) * z, T(2) * y},
                      {T(0), -T(4) * x, -T(4) * y, T(0)}};
  const T sv[3] = {s.x, s.y, s.z};
  const int sym[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
#pragma unroll
  for (int u = 0; u < 6; ++u) {
    const int r = sym[u][0], c = sym[u][1];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      T acc = T(0);
#pragma unroll
      for (int b = 0; b < 3; ++b)
        acc += (M[3 * c + b] * dR[3 * r + b][j] + M[3 * r + b] * dR[3 * c + b][j]) * sv[b];
      dq[4 * u + j] = acc;
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) ds[3 * u + j] = M[3 * c + j] * R[3 * r + j] + M[3 * r + j] * R[3 * c + j];
  }
}

// Jacobians of cov2d = (Sigma'_00 + .3, Sigma'_01, Sigma'_11 + .3) w.r.t. the 6
// unique entries of Sigma and the camera-space centre (clamp not
// differentiated, as in the reference).  M = J Rcw.
template <typename T>
__device__ __forceinline__ void cov2d_jacobians(const T* cov3, const T* M, const T* Rcw, T x, T y,
                                                T z, T fx, T fy, T* d3 /*3x6*/,
                                                T* dp /*3x3*/) {
  const int sym[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  const int out[3][2] = {{0, 0}, {0, 1}, {1, 1}};
#pragma unroll
  for (int o = 0; o < 3; ++o)
#pragma unroll
    for (int u = 0; u < 6; ++u) {
      const int a = out[o][0], b = out[o][1], k = sym[u][0], l = sym[u][1];
      T v = M[3 * a + k] * M[3 * b + l];
      if (k != l) v += M[3 * a + l] * M[3 * b + k];
      d3[6 * o + u] = v;
    }
  const T S[9] = {cov3[0], cov3[1], cov3[2], cov3[1], cov3[3], cov3[4], cov3[2], cov3[4], cov3[5]};
  T dm[3][6];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T sm0 = S[3 * c] * M[0] + S[3 * c + 1] * M[1] + S[3 * c + 2] * M[2];
    const T sm1 = S[3 * c] * M[3] + S[3 * c + 1] * M[4] + S[3 * c + 2] * M[5];
    dm[0][c] = T(2) * sm0;
    dm[0][3 + c] = T(0);
    dm[1][c] = sm1;
    dm[1][3 + c] = sm0;
    dm[2][c] = T(0);
    dm[2][3 + c] = T(2) * sm1;
  }
  const T zi2 = T(1) / (z * z), zi3 = zi2 / z;
  T dmp[6][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    dmp[c][0] = -fx * Rcw[6 + c] * zi2;
    dmp[c][1] = T(0);
    dmp[c][2] = -fx * Rcw[c] * zi2 + T(2) * fx * Rcw[6 + c] * x * zi3;
    dmp[3 + c][0] = T(0);
    dmp[3 + c][1] = -fy * Rcw[6 + c] * zi2;
    dmp[3 + c][2] = -fy * Rcw[3 + c] * zi2 + T(2) * fy * Rcw[6 + c] * y * zi3;
  }
#pragma unroll
  for (int o = 0; o < 3; ++o)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      T acc = T(0);
#pragma unroll
      for (int m = 0; m < 6; ++m) acc += dm[o][m] * dmp[m][j];
      dp[3 * o + j] = acc;
    }
}

// d dir / d pw = I/|d| - d d^T/|d|^3 (symmetric 3x3).
__device__ __forceinline__ void dir_jacobian(const float* nd, float ninv, float* J) {
  const float n3 = ninv * ninv * ninv;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) J[3 * r + c] = -nd[r] * nd[c] * n3 + (r == c ? ninv : 0.f);
}

}  // namespace gsb
