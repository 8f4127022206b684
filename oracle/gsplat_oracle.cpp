// CPU oracle for the palette-weight Gaussian rasterizer -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, from scratch and in scalar C++, the arithmetic of the
// reference CUDA extension `gsplatcu` (ReparamGS-Palette), so that the B200
// kernels can be checked against it.  Nothing in the product links or calls
// this code: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg load it, and only as the checker / the timed CPU baseline.
//
// Every routine is a template on the arithmetic type `R`:
//   * R = float  mirrors the reference's FP32 operation order, so that tile
//                lists, sort order and ranges can be compared bit-for-bit
//                given identical projected inputs;
//   * R = double is the FP64 oracle used for error tables and central finite
//                differences.
// Exported entry points carry the suffix _f32 / _f64.
//
// Parity pin: this restatement is checked against golden vectors produced by
// running the reference extension itself (tests/golden/, generated by
// tests/golden/make_golden.py on a B200).  The reference ships no tests or
// golden vectors of its own.
//
// Reference citations are to files inside the ReparamGS-Palette project.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------- constants
// gsplatcu/kernel.cu:10-12 and gsplatcu/common.cuh:13-14
constexpr int kTile = 16;
constexpr double kMinDepth = 0.2;
constexpr double kAlphaMax = 0.99;
constexpr double kAlphaMin = 0.002;
constexpr double kTransMin = 0.0001;

// Real spherical-harmonic basis constants, l <= 3 (gsplatcu/common.cuh:29-44).
// These are the standard normalisation constants of the real SH basis.
constexpr double C0 = 0.28209479177387814;
constexpr double C1 = 0.4886025119029199;
constexpr double C2_0 = 1.0925484305920792;
constexpr double C2_2 = 0.31539156525252005;
constexpr double C2_4 = 0.5462742152960396;
constexpr double C3_0 = 0.5900435899266435;
constexpr double C3_1 = 2.890611442640554;
constexpr double C3_2 = 0.4570457994644658;
constexpr double C3_3 = 0.3731763325901154;
constexpr double C3_5 = 1.445305721320277;

// ------------------------------------------------------------ thread pool
int g_threads = 0;

int n_threads() {
  if (g_threads > 0) return g_threads;
  const char* e = std::getenv("ORACLE_THREADS");
  if (e && std::atoi(e) > 0) return std::atoi(e);
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// Split [0, n) into contiguous chunks handed out dynamically to worker threads.
void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)>& fn,
                  int64_t grain = 256) {
  int nt = n_threads();
  if (nt <= 1 || n <= grain) {
    fn(0, n);
    return;
  }
  std::atomic<int64_t> next{0};
  auto work = [&]() {
    for (;;) {
      int64_t b = next.fetch_add(grain);
      if (b >= n) break;
      fn(b, std::min(n, b + grain));
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

// GPU-style saturating float -> int conversions (cvt.rzi.s32/u32.f32):
// NaN -> 0, out-of-range values clamp to the type's limits.
int32_t f2i_rz(float v) {
  if (std::isnan(v)) return 0;
  if (v >= 2147483648.0f) return INT32_MAX;
  if (v <= -2147483648.0f) return INT32_MIN;
  return (int32_t)v;
}
int32_t f2i_rz(double v) {
  if (std::isnan(v)) return 0;
  if (v >= 2147483648.0) return INT32_MAX;
  if (v <= -2147483648.0) return INT32_MIN;
  return (int32_t)v;
}
uint32_t f2u_rz(double v) {
  if (std::isnan(v) || v <= 0.0) return 0u;
  if (v >= 4294967296.0) return UINT32_MAX;
  return (uint32_t)v;
}

// ================================================================ geometry

// Multiply-add with one rounding in the FP32 instantiation: the reference
// build's FP32 results follow a fixed pattern of fused multiply-adds (which
// product of each sum is fused and which is rounded on its own was pinned by
// reproducing its outputs bit for bit from its inputs); the FP64 oracle
// evaluates the same expressions unfused (the file is built with
// -ffp-contract=off, so nothing else is fused).
inline float fmadd(float a, float b, float c) { return std::fmaf(a, b, c); }
inline double fmadd(double a, double b, double c) { return a * b + c; }

// a0 b0 + a1 b1 + a2 b2 from zero in index order, each later product fused.
template <typename R>
R dot3_fused(R a0, R a1, R a2, R b0, R b1, R b2) {
  return fmadd(a2, b2, fmadd(a1, b1, a0 * b0));
}

// Mahalanobis form qa dx^2 + qc dy^2 + 2 qb dx dy (gsplatcu/common.cuh:89-92)
// in the reference build's FP32 order: the qc term rounded alone, the qa
// term fused onto it, the cross term fused last.
template <typename R>
R maha_form(R qa, R qb, R qc, R dx, R dy) {
  return fmadd(R(2) * qb * dx, dy, fmadd(qa * dx, dx, qc * dy * dy));
}



// gsplatcu/kernel.cu:618-663 (project).  pc = Rcw*pw + tcw; depth = -1 when
// z < 0.2 (us/pcs are then left untouched); u = f*xy/z + c.
template <typename R>
void project(int64_t n, const R* pws, const R* Rcw, const R* tcw, R fx, R fy, R cx, R cy,
             R* us, R* pcs, R* depths, R* du_dpcs) {
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      const R* p = pws + 3 * i;
      R pc[3];
      for (int r = 0; r < 3; ++r)
        pc[r] = dot3_fused(Rcw[3 * r], Rcw[3 * r + 1], Rcw[3 * r + 2], p[0], p[1], p[2]) + tcw[r];
      if (pc[2] < (R)kMinDepth) {
        depths[i] = R(-1);
        continue;
      }
      R zi = R(1) / pc[2];
      R zi2 = zi * zi;
      R xf = pc[0] * fx, yf = pc[1] * fy;
      us[2 * i] = fmadd(xf, zi, cx);
      us[2 * i + 1] = fmadd(yf, zi, cy);
      pcs[3 * i] = pc[0];
      pcs[3 * i + 1] = pc[1];
      pcs[3 * i + 2] = pc[2];
      depths[i] = pc[2];
      if (du_dpcs) {  // [2,3]; entries 1 and 3 stay zero
        du_dpcs[6 * i + 0] = fx * zi;
        du_dpcs[6 * i + 2] = -xf * zi2;
        du_dpcs[6 * i + 4] = fy * zi;
        du_dpcs[6 * i + 5] = -yf * zi2;
      }
    }
  });
}

// Rotation matrix of an (unnormalised) quaternion (w, x, y, z), row-major.
template <typename R>
void quat_to_rot(const R* q, R* Rm) {
  R w = q[0], x = q[1], y = q[2], z = q[3];
  R yy = y * y, zz = z * z, xz = x * z, xw = x * w, zw = z * w;
  Rm[0] = R(1) - R(2) * (yy + zz);
  Rm[1] = R(2) * fmadd(x, y, -zw);
  Rm[2] = R(2) * fmadd(y, w, xz);
  Rm[3] = R(2) * fmadd(x, y, zw);
  Rm[4] = R(1) - R(2) * fmadd(x, x, zz);
  Rm[5] = R(2) * fmadd(y, z, -xw);
  Rm[6] = R(2) * fmadd(-y, w, xz);
  Rm[7] = R(2) * fmadd(y, z, xw);
  Rm[8] = R(1) - R(2) * fmadd(x, x, yy);
}

// d R_ab / d(w,x,y,z) for the map above, as a [9][4] table.
template <typename R>
void drot_dquat(const R* q, R (*d)[4]) {
  R w = q[0], x = q[1], y = q[2], z = q[3];
  R t[9][4] = {{0, 0, -4 * y, -4 * z},       {-2 * z, 2 * y, 2 * x, -2 * w},
               {2 * y, 2 * z, 2 * w, 2 * x}, {2 * z, 2 * y, 2 * x, 2 * w},
               {0, -4 * x, 0, -4 * z},       {-2 * x, -2 * w, 2 * z, 2 * y},
               {-2 * y, 2 * z, -2 * w, 2 * x}, {2 * x, 2 * w, 2 * z, 2 * y},
               {0, -4 * x, -4 * y, 0}};
  std::memcpy(d, t, sizeof(t));
}

// Upper triangle index pairs of a symmetric 3x3 in the order (00,01,02,11,12,22).
constexpr int kSym3[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};

// gsplatcu/kernel.cu:422-501 (computeCov3D).  Sigma = M M^T with
// M = R(q) diag(s); skipped (left at zero) when depth < 0.2.  Jacobians are
// [6,4] w.r.t. (w,x,y,z) and [6,3] w.r.t. the scales.
template <typename R>
void cov3d(int64_t n, const R* rots, const R* scales, const R* depths, R* cov3ds, R* drot,
           R* dscale) {
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      if (depths[i] < (R)kMinDepth) continue;
      const R* q = rots + 4 * i;
      const R* s = scales + 3 * i;
      R Rm[9], M[9];
      quat_to_rot(q, Rm);
      for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) M[3 * a + c] = Rm[3 * a + c] * s[c];
      for (int u = 0; u < 6; ++u) {
        int r = kSym3[u][0], c = kSym3[u][1];
        cov3ds[6 * i + u] = dot3_fused(M[3 * r], M[3 * r + 1], M[3 * r + 2], M[3 * c],
                                       M[3 * c + 1], M[3 * c + 2]);
      }
      if (drot && dscale) {
        R dR[9][4];
        drot_dquat(q, dR);
        // dSigma_rc / dM_ab = delta_ra M_cb + delta_ca M_rb
        for (int u = 0; u < 6; ++u) {
          int r = kSym3[u][0], c = kSym3[u][1];
          for (int j = 0; j < 4; ++j) {
            R acc = 0;
            for (int bb = 0; bb < 3; ++bb) {
              // dM_rb/dq_j = dR_rb/dq_j * s_b
              acc += M[3 * c + bb] * dR[3 * r + bb][j] * s[bb];
              acc += M[3 * r + bb] * dR[3 * c + bb][j] * s[bb];
            }
            drot[24 * i + 4 * u + j] = acc;
          }
          for (int j = 0; j < 3; ++j) {
            // dM_ab/ds_j = R_ab delta_bj
            dscale[18 * i + 3 * u + j] = M[3 * c + j] * Rm[3 * r + j] + M[3 * r + j] * Rm[3 * c + j];
          }
        }
      }
    }
  });
}

// gsplatcu/kernel.cu:508-611 (computeCov2D) with tan_fov = W/(2 fx), H/(2 fy)
// (gsplatcu/gausplat.cu:357-358).  Sigma' = M Sigma M^T, M = J Rcw, where J is
// the perspective Jacobian at the frustum-clamped point; +0.3 on the diagonal.
template <typename R>
void cov2d(int64_t n, const R* cov3ds, const R* pcs, const R* Rcw, const R* depths, R fx, R fy,
           R tanx, R tany, R* cov2ds, R* dcov3d, R* dpc) {
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      if (depths[i] < (R)kMinDepth) continue;
      R x = pcs[3 * i], y = pcs[3 * i + 1], z = pcs[3 * i + 2];
      const R* S6 = cov3ds + 6 * i;
      R limx = R(1.3) * tanx, limy = R(1.3) * tany;
      x = std::min(limx, std::max(-limx, x / z)) * z;
      y = std::min(limy, std::max(-limy, y / z)) * z;
      R z2 = z * z;
      R J[6] = {fx / z, 0, -(fx * x) / z2, 0, fy / z, -(fy * y) / z2};
      R M[6];
      for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c)
          M[3 * r + c] = dot3_fused(J[3 * r], J[3 * r + 1], J[3 * r + 2], Rcw[c], Rcw[3 + c],
                                    Rcw[6 + c]);
      R S[9] = {S6[0], S6[1], S6[2], S6[1], S6[3], S6[4], S6[2], S6[4], S6[5]};
      // M Sigma: only the last product of entry (0,0) is fused; every other
      // entry rounds its three products before summing them
      R MS[6];
      for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c)
          MS[3 * r + c] = (M[3 * r] * S[c] + M[3 * r + 1] * S[3 + c]) + M[3 * r + 2] * S[6 + c];
      MS[0] = fmadd(M[2], S[6], M[0] * S[0] + M[1] * S[3]);
      R s00 = dot3_fused(MS[0], MS[1], MS[2], M[0], M[1], M[2]);
      R s01 = dot3_fused(MS[0], MS[1], MS[2], M[3], M[4], M[5]);
      R s11 = dot3_fused(MS[3], MS[4], MS[5], M[3], M[4], M[5]);
      cov2ds[3 * i] = s00 + R(0.3);
      cov2ds[3 * i + 1] = s01;
      cov2ds[3 * i + 2] = s11 + R(0.3);
      if (dcov3d && dpc) {
        // d cov2d / d Sigma (unique entries): d Sigma'_ij / d Sigma_kl summed over
        // the symmetric pair.
        const int out[3][2] = {{0, 0}, {0, 1}, {1, 1}};
        for (int o = 0; o < 3; ++o) {
          int a = out[o][0], bq = out[o][1];
          for (int u = 0; u < 6; ++u) {
            int k = kSym3[u][0], l = kSym3[u][1];
            R v = M[3 * a + k] * M[3 * bq + l];
            if (k != l) v += M[3 * a + l] * M[3 * bq + k];
            dcov3d[18 * i + 6 * o + u] = v;
          }
        }
        // d cov2d / d M  (rows: 00, 01, 11; columns: M00..M02, M10..M12)
        R dm[3][6] = {};
        for (int c = 0; c < 3; ++c) {
          R sm0 = S[3 * c] * M[0] + S[3 * c + 1] * M[1] + S[3 * c + 2] * M[2];  // (Sigma M0^T)_c
          R sm1 = S[3 * c] * M[3] + S[3 * c + 1] * M[4] + S[3 * c + 2] * M[5];  // (Sigma M1^T)_c
          dm[0][c] = 2 * sm0;
          dm[1][c] = sm1;
          dm[1][3 + c] = sm0;
          dm[2][3 + c] = 2 * sm1;
        }
        // d M / d pc (the clamp is not differentiated, as in the reference)
        R zi2 = R(1) / (z * z), zi3 = zi2 / z;
        R dmp[6][3] = {};
        for (int c = 0; c < 3; ++c) {
          dmp[c][0] = -fx * Rcw[6 + c] * zi2;
          dmp[c][2] = -fx * Rcw[c] * zi2 + 2 * fx * Rcw[6 + c] * x * zi3;
          dmp[3 + c][1] = -fy * Rcw[6 + c] * zi2;
          dmp[3 + c][2] = -fy * Rcw[3 + c] * zi2 + 2 * fy * Rcw[6 + c] * y * zi3;
        }
        for (int o = 0; o < 3; ++o)
          for (int j = 0; j < 3; ++j) {
            R acc = 0;
            for (int m = 0; m < 6; ++m) acc += dm[o][m] * dmp[m][j];
            dpc[9 * i + 3 * o + j] = acc;
          }
      }
    }
  });
}

// gsplatcu/kernel.cu:379-415 (inverseCov2D).  No epsilon: a NaN 1/det marks the
// Gaussian bad (depth := -1, in place).  areas = ceil(3 sqrt|diag|).
template <typename R>
void inverse_cov2d(int64_t n, const R* cov2ds, R* depths, R* cinv, int32_t* areas, R* dcinv) {
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      if (depths[i] < (R)kMinDepth) continue;
      R a = cov2ds[3 * i], bb = cov2ds[3 * i + 1], c = cov2ds[3 * i + 2];
      R det_inv = R(1) / fmadd(a, c, -(bb * bb));
      if (std::isnan(det_inv)) {
        depths[i] = R(-1);
        continue;
      }
      cinv[3 * i] = det_inv * c;
      cinv[3 * i + 1] = -det_inv * bb;
      cinv[3 * i + 2] = det_inv * a;
      areas[2 * i] = f2i_rz(std::ceil(R(3) * std::sqrt(std::abs(a))));
      areas[2 * i + 1] = f2i_rz(std::ceil(R(3) * std::sqrt(std::abs(c))));
      if (dcinv) {
        R d2 = det_inv * det_inv;
        R* J = dcinv + 9 * i;
        J[0] = -c * c * d2;
        J[1] = 2 * bb * c * d2;
        J[2] = -a * c * d2 + det_inv;
        J[3] = bb * c * d2;
        J[4] = -2 * bb * bb * d2 - det_inv;
        J[5] = a * bb * d2;
        J[6] = -a * c * d2 + det_inv;
        J[7] = 2 * a * bb * d2;
        J[8] = -a * a * d2;
      }
    }
  });
}

// ===================================================== spherical harmonics

// Real SH basis Y_lm(dir) for l <= 3 in the band-major order used by the
// reference (gsplatcu/kernel.cu:712-763): Y[0] = C0, Y[1..3] = order 1, ...
template <typename R>
void sh_basis(R x, R y, R z, int nb, R* Y) {
  Y[0] = (R)C0;
  if (nb <= 1) return;
  Y[1] = -(R)C1 * y;
  Y[2] = (R)C1 * z;
  Y[3] = -(R)C1 * x;
  if (nb <= 4) return;
  R xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  Y[4] = (R)C2_0 * xy;
  Y[5] = -(R)C2_0 * yz;
  Y[6] = (R)C2_2 * (R(2) * zz - xx - yy);
  Y[7] = -(R)C2_0 * xz;
  Y[8] = (R)C2_4 * (xx - yy);
  if (nb <= 9) return;
  Y[9] = -(R)C3_0 * y * (R(3) * xx - yy);
  Y[10] = (R)C3_1 * xy * z;
  Y[11] = -(R)C3_2 * y * (R(4) * zz - xx - yy);
  Y[12] = (R)C3_3 * z * (R(2) * zz - R(3) * xx - R(3) * yy);
  Y[13] = -(R)C3_2 * x * (R(4) * zz - xx - yy);
  Y[14] = (R)C3_5 * z * (xx - yy);
  Y[15] = -(R)C3_0 * x * (xx - R(3) * yy);
}

// dY_lm / d(dir) as a [16][3] table.  `ref_quirk` reproduces the reference's
// d Y_9 / d y = C3_0 (3x^2 - 2y^2) (gsplatcu/kernel.cu:840); the true
// derivative is C3_0 (3x^2 - 3y^2) (sign folded into the constant).
template <typename R>
void sh_basis_grad(R x, R y, R z, int nb, bool ref_quirk, R (*G)[3]) {
  for (int l = 0; l < 16; ++l) G[l][0] = G[l][1] = G[l][2] = 0;
  if (nb <= 1) return;
  G[1][1] = -(R)C1;
  G[2][2] = (R)C1;
  G[3][0] = -(R)C1;
  if (nb <= 4) return;
  R xx = x * x, yy = y * y, zz = z * z;
  G[4][0] = (R)C2_0 * y;
  G[4][1] = (R)C2_0 * x;
  G[5][1] = -(R)C2_0 * z;
  G[5][2] = -(R)C2_0 * y;
  G[6][0] = -(R)C2_2 * 2 * x;
  G[6][1] = -(R)C2_2 * 2 * y;
  G[6][2] = (R)C2_2 * 4 * z;
  G[7][0] = -(R)C2_0 * z;
  G[7][2] = -(R)C2_0 * x;
  G[8][0] = (R)C2_4 * 2 * x;
  G[8][1] = -(R)C2_4 * 2 * y;
  if (nb <= 9) return;
  G[9][0] = -(R)C3_0 * 6 * x * y;
  G[9][1] = -(R)C3_0 * (R(3) * xx - (ref_quirk ? R(2) : R(3)) * yy);
  G[10][0] = (R)C3_1 * y * z;
  G[10][1] = (R)C3_1 * x * z;
  G[10][2] = (R)C3_1 * x * y;
  G[11][0] = (R)C3_2 * 2 * x * y;
  G[11][1] = -(R)C3_2 * (R(4) * zz - xx - R(3) * yy);
  G[11][2] = -(R)C3_2 * 8 * y * z;
  G[12][0] = -(R)C3_3 * 6 * x * z;
  G[12][1] = -(R)C3_3 * 6 * y * z;
  G[12][2] = (R)C3_3 * (R(6) * zz - R(3) * xx - R(3) * yy);
  G[13][0] = -(R)C3_2 * (R(4) * zz - R(3) * xx - yy);
  G[13][1] = (R)C3_2 * 2 * x * y;
  G[13][2] = -(R)C3_2 * 8 * x * z;
  G[14][0] = (R)C3_5 * 2 * x * z;
  G[14][1] = -(R)C3_5 * 2 * y * z;
  G[14][2] = (R)C3_5 * (xx - yy);
  G[15][0] = -(R)C3_0 * (R(3) * xx - R(3) * yy);
  G[15][1] = (R)C3_0 * 6 * x * y;
}

// Unit view direction (pw - twc)/|pw - twc| and d dir / d pw.
template <typename R>
void view_dir(const R* pw, const R* twc, R* dir, R* ddir /*3x3 or null*/) {
  R d[3] = {pw[0] - twc[0], pw[1] - twc[1], pw[2] - twc[2]};
  R ninv = R(1) / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (int r = 0; r < 3; ++r) dir[r] = d[r] * ninv;
  if (ddir) {
    R n3 = ninv * ninv * ninv;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) ddir[3 * r + c] = -d[r] * d[c] * n3 + (r == c ? ninv : R(0));
  }
}

// gsplatcu/kernel.cu:670-870 (sh2Weight) and kernel.cu:1040-1169 (sh2Color,
// the same map with K = 3).  feat_k = sum_lm Y_lm * shs[i][lm*K + k]
// (band-major).  Evaluated for every Gaussian (no depth test).  Jacobians:
// dfeat/dshs = Y_lm [N,1,nb] and dfeat/dpw [N,K,3].
template <typename R>
void sh2feat(int64_t n, const R* shs, const R* pws, const R* twc, int nb, int K, R* feat,
             R* dshs, R* dpws, bool ref_quirk) {
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      R dir[3] = {0, 0, 0}, ddir[9];
      if (nb > 1) view_dir(pws + 3 * i, twc, dir, ddir);
      R Y[16];
      sh_basis(dir[0], dir[1], dir[2], nb, Y);
      const R* c = shs + (int64_t)i * nb * K;
      for (int k = 0; k < K; ++k) {
        R acc = 0;
        for (int l = 0; l < nb; ++l) acc += Y[l] * c[l * K + k];
        feat[i * K + k] = acc;
      }
      if (dshs && dpws) {
        for (int l = 0; l < nb; ++l) dshs[i * nb + l] = Y[l];
        R G[16][3];
        sh_basis_grad(dir[0], dir[1], dir[2], nb, ref_quirk, G);
        for (int k = 0; k < K; ++k) {
          R dd[3] = {0, 0, 0};
          for (int l = 1; l < nb; ++l)
            for (int r = 0; r < 3; ++r) dd[r] += G[l][r] * c[l * K + k];
          for (int j = 0; j < 3; ++j) {
            R acc = 0;
            if (nb > 1)
              for (int r = 0; r < 3; ++r) acc += dd[r] * ddir[3 * r + j];
            dpws[(i * K + k) * 3 + j] = acc;
          }
        }
      }
    }
  });
}

// gsplatcu/kernel.cu:884-987 (sh2Weight_fast), generalised from rank 1 to
// rank r: the L*K higher-order coefficients of Gaussian i, flattened band-
// major (index g = lm*K + k), are the P x Q matrix C = A B with A [P,r],
// B [r,Q] (gsplat/gsmodel.py:90-97 for r = 1):
//   w_k = C0 dc_k + sum_lm C[g / Q][g % Q] Y_lm.
// Outputs dweight_ddc (= C0) and the basis Y_lm (l >= 1) when requested.
template <typename R>
void sh2weight_lowrank(int64_t n, const R* dc, const R* A, const R* B, const R* pws, const R* twc,
                       int K, int P, int Q, int rank, int L, R* w, R* ddc, R* ylm) {
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      for (int k = 0; k < K; ++k) {
        w[i * K + k] = (R)C0 * dc[i * K + k];
        if (ddc) ddc[i * K + k] = (R)C0;
      }
      if (L == 0) continue;
      R dir[3];
      view_dir(pws + 3 * i, twc, dir, (R*)nullptr);
      R Y[16];
      sh_basis(dir[0], dir[1], dir[2], L + 1, Y);
      if (ylm)
        for (int l = 0; l < L; ++l) ylm[i * L + l] = Y[l + 1];
      const R* a = A + (int64_t)i * P * rank;
      const R* bm = B + (int64_t)i * rank * Q;
      for (int k = 0; k < K; ++k) {
        R acc = 0;
        for (int l = 0; l < L; ++l) {
          int g = l * K + k, row = g / Q, col = g % Q;
          R cval = 0;
          for (int r = 0; r < rank; ++r) cval += a[row * rank + r] * bm[r * Q + col];
          acc += cval * Y[l + 1];
        }
        w[i * K + k] += acc;
      }
    }
  });
}

// gsplatcu/kernel.cu:994-1032 (sh2Weight_fast_B), rank r:
//   dA[row][r] += dw_k Y_lm B[r][col],  dB[r][col] += dw_k Y_lm A[row][r].
template <typename R>
void sh2weight_lowrank_b(int64_t n, const R* A, const R* B, const R* ylm, const R* dw, int K, int P,
                         int Q, int rank, int L, R* dA, R* dB) {
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      const R* a = A + (int64_t)i * P * rank;
      const R* bm = B + (int64_t)i * rank * Q;
      R* da = dA + (int64_t)i * P * rank;
      R* db = dB + (int64_t)i * rank * Q;
      for (int k = 0; k < K; ++k) {
        R g0 = dw[i * K + k];
        for (int l = 0; l < L; ++l) {
          int g = l * K + k, row = g / Q, col = g % Q;
          R t = g0 * ylm[i * L + l];
          for (int r = 0; r < rank; ++r) {
            da[row * rank + r] += t * bm[r * Q + col];
            db[r * Q + col] += t * a[row * rank + r];
          }
        }
      }
    }
  });
}

// ================================================================= binning

struct Rect {
  uint32_t x0, y0, x1, y1;
};

// gsplatcu/kernel.cu:127-162 (getRects).  Tile rectangle of a Gaussian from
// its centre and 3-sigma extents; an empty rectangle marks it bad
// (depth := -1, areas := 0, in place).  Float arithmetic mirrors the
// reference's FP32 expressions exactly, including DIV_ROUND_UP's
// ((u + r) + 16) - 1 evaluation order.
void rects_and_counts(int64_t n, const float* us, int32_t* areas, float* depths, uint32_t gx,
                      uint32_t gy, Rect* rects, uint32_t* counts) {
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      counts[i] = 0;
      rects[i] = {0, 0, 0, 0};
      if (depths[i] < (float)kMinDepth) continue;
      float ux = us[2 * i], uy = us[2 * i + 1];
      float xs = (float)areas[2 * i], ys = (float)areas[2 * i + 1];
      auto lo = [](float v, uint32_t g) {
        int32_t t = std::max(0, f2i_rz(v / (float)kTile));
        return std::min(g, (uint32_t)t);
      };
      auto hi = [](float v, uint32_t g) {
        float up = (v + (float)kTile) - 1.0f;
        int32_t t = std::max(0, f2i_rz(up / (float)kTile));
        return std::min(g, (uint32_t)t);
      };
      Rect r = {lo(ux - xs, gx), lo(uy - ys, gy), hi(ux + xs, gx), hi(uy + ys, gy)};
      uint32_t cnt = (r.y1 - r.y0) * (r.x1 - r.x0);
      if (cnt == 0) {
        depths[i] = -1.0f;
        areas[2 * i] = 0;
        areas[2 * i + 1] = 0;
        continue;
      }
      rects[i] = r;
      counts[i] = cnt;
    }
  }, 4096);
}

}  // namespace

// ==================================================== compositing (forward)
namespace {

// gsplatcu/kernel.cu:194-372 (draw_color / draw_weight) for K channels.
// Per pixel of each 16x16 tile, Gaussians are visited front to back:
//   alpha' = min(0.99, alpha exp(-max(0, d^T Q d)/2)), skipped if < 0.002;
//   out_k += T alpha' f_k; contrib := 1-based list index of the last blend;
//   T *= (1 - alpha'); the pixel stops once T < 1e-4 (tested after blending).
// Pixel coordinates are the integer pixel index (no +0.5).  Empty tiles keep
// the caller's initial values (final_tau is 0 for weights, 1 for colours).
template <typename R>
void draw(int H, int W, int K, const int32_t* ranges, const int32_t* gsid, const R* us,
          const R* cinv, const R* alphas, const R* feat, R* out, int32_t* contrib, R* final_tau,
          int32_t* blends = nullptr) {
  int gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
  parallel_for((int64_t)gx * gy, [&](int64_t b, int64_t e) {
    std::vector<R> acc(K);
    for (int64_t t = b; t < e; ++t) {
      int32_t s = ranges[2 * t], en = ranges[2 * t + 1];
      if (en - s == 0) continue;
      int tx = (int)(t % gx), ty = (int)(t / gx);
      for (int py = ty * kTile; py < std::min(H, ty * kTile + kTile); ++py)
        for (int px = tx * kTile; px < std::min(W, tx * kTile + kTile); ++px) {
          std::fill(acc.begin(), acc.end(), R(0));
          R T = 1;
          int32_t cont = 0, nblend = 0;
          for (int32_t j = s; j < en; ++j) {
            int32_t g = gsid[j];
            R dx = us[2 * g] - (R)px, dy = us[2 * g + 1] - (R)py;
            const R* q = cinv + 3 * g;
            R maha = std::max(R(0), maha_form(q[0], q[1], q[2], dx, dy));
            R ap = std::min((R)kAlphaMax, alphas[g] * std::exp(R(-0.5) * maha));
            if (ap < (R)kAlphaMin) continue;
            R ta = T * ap;
            for (int k = 0; k < K; ++k) acc[k] += ta * feat[(int64_t)g * K + k];
            cont = j - s + 1;
            ++nblend;
            T *= (R(1) - ap);
            if (T < (R)kTransMin) break;
          }
          int64_t pix = (int64_t)py * W + px;
          for (int k = 0; k < K; ++k) out[(int64_t)k * H * W + pix] = acc[k];
          contrib[pix] = cont;
          final_tau[pix] = T;
          if (blends) blends[pix] = nblend;
        }
    }
  }, 1);
}

// Reverse-mode adjoint of draw() -- gsplatcu/kernel.cu:1176-1379
// (draw_color_B / draw_weight_B) with the final-transmittance term of
// vanilla_3dgs/gsplatcu/kernel.cu:811-972, generalised to K channels.
// Walks each pixel's contributors back to front from `contrib`, recovering
// T by division by (1 - alpha') from the saved final T:
//   dL/df_k      = dL/dout_k T alpha'
//   dL/dalpha'   = sum_k dL/dout_k T (f_k - G_k) - dL/dT_final T_final/(1-alpha')
//   dL/dalpha    = dL/dalpha' g,     dL/du = dL/dalpha' alpha' (-Q d)
//   dL/dQ        = dL/dalpha' alpha' (-d_x^2/2, -d_x d_y, -d_y^2/2)
// where G accumulates the colour behind the current Gaussian.  As in the
// reference, neither the 0.99 clamp nor max(0, .) is differentiated.
// Gradient outputs are accumulated (+=); any may be null.
template <typename R>
inline void atomic_add(R* p, R v) {
  std::atomic_ref<R>(*p).fetch_add(v, std::memory_order_relaxed);
}

template <typename R>
void draw_backward(int H, int W, int K, const int32_t* ranges, const int32_t* gsid, const R* us,
                   const R* cinv, const R* alphas, const R* feat, const R* final_tau,
                   const int32_t* contrib, const R* dout, const R* dT, R* dfeat, R* dalpha, R* du,
                   R* dq) {
  int gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
  int64_t n_tiles = (int64_t)gx * gy;
  // Tiles run in parallel; the per-Gaussian gradient sums they share are
  // accumulated with atomic adds.
  parallel_for(n_tiles, [&](int64_t tb, int64_t te) {
    std::vector<R> G(K), dl(K);
    for (int64_t t = tb; t < te; ++t) {
      int32_t s = ranges[2 * t], en = ranges[2 * t + 1];
      if (en - s == 0) continue;
      int tx = (int)(t % gx), ty = (int)(t / gx);
      for (int py = ty * kTile; py < std::min(H, ty * kTile + kTile); ++py)
        for (int px = tx * kTile; px < std::min(W, tx * kTile + kTile); ++px) {
          int64_t pix = (int64_t)py * W + px;
          for (int k = 0; k < K; ++k) {
            dl[k] = dout[(int64_t)k * H * W + pix];
            G[k] = 0;
          }
          R Tf = final_tau[pix];
          R dTf = dT ? dT[pix] : R(0);
          R T = Tf;
          int32_t top = std::min(contrib[pix], en - s);
          for (int32_t j = s + top - 1; j >= s; --j) {
            int32_t g = gsid[j];
            R dx = us[2 * g] - (R)px, dy = us[2 * g + 1] - (R)py;
            const R* q = cinv + 3 * g;
            R maha = std::max(R(0), maha_form(q[0], q[1], q[2], dx, dy));
            R gg = std::exp(R(-0.5) * maha);
            R ap = std::min((R)kAlphaMax, alphas[g] * gg);
            if (ap < (R)kAlphaMin) continue;
            T = T / (R(1) - ap);
            R dap = 0;
            for (int k = 0; k < K; ++k) {
              R f = feat[(int64_t)g * K + k];
              if (dfeat) atomic_add(dfeat + (int64_t)g * K + k, dl[k] * (ap * T));
              dap += dl[k] * (T * (f - G[k]));
              G[k] = ap * f + (R(1) - ap) * G[k];
            }
            dap += dTf * (-Tf / (R(1) - ap));
            if (dalpha) atomic_add(dalpha + g, dap * gg);
            if (du) {
              atomic_add(du + 2 * g, dap * ((-q[0] * dx - q[1] * dy) * ap));
              atomic_add(du + 2 * g + 1, dap * ((-q[1] * dx - q[2] * dy) * ap));
            }
            if (dq) {
              atomic_add(dq + 3 * g, dap * (R(-0.5) * ap * dx * dx));
              atomic_add(dq + 3 * g + 1, dap * (R(-1) * ap * dx * dy));
              atomic_add(dq + 3 * g + 2, dap * (R(-0.5) * ap * dy * dy));
            }
          }
        }
    }
  }, 1);
}

}  // namespace

// ================================================================ C ABI

#define ORACLE_EXPORT extern "C" __attribute__((visibility("default")))

ORACLE_EXPORT void oracle_set_threads(int n) { g_threads = n; }
ORACLE_EXPORT int oracle_get_threads() { return n_threads(); }

#define DEF_BOTH(NAME, SIG, CALL)        \
  ORACLE_EXPORT void NAME##_f32 SIG(float) { CALL(float) } \
  ORACLE_EXPORT void NAME##_f64 SIG(double) { CALL(double) }

#define SIG_PROJECT(R) \
  (int64_t n, const R* pws, const R* Rcw, const R* tcw, R fx, R fy, R cx, R cy, R* us, R* pcs, R* depths, R* du_dpcs)
#define CALL_PROJECT(R) project<R>(n, pws, Rcw, tcw, fx, fy, cx, cy, us, pcs, depths, du_dpcs);
DEF_BOTH(oracle_project, SIG_PROJECT, CALL_PROJECT)

#define SIG_COV3D(R) \
  (int64_t n, const R* rots, const R* scales, const R* depths, R* cov3ds, R* drot, R* dscale)
#define CALL_COV3D(R) cov3d<R>(n, rots, scales, depths, cov3ds, drot, dscale);
DEF_BOTH(oracle_cov3d, SIG_COV3D, CALL_COV3D)

#define SIG_COV2D(R)                                                                           \
  (int64_t n, const R* cov3ds, const R* pcs, const R* Rcw, const R* depths, R fx, R fy, R tanx, \
   R tany, R* cov2ds, R* dcov3d, R* dpc)
#define CALL_COV2D(R) cov2d<R>(n, cov3ds, pcs, Rcw, depths, fx, fy, tanx, tany, cov2ds, dcov3d, dpc);
DEF_BOTH(oracle_cov2d, SIG_COV2D, CALL_COV2D)

#define SIG_INV(R) (int64_t n, const R* cov2ds, R* depths, R* cinv, int32_t* areas, R* dcinv)
#define CALL_INV(R) inverse_cov2d<R>(n, cov2ds, depths, cinv, areas, dcinv);
DEF_BOTH(oracle_inverse_cov2d, SIG_INV, CALL_INV)

#define SIG_SH(R)                                                                           \
  (int64_t n, const R* shs, const R* pws, const R* twc, int nb, int K, R* feat, R* dshs, R* dpws, \
   int ref_quirk)
#define CALL_SH(R) sh2feat<R>(n, shs, pws, twc, nb, K, feat, dshs, dpws, ref_quirk != 0);
DEF_BOTH(oracle_sh2feat, SIG_SH, CALL_SH)

#define SIG_LR(R)                                                                            \
  (int64_t n, const R* dc, const R* A, const R* B, const R* pws, const R* twc, int K, int P, int Q, \
   int rank, int L, R* w, R* ddc, R* ylm)
#define CALL_LR(R) sh2weight_lowrank<R>(n, dc, A, B, pws, twc, K, P, Q, rank, L, w, ddc, ylm);
DEF_BOTH(oracle_sh2weight_lowrank, SIG_LR, CALL_LR)

#define SIG_LRB(R)                                                                                \
  (int64_t n, const R* A, const R* B, const R* ylm, const R* dw, int K, int P, int Q, int rank, int L, \
   R* dA, R* dB)
#define CALL_LRB(R) sh2weight_lowrank_b<R>(n, A, B, ylm, dw, K, P, Q, rank, L, dA, dB);
DEF_BOTH(oracle_sh2weight_lowrank_b, SIG_LRB, CALL_LRB)

#define SIG_DRAW(R)                                                                              \
  (int H, int W, int K, const int32_t* ranges, const int32_t* gsid, const R* us, const R* cinv, \
   const R* alphas, const R* feat, R* out, int32_t* contrib, R* final_tau)
#define CALL_DRAW(R) draw<R>(H, W, K, ranges, gsid, us, cinv, alphas, feat, out, contrib, final_tau);
DEF_BOTH(oracle_draw, SIG_DRAW, CALL_DRAW)

// Forward compositing (FP32) that also counts, per pixel, the Gaussians
// blended into it (the (pixel, Gaussian) pairs the adjoint revisits).
ORACLE_EXPORT void oracle_draw_count_f32(int H, int W, int K, const int32_t* ranges,
                                         const int32_t* gsid, const float* us, const float* cinv,
                                         const float* alphas, const float* feat, float* out,
                                         int32_t* contrib, float* final_tau, int32_t* blends) {
  draw<float>(H, W, K, ranges, gsid, us, cinv, alphas, feat, out, contrib, final_tau, blends);
}

#define SIG_DRAWB(R)                                                                             \
  (int H, int W, int K, const int32_t* ranges, const int32_t* gsid, const R* us, const R* cinv, \
   const R* alphas, const R* feat, const R* final_tau, const int32_t* contrib, const R* dout,    \
   const R* dT, R* dfeat, R* dalpha, R* du, R* dq)
#define CALL_DRAWB(R)                                                                              \
  draw_backward<R>(H, W, K, ranges, gsid, us, cinv, alphas, feat, final_tau, contrib, dout, dT, \
                   dfeat, dalpha, du, dq);
DEF_BOTH(oracle_draw_backward, SIG_DRAWB, CALL_DRAWB)

// Binning, step 1 (gsplatcu/kernel.cu:127-162 + the inclusive scan of
// gsplatcu/gausplat.cu:199-201): rectangles, per-Gaussian patch counts and
// their inclusive prefix sum.  Updates depths/areas in place exactly as the
// reference does.  Returns the total patch count M.
ORACLE_EXPORT int64_t oracle_bin_count(int64_t n, const float* us, int32_t* areas, float* depths,
                                       int H, int W, uint32_t* rects, uint32_t* counts,
                                       uint32_t* offsets) {
  uint32_t gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
  rects_and_counts(n, us, areas, depths, gx, gy, reinterpret_cast<Rect*>(rects), counts);
  uint32_t run = 0;  // 32-bit, as the reference's uint scan
  for (int64_t i = 0; i < n; ++i) {
    run += counts[i];
    offsets[i] = run;
  }
  return n ? (int64_t)run : 0;
}

// Binning, step 2 (gsplatcu/kernel.cu:96-124 createKeys, the stable
// thrust::sort_by_key of gsplatcu/gausplat.cu:216 and getRanges,
// gsplatcu/kernel.cu:165-187).  Keys are (tile << 32) | uint32(depth * 1000),
// emitted in Gaussian-id order, tiles of one Gaussian row-major; the stable
// sort therefore orders each tile by (quantised depth, Gaussian id).
// `ranges` [T,2] must be zero-initialised by the caller.  getRanges never
// writes the end of the only tile when M == 1; that is reproduced.
ORACLE_EXPORT void oracle_bin_sort(int64_t n, const float* depths, const uint32_t* rects,
                                   const uint32_t* offsets, int H, int W, int64_t M,
                                   int32_t* gsid_out, int32_t* ranges, uint64_t* keys_out) {
  uint32_t gx = (W + kTile - 1) / kTile;
  std::vector<uint64_t> keys(M);
  std::vector<int32_t> vals(M);
  const Rect* R = reinterpret_cast<const Rect*>(rects);
  for (int64_t i = 0; i < n; ++i) {
    float d = depths[i];
    if (d < (float)kMinDepth) continue;
    uint32_t off = i == 0 ? 0 : offsets[i - 1];
    uint32_t dq = f2u_rz((double)(d * 1000.0f));
    for (uint32_t y = R[i].y0; y < R[i].y1; ++y)
      for (uint32_t x = R[i].x0; x < R[i].x1; ++x) {
        keys[off] = ((uint64_t)(y * gx + x) << 32) | dq;
        vals[off] = (int32_t)i;
        ++off;
      }
  }
  std::vector<int64_t> perm(M);
  for (int64_t p = 0; p < M; ++p) perm[p] = p;
  std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });
  for (int64_t p = 0; p < M; ++p) {
    gsid_out[p] = vals[perm[p]];
    if (keys_out) keys_out[p] = keys[perm[p]];
  }
  for (int64_t p = 0; p < M; ++p) {
    uint32_t cur = (uint32_t)(keys[perm[p]] >> 32);
    uint32_t prv = (uint32_t)(keys[perm[p == 0 ? 0 : p - 1]] >> 32);
    if (p == 0)
      ranges[2 * cur] = 0;
    else if (p == M - 1)
      ranges[2 * cur + 1] = (int32_t)M;
    if (prv != cur) {
      ranges[2 * prv + 1] = (int32_t)p;
      ranges[2 * cur] = (int32_t)p;
    }
  }
}

// CIE L*a*b* -> sRGB per pixel (gsplatcu/kernel.cu:1385-1428); L is given in
// [0, 1] and scaled by 100.
ORACLE_EXPORT void oracle_lab2rgb(int H, int W, const float* lab, float* rgb) {
  int64_t P = (int64_t)H * W;
  auto finv = [](float t) {
    const float d = 6.0f / 29.0f;
    return t > d ? t * t * t : 3.0f * d * d * (t - 4.0f / 29.0f);
  };
  auto gam = [](float c) { return c <= 0.0031308f ? 12.92f * c : 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f; };
  for (int64_t p = 0; p < P; ++p) {
    float L = lab[p] * 100.0f, a = lab[P + p], b = lab[2 * P + p];
    float fy = (L + 16.0f) / 116.0f, fx = a / 500.0f + fy, fz = fy - b / 200.0f;
    float X = 0.95047f * finv(fx), Y = 1.0f * finv(fy), Z = 1.08883f * finv(fz);
    float r = std::max(0.0f, std::min(1.0f, 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z));
    float g = std::max(0.0f, std::min(1.0f, -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z));
    float bb = std::max(0.0f, std::min(1.0f, 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z));
    rgb[p] = gam(r);
    rgb[P + p] = gam(g);
    rgb[2 * P + p] = gam(bb);
  }
}
