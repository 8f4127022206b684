// Loss side of a finetune step, fused into one pass over the image: the
// palette colour composite img_c = sum_k palette[k][c] layer_k (compositing
// is linear in the per-Gaussian features, so this equals rendering with the
// baked colours weights . palette), the L1 loss against a target, and its
// adjoint w.r.t. the layer stack and the palette.
#include <algorithm>

#include "gsb_common.cuh"
#include "gsb_internal.h"

namespace gsb {

constexpr int kLossThreads = 256;

template <int K>
__global__ void __launch_bounds__(kLossThreads)
    k_palette_l1(int64_t hw, const float* __restrict__ layer, const float* __restrict__ palette,
                 const float* __restrict__ target, float scale, float* __restrict__ image,
                 float* __restrict__ loss, float* __restrict__ dlayer, float* __restrict__ dpal) {
  pdl_wait();
  constexpr int KC = 3 * K;
  __shared__ float sP[KC];
  __shared__ float red[kLossThreads / 32][KC + 1];
  if (threadIdx.x < KC) sP[threadIdx.x] = palette[threadIdx.x];
  __syncthreads();
  float lsum = 0.f, dp[KC];
#pragma unroll
  for (int j = 0; j < KC; ++j) dp[j] = 0.f;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < hw; p += stride) {
    float l[K], s[3];
#pragma unroll
    for (int k = 0; k < K; ++k) l[k] = layer[k * hw + p];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float v = 0.f;
#pragma unroll
      for (int k = 0; k < K; ++k) v += sP[3 * k + c] * l[k];
      if (image) image[c * hw + p] = v;
      const float d = v - target[c * hw + p];
      lsum += fabsf(d);
      s[c] = d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f);
    }
    if (dlayer)
#pragma unroll
      for (int k = 0; k < K; ++k)
        dlayer[k * hw + p] = scale * (sP[3 * k] * s[0] + sP[3 * k + 1] * s[1] + sP[3 * k + 2] * s[2]);
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) dp[3 * k + c] += l[k] * s[c];
  }
  // block reduction: warp shuffles, then one atomic per block and value
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
#pragma unroll
  for (int j = 0; j < KC; ++j)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dp[j] += __shfl_xor_sync(0xffffffffu, dp[j], o);
  if (lane == 0) {
    red[w][KC] = lsum;
#pragma unroll
    for (int j = 0; j < KC; ++j) red[w][j] = dp[j];
  }
  __syncthreads();
  if (threadIdx.x <= KC) {
    float t = 0.f;
#pragma unroll
    for (int k = 0; k < kLossThreads / 32; ++k) t += red[k][threadIdx.x];
    if (threadIdx.x == KC)
      atomicAdd(loss, t * scale);
    else if (dpal)
      atomicAdd(dpal + threadIdx.x, t * scale);
  }
}

int launch_palette_l1(int K, int H, int W, const float* layer, const float* palette,
                      const float* target, float* image, float* loss, float* dlayer, float* dpal,
                      cudaStream_t st) {
  const int64_t hw = (int64_t)H * W;
  {
    const int rc = launch_zero2(loss, 1, dpal, 3 * K, st);
    if (rc) return rc;
  }
  if (hw == 0) return GSB_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t need = (hw + kLossThreads - 1) / kLossThreads;
  const int grid = (int)std::min<int64_t>(need, (int64_t)sms * 4);
  const float scale = 1.f / (float)(3 * hw);
  switch (K) {
#define GSB_K(KK)                                                                                 \
  case KK:                                                                                        \
    launch_pdl(k_palette_l1<KK>, dim3(grid), dim3(kLossThreads), 0, st, hw, layer, palette,      \
               target, scale, image, loss, dlayer, dpal);                                        \
    break;
    GSB_K(1) GSB_K(2) GSB_K(3) GSB_K(4) GSB_K(5) GSB_K(6) GSB_K(7) GSB_K(8)
#undef GSB_K
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
  return check_launch("palette_l1");
}


// ------------------------------------------------- palette-weight loss
// The finetune step's loss on the rendered weights (finetune.py:356-389),
// per pixel, with the barycentric target of gsplat/gsmodel.py:219-285
// recomputed in the same pass (it depends on the palette, which is being
// learnt):
//   for each tetrahedron i (black, white, c_i, c_{i+1}): coords
//     (beta, gamma, delta) = adj(A_i) C / (det A_i + 1e-12), A_i = [1, c_i, c_{i+1}],
//     alpha = 1 - beta - gamma - delta; a softplus-normalised projection of
//     (alpha, beta, gamma, delta) reconstructs the colour with error err_i;
//   W = sum_i softmax(-err / 1e-9)_i raw_i (raw_i: the coords on their channels);
//   optional clamp: W <- max(W, 0) / max(sum max(W, 0), 1e-8);
//   loss = mean over the K x H x W values of (layer - W)^2 (MSE) or |layer - W|
//   (L1), plus lambda_pos * mean(relu(-layer)).
// Gradients: d/d layer per pixel, and d/d palette through the target (the
// raw coordinates' dependence on A_i, and the softmax term, which is exactly
// zero unless two tetrahedra's errors tie to within ~1e-7).
constexpr float kBaryTau = 1e-9f, kBaryEps = 1e-12f;
constexpr int kGeoThreads = 128;

template <int KC>
struct TetraConst {
  float adj[9], dinv, ainv[9];  // ainv = A^-1 (for the adjoint)
  int i, j;
};

// The softplus values only rank the tetrahedra by reconstruction error (the
// target weights are the exact coordinates), so the fast exp/log intrinsics
// are used; they can change the choice only between near-tied tetrahedra.
__device__ __forceinline__ float softplus_f(float x) {
  return x > 20.f ? x : __logf(1.f + __expf(x));
}
__device__ __forceinline__ float softplus_grad(float x) {
  return x > 20.f ? 1.f : 1.f / (1.f + expf(-x));
}

// Barycentric coordinates x[4] = (alpha, beta, gamma, delta) of colour C in
// one tetrahedron.
template <int KC>
__device__ __forceinline__ void tetra_coords(const TetraConst<KC>& T, const float* C, float* x) {
  float co[3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
    co[r] = (T.adj[3 * r] * C[0] + T.adj[3 * r + 1] * C[1] + T.adj[3 * r + 2] * C[2]) * T.dinv;
  x[1] = co[0];
  x[2] = co[1];
  x[3] = co[2];
  x[0] = 1.f - co[0] - co[1] - co[2];
}

// Forward of one tetrahedron: coords x[4], softplus values, normaliser,
// projection and reconstruction error.
template <int KC>
__device__ __forceinline__ float tetra_forward(const TetraConst<KC>& T, const float* Pi,
                                               const float* Pj, const float* C, float* x, float* sp,
                                               float& den, float* pr, float* rec) {
  tetra_coords<KC>(T, C, x);
  den = kBaryEps;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    sp[k] = softplus_f(x[k]);
    den += sp[k];
  }
  const float rden = 1.f / den;
#pragma unroll
  for (int k = 0; k < 4; ++k) pr[k] = sp[k] * rden;
  float err = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    rec[c] = pr[1] + pr[2] * Pi[c] + pr[3] * Pj[c];
    const float d = rec[c] - C[c];
    err += d * d;
  }
  return err;
}

// Softmax weights of the tetrahedra at temperature kBaryTau (shifted by the
// smallest error) and their coordinates, as the reference computes them.
template <int KC>
__device__ __forceinline__ void bary_weights(const TetraConst<KC>* s_t, const float (*s_p)[3],
                                             const float* C, float* prob, float (*xs)[4]) {
  float err[KC];
#pragma unroll
  for (int i = 0; i < KC; ++i) {
    float sp[4], den, pr[4], rec[3];
    err[i] = tetra_forward<KC>(s_t[i], s_p[i], s_p[(i + 1) % KC], C, xs[i], sp, den, pr, rec);
  }
  float emin = INFINITY;
#pragma unroll
  for (int i = 0; i < KC; ++i) emin = fminf(emin, err[i]);
  float psum = 0.f;
#pragma unroll
  for (int i = 0; i < KC; ++i) {
    prob[i] = expf((emin - err[i]) * (1.f / kBaryTau));
    psum += prob[i];
  }
  const float rpsum = 1.f / psum;
#pragma unroll
  for (int i = 0; i < KC; ++i) prob[i] *= rpsum;
}

// Pixels whose softmax is not one-hot (tetrahedra tied to within ~1e-7 in
// reconstruction error, or non-finite errors) take these two out-of-line
// functions, which keep every tetrahedron's terms; their registers do not
// weigh on the one-hot path.  Data passes through the thread's slots of a
// shared-memory scratch `scr` (stride kGeoThreads).
// Target weights W = sum_i prob_i raw_i -> scr[k].
template <int KC>
__device__ __noinline__ void bary_target_general(const TetraConst<KC>* s_t,
                                                 const float (*s_p)[3], float c0, float c1,
                                                 float c2, float* scr) {
  constexpr int K = KC + 2;
  const float C[3] = {c0, c1, c2};
  float prob[KC], xs[KC][4];
  bary_weights<KC>(s_t, s_p, C, prob, xs);
  float Wb[K];
#pragma unroll
  for (int k = 0; k < K; ++k) Wb[k] = 0.f;
#pragma unroll
  for (int i = 0; i < KC; ++i) {
    Wb[0] += prob[i] * xs[i][0];
    Wb[1] += prob[i] * xs[i][1];
    Wb[i + 2] += prob[i] * xs[i][2];
    Wb[(i + 1) % KC + 2] += prob[i] * xs[i][3];
  }
#pragma unroll
  for (int k = 0; k < K; ++k) scr[k * kGeoThreads] = Wb[k];
}

// Palette gradient of the target given gWb = dL/dW (scr[k]): the raw
// coordinates' path and the softmax path (the reconstruction error's adjoint
// for tetrahedra with a non-zero error gradient).  Writes the 3 KC values
// d/d chroma[i][c] -> scr[3 i + c].
template <int KC>
__device__ __noinline__ void bary_adjoint_general(const TetraConst<KC>* s_t,
                                                  const float (*s_p)[3], float c0, float c1,
                                                  float c2, float* scr) {
  constexpr int K = KC + 2;
  const float C[3] = {c0, c1, c2};
  float prob[KC], xs[KC][4], gWb[K], dP[KC][3];
#pragma unroll
  for (int k = 0; k < K; ++k) gWb[k] = scr[k * kGeoThreads];
#pragma unroll
  for (int i = 0; i < KC; ++i) dP[i][0] = dP[i][1] = dP[i][2] = 0.f;
  bary_weights<KC>(s_t, s_p, C, prob, xs);
  float gprob[KC], gdot = 0.f;
#pragma unroll
  for (int i = 0; i < KC; ++i) {
    const float* x = xs[i];
    gprob[i] = x[0] * gWb[0] + x[1] * gWb[1] + x[2] * gWb[i + 2] + x[3] * gWb[(i + 1) % KC + 2];
    gdot += prob[i] * gprob[i];
  }
#pragma unroll
  for (int i = 0; i < KC; ++i) {
    const float gerr = -prob[i] * (gprob[i] - gdot) * (1.f / kBaryTau);
    if (prob[i] == 0.f && gerr == 0.f) continue;  // contributes nothing
    const TetraConst<KC>& T = s_t[i];
    const int ti = i, tj = (i + 1) % KC;
    const float* Pi = s_p[ti];
    const float* Pj = s_p[tj];
    const float* x = xs[i];
    float gx[4] = {prob[i] * gWb[0], prob[i] * gWb[1], prob[i] * gWb[ti + 2],
                   prob[i] * gWb[tj + 2]};
    if (gerr != 0.f) {  // error path: err = |rec - C|^2
      float xr[4], sp[4], den, pr[4], rec[3];
      tetra_forward<KC>(T, Pi, Pj, C, xr, sp, den, pr, rec);
      float grec[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) grec[c] = 2.f * (rec[c] - C[c]) * gerr;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        dP[ti][c] += grec[c] * pr[2];
        dP[tj][c] += grec[c] * pr[3];
      }
      const float gpr[4] = {0.f, grec[0] + grec[1] + grec[2],
                            grec[0] * Pi[0] + grec[1] * Pi[1] + grec[2] * Pi[2],
                            grec[0] * Pj[0] + grec[1] * Pj[1] + grec[2] * Pj[2]};
      const float gps = (gpr[0] * sp[0] + gpr[1] * sp[1] + gpr[2] * sp[2] + gpr[3] * sp[3]) /
                        (den * den);
#pragma unroll
      for (int k = 0; k < 4; ++k) gx[k] += (gpr[k] / den - gps) * softplus_grad(xr[k]);
    }
    // coords (beta, gamma, delta) = A^-1 C; alpha = 1 - sum
    const float gco[3] = {gx[1] - gx[0], gx[2] - gx[0], gx[3] - gx[0]};
    float v[3];  // A^-T gco
#pragma unroll
    for (int c = 0; c < 3; ++c)
      v[c] = T.ainv[c] * gco[0] + T.ainv[3 + c] * gco[1] + T.ainv[6 + c] * gco[2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      dP[ti][c] -= v[c] * x[2];
      dP[tj][c] -= v[c] * x[3];
    }
  }
#pragma unroll
  for (int i = 0; i < KC; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) scr[(3 * i + c) * kGeoThreads] = dP[i][c];
}

template <int KC>
__global__ void __launch_bounds__(kGeoThreads)
    k_palette_geo_loss(int64_t hw, const float* __restrict__ layer,
                       const float* __restrict__ target, const float* __restrict__ chroma,
                       int clamp, int kind, float lambda_pos, float inv_n,
                       float* __restrict__ wbary, float* __restrict__ loss,
                       float* __restrict__ dlayer, float* __restrict__ dchroma) {
  pdl_wait();
  constexpr int K = KC + 2;
  __shared__ TetraConst<KC> s_t[KC];
  __shared__ float s_p[KC][3];
  __shared__ float red[kGeoThreads / 32][3 * KC + 2];
  __shared__ float s_scr[3 * KC > KC + 2 ? 3 * KC : KC + 2][kGeoThreads];  // general-path data
  if (threadIdx.x < 3 * KC) s_p[threadIdx.x / 3][threadIdx.x % 3] = chroma[threadIdx.x];
  __syncthreads();
  if (threadIdx.x < KC) {
    const int i = threadIdx.x, j = (i + 1) % KC;
    TetraConst<KC> T;
    T.i = i;
    T.j = j;
    float a[9];  // A = [1 | c_i | c_j] by columns, row-major
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      a[3 * r] = 1.f;
      a[3 * r + 1] = s_p[i][r];
      a[3 * r + 2] = s_p[j][r];
    }
    const float det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                      a[2] * (a[3] * a[7] - a[4] * a[6]);
    T.adj[0] = a[4] * a[8] - a[5] * a[7];
    T.adj[1] = -(a[1] * a[8] - a[2] * a[7]);
    T.adj[2] = a[1] * a[5] - a[2] * a[4];
    T.adj[3] = -(a[3] * a[8] - a[5] * a[6]);
    T.adj[4] = a[0] * a[8] - a[2] * a[6];
    T.adj[5] = -(a[0] * a[5] - a[2] * a[3]);
    T.adj[6] = a[3] * a[7] - a[4] * a[6];
    T.adj[7] = -(a[0] * a[7] - a[1] * a[6]);
    T.adj[8] = a[0] * a[4] - a[1] * a[3];
    T.dinv = 1.f / (det + kBaryEps);
#pragma unroll
    for (int k = 0; k < 9; ++k) T.ainv[k] = T.adj[k] / det;
    s_t[i] = T;
  }
  __syncthreads();
  float dP[KC][3];
#pragma unroll
  for (int i = 0; i < KC; ++i) dP[i][0] = dP[i][1] = dP[i][2] = 0.f;
  float lgeo = 0.f, lpos = 0.f;
  // The next pixel's inputs are loaded while this one is computed (few warps
  // fit per SM at this register count, so the loads would stall otherwise).
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  float Cn[3], Ln[K];
  auto fetch = [&](int64_t q) {
    if (q < hw) {
#pragma unroll
      for (int c = 0; c < 3; ++c) Cn[c] = target[c * hw + q];
#pragma unroll
      for (int k = 0; k < K; ++k) Ln[k] = layer[k * hw + q];
    }
  };
  fetch((int64_t)blockIdx.x * blockDim.x + threadIdx.x);
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < hw; p += stride) {
    const float C[3] = {Cn[0], Cn[1], Cn[2]};
    float Lp[K];
#pragma unroll
    for (int k = 0; k < K; ++k) Lp[k] = Ln[k];
    fetch(p + stride);
    // Reconstruction errors; the softmax over -err / 1e-9 is one-hot unless
    // two errors agree to ~1e-7: then the winner's weight is exp(0) = 1, the
    // others underflow to 0, and the target and its palette gradient involve
    // the winner's coordinates alone (with exactly the values the general
    // expressions give).
    float* scr = &s_scr[0][threadIdx.x];
    float err[KC];
#pragma unroll 1
    for (int i = 0; i < KC; ++i) {  // one tetrahedron at a time (register pressure)
      float x[4], sp[4], den, pr[4], rec[3];
      scr[i * kGeoThreads] =
          tetra_forward<KC>(s_t[i], s_p[i], s_p[i + 1 == KC ? 0 : i + 1], C, x, sp, den, pr, rec);
    }
#pragma unroll
    for (int i = 0; i < KC; ++i) err[i] = scr[i * kGeoThreads];
    float emin = INFINITY;
#pragma unroll
    for (int i = 0; i < KC; ++i) emin = fminf(emin, err[i]);
    int nz = 0, win = 0;
#pragma unroll
    for (int i = 0; i < KC; ++i) {
      if (expf((emin - err[i]) * (1.f / kBaryTau)) != 0.f) {
        ++nz;
        win = i;
      }
    }
    const bool onehot = nz == 1;
    const int wj = win + 1 == KC ? 0 : win + 1;
    float Wb[K], xw[4];
    if (onehot) {
      tetra_coords<KC>(s_t[win], C, xw);
      Wb[0] = xw[0];
      Wb[1] = xw[1];
#pragma unroll
      for (int k = 2; k < K; ++k) Wb[k] = k - 2 == win ? xw[2] : k - 2 == wj ? xw[3] : 0.f;
    } else {
      bary_target_general<KC>(s_t, s_p, C[0], C[1], C[2], scr);
#pragma unroll
      for (int k = 0; k < K; ++k) Wb[k] = scr[k * kGeoThreads];
    }
    float Wc[K], m[K], s_raw = 0.f, s = 1.f;
    if (clamp) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        m[k] = fmaxf(Wb[k], 0.f);
        s_raw += m[k];
      }
      s = fmaxf(s_raw, 1e-8f);
      const float rs = 1.f / s;
#pragma unroll
      for (int k = 0; k < K; ++k) Wc[k] = m[k] * rs;
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) Wc[k] = Wb[k];
    }
    float gW[K];  // d loss / d target
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const float wt = Lp[k];
      const float d = wt - Wc[k];
      float g;
      if (kind == 0) {
        lgeo += d * d;
        g = 2.f * d * inv_n;
      } else {
        lgeo += fabsf(d);
        g = (d > 0.f ? 1.f : d < 0.f ? -1.f : 0.f) * inv_n;
      }
      lpos += fmaxf(-wt, 0.f);
      if (dlayer) dlayer[k * hw + p] = g + (wt < 0.f ? -lambda_pos * inv_n : 0.f);
      if (wbary) wbary[k * hw + p] = Wc[k];
      gW[k] = -g;
    }
    if (!dchroma) continue;
    // through the clamp and renormalisation
    float gWb[K];
    if (clamp) {
      float gm_dot = 0.f;
#pragma unroll
      for (int k = 0; k < K; ++k) gm_dot += gW[k] * m[k];
      const float rs = 1.f / s, corr = s_raw > 1e-8f ? gm_dot * rs * rs : 0.f;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const float gm = gW[k] * rs - corr;
        gWb[k] = Wb[k] > 0.f ? gm : 0.f;
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) gWb[k] = gW[k];
    }
    if (onehot) {
      // the winner's raw-coordinate path: coords (beta, gamma, delta) = A^-1 C,
      // alpha = 1 - sum; d/d c_i through A^-1 (the error path carries 0)
      float g2 = 0.f, g3 = 0.f;
#pragma unroll
      for (int k = 2; k < K; ++k) {
        if (k - 2 == win) g2 = gWb[k];
        if (k - 2 == wj) g3 = gWb[k];
      }
      const float gco[3] = {gWb[1] - gWb[0], g2 - gWb[0], g3 - gWb[0]};
      const TetraConst<KC>& T = s_t[win];
      float v[3];  // A^-T gco
#pragma unroll
      for (int c = 0; c < 3; ++c)
        v[c] = T.ainv[c] * gco[0] + T.ainv[3 + c] * gco[1] + T.ainv[6 + c] * gco[2];
#pragma unroll
      for (int i = 0; i < KC; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (i == win) dP[i][c] -= v[c] * xw[2];
          if (i == wj) dP[i][c] -= v[c] * xw[3];
        }
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) scr[k * kGeoThreads] = gWb[k];
      bary_adjoint_general<KC>(s_t, s_p, C[0], C[1], C[2], scr);
#pragma unroll
      for (int i = 0; i < KC; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) dP[i][c] += scr[(3 * i + c) * kGeoThreads];
    }
  }
  // block reduction: dchroma (3 KC values), geo and pos loss sums
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float vals[3 * KC + 2];
#pragma unroll
  for (int i = 0; i < KC; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) vals[3 * i + c] = dP[i][c];
  vals[3 * KC] = lgeo;
  vals[3 * KC + 1] = lpos;
#pragma unroll
  for (int k = 0; k < 3 * KC + 2; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vals[k] += __shfl_xor_sync(0xffffffffu, vals[k], o);
    if (lane == 0) red[w][k] = vals[k];
  }
  __syncthreads();
  if (threadIdx.x < 3 * KC + 2) {
    float t = 0.f;
#pragma unroll
    for (int k = 0; k < kGeoThreads / 32; ++k) t += red[k][threadIdx.x];
    if (threadIdx.x < 3 * KC) {
      if (dchroma) atomicAdd(dchroma + threadIdx.x, t);
    } else if (threadIdx.x == 3 * KC) {
      atomicAdd(loss + 1, t * inv_n);
      atomicAdd(loss, t * inv_n);
    } else {
      atomicAdd(loss + 2, t * lambda_pos * inv_n);
      atomicAdd(loss, t * lambda_pos * inv_n);
    }
  }
}

int launch_palette_geo_loss(int KC, int H, int W, const float* layer, const float* target,
                            const float* chroma, int clamp, int kind, float lambda_pos,
                            float* wbary, float* loss, float* dlayer, float* dchroma,
                            cudaStream_t st) {
  const int64_t hw = (int64_t)H * W;
  {
    const int rc = launch_zero2(loss, 3, dchroma, 3 * KC, st);
    if (rc) return rc;
  }
  if (hw == 0) return GSB_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t need = (hw + kGeoThreads - 1) / kGeoThreads;
  const float inv_n = 1.f / (float)((int64_t)(KC + 2) * hw);
  // one wave of resident blocks, each striding over the pixels (3 waves of
  // 12 blocks per SM measured 0.084 ms at 1920x1080, K = 5; one wave 0.080)
  switch (KC) {
#define GSB_KC(KK)                                                                                \
  case KK: {                                                                                      \
    static int per_sm = 0;                                                                        \
    if (per_sm == 0 && cudaOccupancyMaxActiveBlocksPerMultiprocessor(                            \
                           &per_sm, k_palette_geo_loss<KK>, kGeoThreads, 0) != cudaSuccess) {   \
      (void)cudaGetLastError();                                                                   \
      per_sm = 4;                                                                                 \
    }                                                                                             \
    const int grid = (int)std::min<int64_t>(need, (int64_t)sms * std::max(per_sm, 1));          \
    launch_pdl(k_palette_geo_loss<KK>, dim3(grid), dim3(kGeoThreads), 0, st, hw, layer, target, \
               chroma, clamp, kind, lambda_pos, inv_n, wbary, loss, dlayer, dchroma);           \
    break;                                                                                        \
  }
    GSB_KC(2) GSB_KC(3) GSB_KC(4) GSB_KC(5) GSB_KC(6)
#undef GSB_KC
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
  return check_launch("palette_geo_loss");
}

}  // namespace gsb
