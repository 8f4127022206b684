// The differentiation workload's loss in one kernel: the palette colour image
// img_c = sum_k palette[k][c] layer_k, the L1 + SSIM loss of gau_loss
// (vanilla_3dgs/gsplat/pytorch_ssim.py:26-67) against a target, the
// negative-weight penalty of finetune.py:375,381, and the gradient of all of
// it w.r.t. the layer stack and the palette.
//
// SSIM's gradient at a pixel q needs the SSIM partials at every pixel within
// the window radius R = 5 of q, and each partial needs the window statistics
// (mean, second moments) of the pixels within R of it.  A block therefore
// owns a 32x32 output tile and stages the image (all three channels, from one
// read of the layer stack) and the target over the tile plus 2R on every side; the statistics and partials are computed on the tile
// plus R, and the partials are filtered back onto the tile.  The halo work is
// recomputed by the neighbouring blocks instead of exchanged, so the loss and
// its full gradient come out of one launch (the gradient of a mean does not
// depend on the loss value).  The 11x11 Gaussian window is applied as two
// 11-tap passes (the window is the outer product of the 1-D Gaussian),
// register-blocked so each shared-memory read feeds several outputs.
#include <algorithm>
#include <cmath>

#include "gsb_common.cuh"
#include "gsb_internal.h"

namespace gsb {

constexpr int kSsimTile = 32;                      // output tile edge
constexpr int kSsimR = 5;                          // window radius (11 taps)
constexpr int kSsimTaps = 2 * kSsimR + 1;
constexpr int kSsimXR = kSsimTile + 4 * kSsimR;    // 52: staged image / target edge
constexpr int kSsimMR = kSsimTile + 2 * kSsimR;    // 42: statistics / partials edge
constexpr int kSsimThreads = 256;
constexpr int kSsimPix = kSsimTile * kSsimTile / kSsimThreads;  // output rows per thread
// register blocking of the four filter passes (outputs per work item)
constexpr int kRunH1 = 3, kRunV1 = 3, kRunH2 = 4;
static_assert(kSsimMR % kRunH1 == 0 && kSsimMR % kRunV1 == 0 && kSsimTile % kRunH2 == 0, "runs");
static_assert(kSsimThreads == 8 * kSsimTile && kSsimPix == 4, "thread layout");

constexpr size_t kSsimSmemFloats = 3 * kSsimXR * kSsimXR   // image, 3 channels
                                   + kSsimXR * kSsimXR      // target, one channel
                                   + 5 * kSsimXR * kSsimMR  // horizontal pass of 5 statistics
                                   + 3 * kSsimMR * kSsimMR  // SSIM partials
                                   + 3 * 8;                 // palette
constexpr size_t kSsimSmemBytes = kSsimSmemFloats * sizeof(float);  // 108.3 KB: 2 blocks/SM

struct SsimWindow {
  float g[kSsimTaps];
};

struct SsimScales {
  float c1, c2;    // (0.01 range)^2, (0.03 range)^2
  float inv_n;     // 1 / (3 H W)
  float w_l1;      // (1 - lambda_ssim) / (3 H W)
  float w_ssim;    // lambda_ssim / (3 H W)
  float w_pos;     // lambda_pos / (K H W)
};

__global__ void k_l1_ssim_init(float* __restrict__ loss, float* __restrict__ dpal, int n_pal,
                               float lambda_ssim) {
  pdl_wait();
  // total = lambda_ssim * (1 - mean SSIM) + ...: the blocks add -w_ssim * sum S
  if (threadIdx.x < 4) loss[threadIdx.x] = threadIdx.x == 0 ? lambda_ssim : 0.f;
  if (dpal && threadIdx.x < n_pal) dpal[threadIdx.x] = 0.f;
}

template <int K, bool PAL>
__global__ void __launch_bounds__(kSsimThreads, 2)
    k_palette_l1_ssim(int H, int W, const float* __restrict__ layer,
                      const float* __restrict__ palette, const float* __restrict__ target,
                      SsimWindow win, SsimScales sc, float* __restrict__ image,
                      float* __restrict__ loss, float* __restrict__ dlayer,
                      float* __restrict__ dpal) {
  pdl_wait();
  constexpr int XR2 = kSsimXR * kSsimXR;
  extern __shared__ float smem[];
  float* sX3 = smem;                            // [3][52][52] image
  float* sY = sX3 + 3 * XR2;                    // [52][52] target channel c
  float* sH = sY + XR2;                         // [5][52][42], later [3][42][32]
  float* sM = sH + 5 * kSsimXR * kSsimMR;       // [3][42][42]
  float* sP = sM + 3 * kSsimMR * kSsimMR;       // [K][3]
  __shared__ float red[kSsimThreads / 32][3 + 3 * K];

  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * kSsimTile, y0 = blockIdx.y * kSsimTile;
  const int64_t hw = (int64_t)H * W;
  if (tid < 3 * K) sP[tid] = PAL ? palette[tid] : (tid / 3 == tid % 3 ? 1.f : 0.f);
  __syncthreads();

  // 0. the image over the tile + 2R, all three channels (zero outside), from
  //    one read of the layer stack; positions four at a time so each thread
  //    has 4K loads in flight
  constexpr int kStage = (XR2 + kSsimThreads - 1) / kSsimThreads;  // 11 positions per thread
#pragma unroll 1
  for (int e0 = 0; e0 < kStage; e0 += 4) {
    float l[4][K];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + (e0 + u) * kSsimThreads;
      const int r = e / kSsimXR, q = e - r * kSsimXR;
      const int iy = y0 - 2 * kSsimR + r, ix = x0 - 2 * kSsimR + q;
      const bool in = e0 + u < kStage && e < XR2 && iy >= 0 && iy < H && ix >= 0 && ix < W;
      const int64_t p = in ? (int64_t)iy * W + ix : 0;
#pragma unroll
      for (int k = 0; k < K; ++k) l[u][k] = in ? layer[k * hw + p] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + (e0 + u) * kSsimThreads;
      if (e0 + u < kStage && e < XR2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float xv = 0.f;
#pragma unroll
          for (int k = 0; k < K; ++k) xv = fmaf(sP[3 * k + c], l[u][k], xv);
          sX3[c * XR2 + e] = xv;
        }
      }
    }
  }

  // this thread's output pixels: column tx, rows ty0 .. ty0 + 3 of the tile;
  // dxs = d loss / d image there, per channel
  const int tx = tid & 31, ty0 = (tid >> 5) * kSsimPix;
  const int gx = x0 + tx;
  float dxs[3][kSsimPix];
  float l1 = 0.f, ssum = 0.f;

#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    const float* sX = sX3 + c * XR2;
    // 1. the target channel over the tile + 2R (zero outside), loads first
    {
      float yv[kStage];
#pragma unroll
      for (int u = 0; u < kStage; ++u) {
        const int e = tid + u * kSsimThreads;
        const int r = e / kSsimXR, q = e - r * kSsimXR;
        const int iy = y0 - 2 * kSsimR + r, ix = x0 - 2 * kSsimR + q;
        const bool in = e < XR2 && iy >= 0 && iy < H && ix >= 0 && ix < W;
        yv[u] = in ? target[c * hw + (int64_t)iy * W + ix] : 0.f;
      }
#pragma unroll
      for (int u = 0; u < kStage; ++u) {
        const int e = tid + u * kSsimThreads;
        if (e < XR2) sY[e] = yv[u];
      }
    }
    __syncthreads();

    // 2. horizontal pass of x, y, x^2, y^2, xy: 52 rows x 42 columns
    constexpr int kRunsH1 = kSsimMR / kRunH1;
    for (int e = tid; e < kSsimXR * kRunsH1; e += kSsimThreads) {
      const int r = e / kRunsH1, j0 = (e - r * kRunsH1) * kRunH1;
      const float* px = sX + r * kSsimXR + j0;
      const float* py = sY + r * kSsimXR + j0;
      float a[5][kRunH1];
#pragma unroll
      for (int q = 0; q < 5; ++q)
#pragma unroll
        for (int o = 0; o < kRunH1; ++o) a[q][o] = 0.f;
#pragma unroll
      for (int t = 0; t < kRunH1 + 2 * kSsimR; ++t) {
        const float xv = px[t], yv = py[t];
        const float v[5] = {xv, yv, xv * xv, yv * yv, xv * yv};
#pragma unroll
        for (int o = 0; o < kRunH1; ++o) {
          const int i = t - o;
          if (i >= 0 && i < kSsimTaps)
#pragma unroll
            for (int q = 0; q < 5; ++q) a[q][o] = fmaf(win.g[i], v[q], a[q][o]);
        }
      }
#pragma unroll
      for (int q = 0; q < 5; ++q)
#pragma unroll
        for (int o = 0; o < kRunH1; ++o) sH[(q * kSsimXR + r) * kSsimMR + j0 + o] = a[q][o];
    }
    __syncthreads();

    // 3. vertical pass -> window statistics on the tile + R, then the SSIM map
    //    and its partials w.r.t. mu_x, s_xx and s_xy (zero outside the image)
    constexpr int kRunsV1 = kSsimMR / kRunV1;
    for (int e = tid; e < kSsimMR * kRunsV1; e += kSsimThreads) {
      const int j = e % kSsimMR, r0 = (e / kSsimMR) * kRunV1;
      float a[5][kRunV1];
#pragma unroll
      for (int q = 0; q < 5; ++q)
#pragma unroll
        for (int o = 0; o < kRunV1; ++o) a[q][o] = 0.f;
#pragma unroll
      for (int t = 0; t < kRunV1 + 2 * kSsimR; ++t) {
        float v[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) v[q] = sH[(q * kSsimXR + r0 + t) * kSsimMR + j];
#pragma unroll
        for (int o = 0; o < kRunV1; ++o) {
          const int i = t - o;
          if (i >= 0 && i < kSsimTaps)
#pragma unroll
            for (int q = 0; q < 5; ++q) a[q][o] = fmaf(win.g[i], v[q], a[q][o]);
        }
      }
      const int ix = x0 - kSsimR + j;
      const bool col_in = ix >= 0 && ix < W;
      const bool col_tile = j >= kSsimR && j < kSsimR + kSsimTile;
#pragma unroll
      for (int o = 0; o < kRunV1; ++o) {
        const int r = r0 + o, iy = y0 - kSsimR + r;
        float dm = 0.f, dxx = 0.f, dxy = 0.f;
        if (col_in && iy >= 0 && iy < H) {
          const float mx = a[0][o], my = a[1][o];
          const float mxy = mx * my, mxx = mx * mx, myy = my * my;
          const float A1 = 2.f * mxy + sc.c1;
          const float A2 = 2.f * (a[4][o] - mxy) + sc.c2;
          const float B1 = mxx + myy + sc.c1;
          const float B2 = (a[2][o] - mxx) + (a[3][o] - myy) + sc.c2;
          // B1 >= C1 > 0 and B2 > 0 up to rounding: the fast reciprocal's
          // relative error (2 ulp) is far below the gradient tolerance
          const float rB1 = __fdividef(1.f, B1), rB2 = __fdividef(1.f, B2);
          const float inv = rB1 * rB2;
          const float S = A1 * A2 * inv;
          dm = 2.f * my * (A2 - A1) * inv - 2.f * mx * S * (rB1 - rB2);
          dxx = -S * rB2;
          dxy = 2.f * A1 * inv;
          if (col_tile && r >= kSsimR && r < kSsimR + kSsimTile) ssum += S;
        }
        sM[(0 * kSsimMR + r) * kSsimMR + j] = dm;
        sM[(1 * kSsimMR + r) * kSsimMR + j] = dxx;
        sM[(2 * kSsimMR + r) * kSsimMR + j] = dxy;
      }
    }
    __syncthreads();

    // 4. horizontal pass of the partials: 42 rows x 32 columns (into sH)
    constexpr int kRunsH2 = kSsimTile / kRunH2;
    for (int e = tid; e < kSsimMR * kRunsH2; e += kSsimThreads) {
      const int r = e / kRunsH2, j0 = (e - r * kRunsH2) * kRunH2;
      float b[3][kRunH2];
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int o = 0; o < kRunH2; ++o) b[m][o] = 0.f;
#pragma unroll
      for (int t = 0; t < kRunH2 + 2 * kSsimR; ++t) {
        float v[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) v[m] = sM[(m * kSsimMR + r) * kSsimMR + j0 + t];
#pragma unroll
        for (int o = 0; o < kRunH2; ++o) {
          const int i = t - o;
          if (i >= 0 && i < kSsimTaps)
#pragma unroll
            for (int m = 0; m < 3; ++m) b[m][o] = fmaf(win.g[i], v[m], b[m][o]);
        }
      }
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int o = 0; o < kRunH2; ++o) sH[(m * kSsimMR + r) * kSsimTile + j0 + o] = b[m][o];
    }
    __syncthreads();

    // 5. vertical pass onto this thread's pixels, and d loss / d image there
    float gs[3][kSsimPix];
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int o = 0; o < kSsimPix; ++o) gs[m][o] = 0.f;
#pragma unroll
    for (int t = 0; t < kSsimPix + 2 * kSsimR; ++t) {
      float v[3];
#pragma unroll
      for (int m = 0; m < 3; ++m) v[m] = sH[(m * kSsimMR + ty0 + t) * kSsimTile + tx];
#pragma unroll
      for (int o = 0; o < kSsimPix; ++o) {
        const int i = t - o;
        if (i >= 0 && i < kSsimTaps)
#pragma unroll
          for (int m = 0; m < 3; ++m) gs[m][o] = fmaf(win.g[i], v[m], gs[m][o]);
      }
    }
#pragma unroll
    for (int o = 0; o < kSsimPix; ++o) {
      const int ty = ty0 + o, gy = y0 + ty;
      float dx = 0.f;
      if (gx < W && gy < H) {
        const int s = (ty + 2 * kSsimR) * kSsimXR + tx + 2 * kSsimR;
        const float xv = sX[s], yv = sY[s];
        const float dS = gs[0][o] + 2.f * xv * gs[1][o] + yv * gs[2][o];
        const float d = xv - yv;
        l1 += fabsf(d);
        const float sg = d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f);
        dx = sc.w_l1 * sg - sc.w_ssim * dS;
        if (image) image[c * hw + (int64_t)gy * W + gx] = xv;
      }
      // c is not a compile-time index: select, so dxs stays in registers
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
        if (cc == c) dxs[cc][o] = dx;
    }
    __syncthreads();  // the next channel overwrites the staged target and passes
  }

  // layer and palette gradients, negative-weight penalty
  float pen = 0.f, dp[K][3];
#pragma unroll
  for (int k = 0; k < K; ++k) dp[k][0] = dp[k][1] = dp[k][2] = 0.f;
#pragma unroll
  for (int o = 0; o < kSsimPix; ++o) {
    const int gy = y0 + ty0 + o;
    if (gx < W && gy < H) {
      const int64_t p = (int64_t)gy * W + gx;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const float l = layer[k * hw + p];
        pen += fmaxf(-l, 0.f);
        float g = l < 0.f ? -sc.w_pos : 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          g = fmaf(sP[3 * k + c], dxs[c][o], g);
          dp[k][c] = fmaf(l, dxs[c][o], dp[k][c]);
        }
        if (dlayer) dlayer[k * hw + p] = g;
      }
    }
  }

  // block reduction of the loss sums and the palette gradient
  const int lane = tid & 31, w = tid >> 5;
  float v[3 + 3 * K];
  v[0] = l1;
  v[1] = ssum;
  v[2] = pen;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    v[3 + 3 * k] = dp[k][0];
    v[4 + 3 * k] = dp[k][1];
    v[5 + 3 * k] = dp[k][2];
  }
#pragma unroll
  for (int j = 0; j < 3 + 3 * K; ++j) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
    if (lane == 0) red[w][j] = v[j];
  }
  __syncthreads();
  if (tid < 3 + 3 * K) {
    float t = 0.f;
#pragma unroll
    for (int q = 0; q < kSsimThreads / 32; ++q) t += red[q][tid];
    if (tid == 0) {
      atomicAdd(loss + 1, t * sc.inv_n);
      atomicAdd(loss, t * sc.w_l1);
    } else if (tid == 1) {
      atomicAdd(loss + 2, t * sc.inv_n);
      atomicAdd(loss, -t * sc.w_ssim);
    } else if (tid == 2) {
      atomicAdd(loss + 3, t * sc.w_pos);
      atomicAdd(loss, t * sc.w_pos);
    } else if (dpal) {
      atomicAdd(dpal + (tid - 3), t);
    }
  }
}

template <int K, bool PAL>
static int launch_l1_ssim_k(dim3 grid, const float* layer, const float* palette,
                            const float* target, int H, int W, const SsimWindow& win,
                            const SsimScales& sc, float* image, float* loss, float* dlayer,
                            float* dpal, cudaStream_t st) {
  // opt in to > 48 KB of dynamic shared memory, once per device
  static bool attr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !attr[dev]) {
    if (cudaFuncSetAttribute(k_palette_l1_ssim<K, PAL>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSsimSmemBytes) != cudaSuccess)
      return check_launch("palette_l1_ssim (shared memory attribute)", 0);
    if (dev >= 0 && dev < 64) attr[dev] = true;
  }
  launch_pdl(k_palette_l1_ssim<K, PAL>, grid, dim3(kSsimThreads), kSsimSmemBytes, st, H, W,
             layer, palette, target, win, sc, image, loss, dlayer, dpal);
  return check_launch("palette_l1_ssim");
}

int launch_palette_l1_ssim(int K, int H, int W, const float* layer, const float* palette,
                           const float* target, float lambda_ssim, float lambda_pos,
                           float data_range, float* image, float* loss, float* dlayer,
                           float* dpal, cudaStream_t st) {
  // the reference's window: the 1-D Gaussian rounded to FP32, divided by its
  // FP32 sum (pytorch_ssim.py:12-14)
  SsimWindow win;
  double e[kSsimTaps], sum = 0.0;
  for (int i = 0; i < kSsimTaps; ++i) {
    const double x = i - kSsimR;
    e[i] = (double)(float)std::exp(-x * x / (2.0 * 1.5 * 1.5));
    sum += e[i];
  }
  const float fsum = (float)sum;
  for (int i = 0; i < kSsimTaps; ++i) win.g[i] = (float)e[i] / fsum;
  const int64_t hw = (int64_t)H * W;
  SsimScales sc;
  sc.c1 = (0.01f * data_range) * (0.01f * data_range);
  sc.c2 = (0.03f * data_range) * (0.03f * data_range);
  sc.inv_n = hw ? (float)(1.0 / (3.0 * (double)hw)) : 0.f;
  sc.w_l1 = (1.f - lambda_ssim) * sc.inv_n;
  sc.w_ssim = lambda_ssim * sc.inv_n;
  sc.w_pos = hw ? (float)((double)lambda_pos / ((double)K * (double)hw)) : 0.f;
  // an empty image has no pixels to average: its loss and gradients are 0
  launch_pdl(k_l1_ssim_init, dim3(1), dim3(32), 0, st, loss, dpal, 3 * K,
             hw ? lambda_ssim : 0.f);
  int rc = check_launch("palette_l1_ssim (init)");
  if (rc || hw == 0) return rc;
  const dim3 grid((W + kSsimTile - 1) / kSsimTile, (H + kSsimTile - 1) / kSsimTile);
  if (!palette) return launch_l1_ssim_k<3, false>(grid, layer, nullptr, target, H, W, win, sc,
                                                  image, loss, dlayer, nullptr, st);
  switch (K) {
#define GSB_K(KK)                                                                          \
  case KK:                                                                                 \
    return launch_l1_ssim_k<KK, true>(grid, layer, palette, target, H, W, win, sc, image, \
                                      loss, dlayer, dpal, st);
    GSB_K(1) GSB_K(2) GSB_K(3) GSB_K(4) GSB_K(5) GSB_K(6) GSB_K(7) GSB_K(8)
#undef GSB_K
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
}

}  // namespace gsb
