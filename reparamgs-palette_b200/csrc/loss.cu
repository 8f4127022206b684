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
  if (cudaMemsetAsync(loss, 0, sizeof(float), st) != cudaSuccess ||
      (dpal && cudaMemsetAsync(dpal, 0, sizeof(float) * 3 * K, st) != cudaSuccess))
    return check_launch("palette_l1 (memset)", 0);
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

}  // namespace gsb
