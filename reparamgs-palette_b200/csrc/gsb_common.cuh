// Shared definitions of the B200 palette-weight rasterizer (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "gsplat_b200.h"

namespace gsb {

// ---------------------------------------------------------------- constants
// Tile edge and thresholds of the reference rasterizer
// (gsplatcu/common.cuh:13-14, gsplatcu/kernel.cu:10-12, 258-265).
constexpr int kTile = 16;
constexpr int kTilePixels = kTile * kTile;
constexpr float kMinDepth = 0.2f;
constexpr float kBadDepth = -1.f;
constexpr float kAlphaMax = 0.99f;
constexpr float kAlphaMin = 0.002f;
constexpr float kTransMin = 0.0001f;
constexpr int kMaxChannels = 8;  // MAX_SPLAT_DIM of the reference

// Real spherical-harmonic basis constants for l <= 3, stored in FP32: the
// B200 path evaluates the basis in FP32 only (gsplatcu/common.cuh:29-44 holds
// the same values as double literals).
constexpr float SH_C0 = 0.28209479177387814f;
constexpr float SH_C1 = 0.4886025119029199f;
constexpr float SH_C2_0 = 1.0925484305920792f;
constexpr float SH_C2_2 = 0.31539156525252005f;
constexpr float SH_C2_4 = 0.5462742152960396f;
constexpr float SH_C3_0 = 0.5900435899266435f;
constexpr float SH_C3_1 = 2.890611442640554f;
constexpr float SH_C3_2 = 0.4570457994644658f;
constexpr float SH_C3_3 = 0.3731763325901154f;
constexpr float SH_C3_5 = 1.445305721320277f;

// Margin (in Mahalanobis units) added to the exact skip threshold
// 2 ln(alpha / 0.002): a pixel farther than the cut is guaranteed to give
// alpha' < 0.002 in the reference's own FP32 evaluation, so skipping it never
// changes a result; pixels inside it are evaluated exactly as the reference.
constexpr float kCutMargin = 1e-3f;

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// ------------------------------------------------------------ element loads
// Per-Gaussian colour parameters may be stored in FP32 or BF16 (selected at
// run time by GSB_DTYPE_*); all arithmetic is FP32.
__device__ __forceinline__ float ld(const float* p, int64_t i) { return __ldg(p + i); }
__device__ __forceinline__ float ld(const __nv_bfloat16* p, int64_t i) {
  return __bfloat162float(p[i]);
}

// Reference Mahalanobis form qa dx^2 + qc dy^2 + 2 qb dx dy
// (gsplatcu/common.cuh:89-92), written with explicit round-to-nearest
// intrinsics in the order the reference build's FP32 results follow: the
// qc term rounded on its own, the qa term fused onto it, the cross term
// fused last (pinned by reproducing the reference build's contributor
// indices and final transmittance bit for bit at 1M Gaussians / 1080p).
// The intrinsics are never re-contracted, so the forward and the adjoint
// (separate kernels) take the same skip (alpha' < 0.002) and stop
// (T < 1e-4) decisions as the reference and as each other.
__device__ __forceinline__ float maha_sq(float qa, float qb, float qc, float dx, float dy) {
  const float cross = __fmul_rn(__fmul_rn(2.f, qb), dx);
  return __fmaf_rn(cross, dy, __fmaf_rn(__fmul_rn(qa, dx), dx, __fmul_rn(__fmul_rn(qc, dy), dy)));
}

// Packed per-Gaussian record read by the compositing kernels (layout in
// gsb_record.cuh): float4 v0 = centre and conic a, b; v1 = conic c, skip
// cut, opacity, channel 0; v2 = support half-extents and the conic
// diagonal's reciprocals; v3.. = channels 1..K-1, zero padded.
template <int K>
struct RecordLayout {
  static constexpr int kFloats = ((11 + K) + 3) / 4 * 4;
  static constexpr int kVec4 = kFloats / 4;
};
// Float index of channel k inside a record (gsb_record.cuh).
__host__ __device__ constexpr int record_channel(int k) { return k == 0 ? 7 : 11 + k; }

// ----------------------------------------------------------- error plumbing
void set_error(const char* fmt, ...);
// Records `launches` kernel launches (when the last launch succeeded) and
// converts a launch error into GSB_ERR_CUDA with a message.
int check_launch(const char* what, int launches = 1);

// Programmatic dependent launch: a kernel launched with launch_pdl may be
// scheduled while the previous kernel on its stream is still finishing, which
// hides the launch gap between the short kernels of one render.  Every kernel
// that can be launched this way calls pdl_wait() before it touches global
// memory; the wait returns once the previous kernel has completed and its
// writes are visible (without the launch attribute it returns at once).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

}  // namespace gsb

#define GSB_CHECK_ARG(cond, ...)        \
  do {                                  \
    if (!(cond)) {                      \
      gsb::set_error(__VA_ARGS__);      \
      return GSB_ERR_INVALID_ARGUMENT;  \
    }                                   \
  } while (0)
