// The packed compositing record of one Gaussian (one per Gaussian, gathered
// per patch by the compositing kernels): floats
//   0-3  support box xmin xmax ymin ymax      4-5  centre ux uy
//   6-8  conic qa qb qc                       9    cut
//   10   opacity                              11.. channel values (weights / colours)
// padded with zeros to whole float4s (RecordLayout<K>).
//
// The box is conservative: pixels outside it satisfy d^T Q d > cut, where
// cut = 2 ln(alpha/0.002) + margin guarantees alpha' < 0.002 in the
// reference's evaluation (gsplatcu/kernel.cu:343-353).  It is widened for the
// rounding error of the FP32 quadratic form (proportional to the conic's
// condition number) and disabled for degenerate or non-finite conics.
#pragma once

#include "gsb_common.cuh"

namespace gsb {

// Fills f[0..10] and zeroes f[11..19] (the caller writes the channels).
__device__ __forceinline__ void record_head(float ux, float uy, float qa, float qb, float qc,
                                            float a, float* f) {
  const float cut = 2.f * logf(a / kAlphaMin) + kCutMargin;
  float xmin = -INFINITY, xmax = INFINITY, ymin = -INFINITY, ymax = INFINITY;
  if (cut < 0.f) {  // alpha < 0.002: never blends, empty box
    xmin = ymin = INFINITY;
    xmax = ymax = -INFINITY;
  } else if (isfinite(cut) && isfinite(ux) && isfinite(uy)) {
    const float det = qa * qc - qb * qb;
    const float kappa = (qa + qc) * (qa + qc) / det;
    if (det > 0.f && qa > 0.f && qc > 0.f && kappa < 1e5f) {
      const float c2 = cut * (1.f + 4e-6f * kappa) + 1e-3f;
      const float hx = sqrtf(c2 * qc / det) * 1.0001f + 0.02f;
      const float hy = sqrtf(c2 * qa / det) * 1.0001f + 0.02f;
      if (isfinite(hx) && isfinite(hy)) {
        xmin = ux - hx;
        xmax = ux + hx;
        ymin = uy - hy;
        ymax = uy + hy;
      }
    }
  }
#pragma unroll
  for (int k = 11; k < 20; ++k) f[k] = 0.f;
  f[0] = xmin;
  f[1] = xmax;
  f[2] = ymin;
  f[3] = ymax;
  f[4] = ux;
  f[5] = uy;
  f[6] = qa;
  f[7] = qb;
  f[8] = qc;
  f[9] = cut;
  f[10] = a;
}

}  // namespace gsb
