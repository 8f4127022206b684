// The packed compositing record of one Gaussian (one per Gaussian, gathered
// per patch by the compositing kernels), as float4s:
//   v0  ux uy qa qb          centre, conic a b
//   v1  qc c2 alpha ch0      conic c, cut, opacity, channel 0
//   v2  hx hy 1/qa 1/qc      support half-extents, reciprocals for the culling
//   v3  ch1 ch2 ch3 ch4 ...  further channels (weights / colours), zero padded
// (record_channel(k) is the float index of channel k; RecordLayout<K>).
//
// Pixels outside the support box u +- (hx, hy) satisfy d^T Q d > c2, and any
// pixel with d^T Q d > c2 has alpha' < 0.002 in the reference's evaluation
// (gsplatcu/kernel.cu:343-353): c2 = 2 ln(alpha/0.002) + margin, widened for
// the rounding error of the FP32 quadratic form (proportional to the conic's
// condition number).  Degenerate or non-finite conics get an unbounded box
// and c2 = +inf (never culled); alpha < 0.002 an empty box (never blends).
#pragma once

#include "gsb_common.cuh"

namespace gsb {

// Fills the record's geometry floats and zeroes the channel slots (the
// caller writes the channels at record_channel(k)).
__device__ __forceinline__ void record_head(float ux, float uy, float qa, float qb, float qc,
                                            float a, float* f) {
  const float cut = 2.f * logf(a / kAlphaMin) + kCutMargin;
  float hx = INFINITY, hy = INFINITY, c2 = INFINITY, ia = 0.f, ic = 0.f;
  if (cut < 0.f) {  // alpha < 0.002: never blends, empty box
    hx = hy = -INFINITY;
    c2 = cut;
  } else if (isfinite(cut) && isfinite(ux) && isfinite(uy)) {
    const float det = qa * qc - qb * qb;
    const float kappa = (qa + qc) * (qa + qc) / det;
    if (det > 0.f && qa > 0.f && qc > 0.f && kappa < 1e5f) {
      const float cw = cut * (1.f + 4e-6f * kappa) + 1e-3f;
      const float ex = sqrtf(cw * qc / det) * 1.0001f + 0.02f;
      const float ey = sqrtf(cw * qa / det) * 1.0001f + 0.02f;
      if (isfinite(ex) && isfinite(ey)) {
        hx = ex;
        hy = ey;
        c2 = cw;
        ia = 1.f / qa;
        ic = 1.f / qc;
      }
    }
  }
#pragma unroll
  for (int k = 12; k < 20; ++k) f[k] = 0.f;
  f[0] = ux;
  f[1] = uy;
  f[2] = qa;
  f[3] = qb;
  f[4] = qc;
  f[5] = c2;
  f[6] = a;
  f[7] = 0.f;
  f[8] = hx;
  f[9] = hy;
  f[10] = ia;
  f[11] = ic;
}

}  // namespace gsb
