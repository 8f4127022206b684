// Fused render path.
//
// Forward: one kernel per view does, per Gaussian, everything the reference
// runs as five operators plus getRects (project, computeCov3D, computeCov2D,
// sh2Weight / sh2Weight_fast, inverseCov2D; gsplat/gsmodel.py:107-118 and
// 155-170): projection, 3D and 2D covariance, conic and extents, view-
// dependent palette weights (full SH order 3 or rank-r low-rank factors,
// FP32 or BF16 storage, FP32 arithmetic), the tile rectangle and the packed
// compositing record, with the same device functions as the separate
// operators.  Sorting and compositing are shared with splat_weight.
//
// Backward: the compositing adjoint (opacity / centre / conic / weight terms,
// raster.cu) followed by a per-Gaussian chain-rule kernel that recomputes the
// forward quantities from the parameters and maps the screen-space gradients
// to the parameters: conic -> 2D covariance -> 3D covariance -> (rotation,
// scale); centre and 2D covariance -> camera-space centre -> world centre;
// weights -> SH coefficients or low-rank factors, and the view direction ->
// world centre.  The frustum clamp and the 0.99 opacity clamp are not
// differentiated, as in the reference's own chain
// (vanilla_3dgs/gsplat/gsmodel.py:65-75).
#include "gsb_geometry.cuh"
#include "gsb_internal.h"
#include "gsb_record.cuh"
#include "gsb_stage.cuh"
#include "gsb_tma.cuh"

namespace gsb {

constexpr int kFuseThreads = 64;
static __device__ uint32_t g_fused_status;

// Row lengths of the colour-parameter arrays (floats per Gaussian).
template <int MODE, int K, int P, int Q, int R>
struct WRows {
  static constexpr int W0 = MODE == GSB_WEIGHTS_FULL ? 16 * K : K;  // shs or dc
  static constexpr int WA = MODE == GSB_WEIGHTS_FULL ? 0 : P * R;
  static constexpr int WB = MODE == GSB_WEIGHTS_FULL ? 0 : R * Q;
  static constexpr int L = MODE == GSB_WEIGHTS_FULL ? 15 : P * Q / K;
  static constexpr int IN = 3 + 4 + 3 + 1 + W0 + WA + WB;  // staged floats per Gaussian
  // The forward stages full-SH rows (16K floats, a multiple of 16) at a stride
  // of an odd number of float4s, so that one thread per row reading float4s
  // touches distinct shared-memory banks; other rows stay contiguous.
  static constexpr int W0S = MODE == GSB_WEIGHTS_FULL ? 4 * ((W0 / 4) | 1) : W0;
  static constexpr int INS = 3 + 4 + 3 + 1 + W0S + WA + WB;  // forward staged floats
};

// Camera: rotation, translation and centre stay in device memory (so a
// captured graph can be replayed for a new camera by rewriting them); the
// intrinsics are kernel arguments.
struct CamRegs {
  float R[9], t[3], c[3];
};

__device__ __forceinline__ CamRegs load_cam(const CamArgs& a) {
  CamRegs r;
#pragma unroll
  for (int k = 0; k < 9; ++k) r.R[k] = __ldg(a.R + k);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    r.t[k] = __ldg(a.t + k);
    r.c[k] = __ldg(a.c + k);
  }
  return r;
}

// Shared-memory regions of one block: the rows of its Gaussians, array by
// array, back to back.
template <int MODE, int K, int P, int Q, int R>
struct Staged {
  using WS = WRows<MODE, K, P, Q, R>;
  const float *p, *q, *s, *al, *w0, *wa, *wb;
  __device__ __forceinline__ explicit Staged(const float* sm) {
    const int nt = blockDim.x;
    p = sm;
    q = p + nt * 3;
    s = q + nt * 4;
    al = s + nt * 3;
    w0 = al + nt;
    wa = w0 + nt * WS::W0S;
    wb = wa + nt * WS::WA;
  }
};

// Extra shared memory of the forward, in floats per thread, past the staged
// rows: the raw bulk-copied BF16 colour rows, converted into the float rows.
template <int MODE, int K, int P, int Q, int R, typename T>
struct FwdExtra {
  using WS = WRows<MODE, K, P, Q, R>;
  static constexpr bool kRawLowrank = sizeof(T) == 2 && MODE != GSB_WEIGHTS_FULL;
  static constexpr int kRawFloats = sizeof(T) == 2 ? (WS::W0 + WS::WA + WS::WB + 1) / 2 : 0;
};

// How the block's colour-parameter rows ended up in shared memory.
enum StageResult { kStageFailed = 0, kStagedFloat = 1, kStagedRawBf16 = 2 };

// Stage one block's parameter rows (pws, rots, scales, alphas, colour
// parameters) into shared memory, by bulk copies when the block is full and
// every span is 16-byte aligned.  FP32 rows land in their float areas; BF16
// colour rows are bulk-copied raw (full SH: into the float area of the SH
// rows; low-rank: into `raw`) and converted by the caller (kStagedRawBf16).
// Without bulk copies every row is converted to float while staged.
// Returns kStageFailed if a bulk wait expired (the status word is set and the
// block must not use the staged rows).
template <int MODE, int K, int P, int Q, int R, typename T>
__device__ __forceinline__ int stage_params(int64_t n, int64_t row0, const float* pws,
                                            const float* rots, const float* scales,
                                            const float* alphas, const T* w0, const T* wa,
                                            const T* wb, float* sm, float* raw, uint64_t* bar) {
  using WS = WRows<MODE, K, P, Q, R>;
  const Staged<MODE, K, P, Q, R> S(sm);
  const int nt = blockDim.x;
  const bool full = row0 + nt <= n;
  bool bulk = full && aligned16(pws + row0 * 3) && aligned16(rots + row0 * 4) &&
              aligned16(scales + row0 * 3) && aligned16(alphas + row0) &&
              aligned16(w0 + row0 * WS::W0) && (nt * WS::W0 * sizeof(T)) % 16 == 0;
  if (MODE != GSB_WEIGHTS_FULL)
    bulk = bulk && aligned16(wa + row0 * WS::WA) && aligned16(wb + row0 * WS::WB) &&
           (nt * WS::WA * sizeof(T)) % 16 == 0 && (nt * WS::WB * sizeof(T)) % 16 == 0;
  const bool raw16 = bulk && sizeof(T) == 2;
  if (bulk && threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(
        bar, (uint32_t)(nt * 11 * 4 + nt * (WS::W0 + WS::WA + WS::WB) * sizeof(T)));
  }
  if constexpr (MODE == GSB_WEIGHTS_FULL && sizeof(T) == 4) {
    if (bulk) __syncthreads();  // the barrier is initialised before any thread's copy
  }
  stage_rows<3>(pws, row0, n, (float*)S.p, bulk, bar);
  stage_rows<4>(rots, row0, n, (float*)S.q, bulk, bar);
  stage_rows<3>(scales, row0, n, (float*)S.s, bulk, bar);
  stage_rows<1>(alphas, row0, n, (float*)S.al, bulk, bar);
  if (raw16) {
    if (threadIdx.x == 0) {
      char* r = (char*)raw;
      bulk_load(r, w0 + row0 * WS::W0, (uint32_t)(nt * WS::W0 * 2), bar);
      if constexpr (MODE != GSB_WEIGHTS_FULL) {
        r += nt * WS::W0 * 2;
        bulk_load(r, wa + row0 * WS::WA, (uint32_t)(nt * WS::WA * 2), bar);
        r += nt * WS::WA * 2;
        bulk_load(r, wb + row0 * WS::WB, (uint32_t)(nt * WS::WB * 2), bar);
      }
    }
  } else if constexpr (MODE == GSB_WEIGHTS_FULL) {
    // one copy per row, into the odd-float4 stride
    float* dst = (float*)S.w0;
    if (bulk) {
      bulk_load(dst + threadIdx.x * WS::W0S, w0 + (row0 + threadIdx.x) * WS::W0,
                (uint32_t)(WS::W0 * sizeof(T)), bar);
    } else {
      const int64_t rows = min((int64_t)nt, n - row0);
      for (int e = threadIdx.x; e < rows * WS::W0; e += nt) {
        const int r = e / WS::W0, c = e - r * WS::W0;
        dst[r * WS::W0S + c] = ld(w0, row0 * WS::W0 + e);
      }
    }
  } else {
    stage_rows<WS::W0>(w0, row0, n, (float*)S.w0, bulk, bar);
    stage_rows<WS::WA>(wa, row0, n, (float*)S.wa, bulk, bar);
    stage_rows<WS::WB>(wb, row0, n, (float*)S.wb, bulk, bar);
  }
  __syncthreads();
  if (bulk && !mbar_wait(bar, 0)) {
    if (threadIdx.x == 0) atomicOr(&g_fused_status, kStatusBulkTimeout);
    mbar_wait(bar, 0);  // bounded second wait for copies still in flight
    return kStageFailed;
  }
  return raw16 ? kStagedRawBf16 : kStagedFloat;
}

// Converts `count` raw BF16 values to floats, shared memory to shared memory.
__device__ __forceinline__ void bf16_rows_to_float(const __nv_bfloat16* src, float* dst,
                                                   int count) {
  for (int e = threadIdx.x; e < count; e += blockDim.x) dst[e] = __bfloat162float(src[e]);
}

// Full-SH rows are 16K floats long, a multiple of 16: written one row per
// thread, the 32 lanes of a warp would hit 2 (or 1) of the 32 shared-memory
// banks.  The adjoint therefore builds its SH-gradient rows at an odd stride
// and packs them before storing them.
template <int W>
struct PadRows {
  static constexpr bool kPad = W > 1 && W % 2 == 0;
  static constexpr int kStride = kPad ? W + 1 : W;
  static constexpr int kExtra = kPad ? W + 1 : 0;  // extra floats per thread
};

// Palette weights of one Gaussian from its staged parameter rows.
template <int MODE, int K, int P, int Q, int R>
__device__ __forceinline__ void weights_of(const float* w0, const float* wa, const float* wb,
                                           const float* Y, float* w) {
  if constexpr (MODE == GSB_WEIGHTS_FULL) {
    sh_weights_full<K>([&](int idx) { return w0[idx]; }, 16, Y, w);
  } else {
    lowrank_weights<K, P, Q, R>(w0, wa, wb, Y, w);
  }
}

// ------------------------------------------------------------- forward
// COL: the record carries the Gaussian's palette colour sum_k w_k pal[k]
// (3 channels) instead of its K weights -- the palette-edit render, which
// the reference gets by baking the palette into RGB SH coefficients and
// rendering those (gsplat/gsmodel.py:488-509, 14-26).
template <int MODE, int K, int P, int Q, int R, typename T, bool COL>
__global__ void __launch_bounds__(kFuseThreads)
    k_render_preprocess(int64_t n, uint32_t gx, uint32_t gy, CamArgs cam,
                        const float* __restrict__ pal,
                        const float* __restrict__ pws, const float* __restrict__ rots,
                        const float* __restrict__ scales, const float* __restrict__ alphas,
                        const T* __restrict__ w0, const T* __restrict__ wa,
                        const T* __restrict__ wb, float4* __restrict__ records,
                        uint2* __restrict__ rects, uint32_t* __restrict__ dkeys,
                        uint32_t* __restrict__ counts, uint32_t* __restrict__ part_sums,
                        uint32_t* __restrict__ part_max, float* __restrict__ depths_out) {
  pdl_wait();
  using WS = WRows<MODE, K, P, Q, R>;
  constexpr int V = RecordLayout<COL ? 3 : K>::kVec4;
  static_assert(WS::INS >= 4 * V, "the record span reuses the input staging area");
  extern __shared__ __align__(16) float sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t warp_tot[kFuseThreads / 32], warp_max[kFuseThreads / 32];
  static_assert(kFuseThreads == kPartBlock, "one part per preprocess block");
  __shared__ float s_pal[COL ? 3 * K : 1];
  if constexpr (COL) {
    if (threadIdx.x < 3 * K) s_pal[threadIdx.x] = pal[threadIdx.x];
  }
  const int nt = blockDim.x, t = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * nt;
  float* raw = sm + nt * WS::INS;
  const int how = stage_params<MODE, K, P, Q, R, T>(n, row0, pws, rots, scales, alphas, w0, wa,
                                                    wb, sm, raw, &bar);
  const bool staged = how != kStageFailed;
  const Staged<MODE, K, P, Q, R> S(sm);
  if constexpr (sizeof(T) == 2) {  // raw BF16 colour rows -> their float rows
    if (how == kStagedRawBf16) {
      const __nv_bfloat16* r = (const __nv_bfloat16*)raw;
      if constexpr (MODE == GSB_WEIGHTS_FULL) {
        // 8 values (16 bytes) at a time into the odd-float4 stride
        constexpr int C8 = WS::W0 / 8;
        for (int e = t; e < nt * C8; e += nt) {
          const int rr = e / C8, c = e - rr * C8;
          const uint4 v = reinterpret_cast<const uint4*>(r)[e];
          const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
          const float2 a = __bfloat1622float2(h[0]), b = __bfloat1622float2(h[1]);
          const float2 c2 = __bfloat1622float2(h[2]), d = __bfloat1622float2(h[3]);
          float4* dst = reinterpret_cast<float4*>((float*)S.w0 + rr * WS::W0S + 8 * c);
          dst[0] = make_float4(a.x, a.y, b.x, b.y);
          dst[1] = make_float4(c2.x, c2.y, d.x, d.y);
        }
      }
      // (low-rank BF16 factors are read raw: their row strides are odd)
    }
    if constexpr (MODE == GSB_WEIGHTS_FULL) __syncthreads();
  }
  const int64_t i = row0 + t;
  uint32_t cnt = 0, dk = 0;
  float f[4 * V];  // this Gaussian's record (kept until the block writes its records)
  if (staged && i < n) {
    const CamRegs cr = load_cam(cam);
    float depth_out = kBadDepth;
    const float3 pw = make_float3(S.p[3 * t], S.p[3 * t + 1], S.p[3 * t + 2]);
    const Projected p = project_point(pw, cr.R, make_float3(cr.t[0], cr.t[1], cr.t[2]), cam.fx,
                                      cam.fy, cam.cx, cam.cy);
    if (p.valid) {
      float cov3[6], cov2[3], conic[3];
      int ext[2];
      covariance_3d(make_float4(S.q[4 * t], S.q[4 * t + 1], S.q[4 * t + 2], S.q[4 * t + 3]),
                    make_float3(S.s[3 * t], S.s[3 * t + 1], S.s[3 * t + 2]), cov3, nullptr,
                    nullptr);
      covariance_2d(cov3, p.x, p.y, p.z, cr.R, cam.fx, cam.fy, cam.tanx, cam.tany, cov2, nullptr,
                    nullptr);
      if (conic_and_extent(cov2[0], cov2[1], cov2[2], conic, ext, nullptr)) {
        const TileRect r = tile_rect(p.ux, p.uy, (float)ext[0], (float)ext[1], gx, gy);
        cnt = (r.y1 - r.y0) * (r.x1 - r.x0);
        if (cnt > 0) {
          depth_out = p.z;
          dk = __float2uint_rz(p.z * 1000);
          rects[i] = make_uint2(r.x0 | (r.y0 << 16), r.x1 | (r.y1 << 16));
          float dir[3], Y[16], w[K];
          view_direction(pw, make_float3(cr.c[0], cr.c[1], cr.c[2]), dir, nullptr, nullptr);
          sh_basis(dir, WS::L + 1, Y);
          if constexpr (MODE == GSB_WEIGHTS_FULL) {
            // the row as float4s (conflict-free at the odd-float4 stride)
            float row[WS::W0];
            const float4* src = reinterpret_cast<const float4*>(S.w0 + t * WS::W0S);
#pragma unroll
            for (int c = 0; c < WS::W0 / 4; ++c) {
              const float4 v = src[c];
              row[4 * c] = v.x;
              row[4 * c + 1] = v.y;
              row[4 * c + 2] = v.z;
              row[4 * c + 3] = v.w;
            }
            sh_weights_full<K>([&](int idx) { return row[idx]; }, 16, Y, w);
          } else if (sizeof(T) == 2 && how == kStagedRawBf16) {
            const __nv_bfloat16* r = (const __nv_bfloat16*)raw;
            lowrank_weights<K, P, Q, R>(r + t * WS::W0, r + nt * WS::W0 + t * WS::WA,
                                        r + nt * (WS::W0 + WS::WA) + t * WS::WB, Y, w);
          } else {
            weights_of<MODE, K, P, Q, R>(S.w0 + t * WS::W0, S.wa + t * WS::WA, S.wb + t * WS::WB,
                                         Y, w);
          }
          record_head(p.ux, p.uy, conic[0], conic[1], conic[2], S.al[t], f);
          if constexpr (COL) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              float acc = 0.f;
#pragma unroll
              for (int k = 0; k < K; ++k) acc += w[k] * s_pal[3 * k + c];
              f[record_channel(c)] = acc;
            }
          } else {
#pragma unroll
            for (int k = 0; k < K; ++k) f[record_channel(k)] = w[k];
          }
        }
      }
    }
    counts[i] = cnt;
    dkeys[i] = dk;
    if (depths_out) depths_out[i] = depth_out;
  }
  // block totals for the patch-count scan and the largest depth key
  const int lane = t & 31, w = t >> 5;
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[w] = incl;
  uint32_t m = dk;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) warp_max[w] = m;
  __syncthreads();  // every thread is done with the staged inputs from here on
  if (t == 0) {  // this block's part of the patch-count scan (k_scan_block_sums)
    uint32_t tot = 0, mx = 0;
    for (int k = 0; k < nt / 32; ++k) {
      tot += warp_tot[k];
      mx = max(mx, warp_max[k]);
    }
    part_sums[blockIdx.x] = tot;
    part_max[blockIdx.x] = mx;
  }
  // records: assembled over the input staging area, written as one span (the
  // rows of Gaussians without patches are never read)
  float4* s_rec = reinterpret_cast<float4*>(sm);
  if (cnt > 0) {
#pragma unroll
    for (int v = 0; v < V; ++v)
      s_rec[t * V + v] = make_float4(f[4 * v], f[4 * v + 1], f[4 * v + 2], f[4 * v + 3]);
  }
  const int64_t rows = min((int64_t)nt, n - row0);
  if (rows == nt && aligned16(records + row0 * V)) {
    fence_proxy_async_shared();
    __syncthreads();
    if (t == 0) {
      bulk_store(records + row0 * V, s_rec, (uint32_t)(nt * V * 16));
      bulk_store_drain();
    }
  } else {
    __syncthreads();
    for (int j = t; j < rows * V; j += nt) records[row0 * V + j] = s_rec[j];
  }
}

// ------------------------------------------------------------ backward
// Shared-memory plan of the backward kernel: only the rows it reads are
// staged -- the centre (view direction), the weight gradients from the
// compositing adjoint, the low-rank factors (their gradients need each
// other), and with GEOM also rotation, scale, opacity and the SH
// coefficients (the view-direction term); the parameter gradients are
// assembled in shared memory and written back as contiguous spans.
template <int MODE, int K, int P, int Q, int R, bool GEOM>
struct BwdPlan {
  using WS = WRows<MODE, K, P, Q, R>;
  static constexpr bool kW0 = GEOM && MODE == GSB_WEIGHTS_FULL;  // shs needed
  static constexpr bool kAB = MODE != GSB_WEIGHTS_FULL;
  // input regions, in floats per Gaussian (offset = prefix * blockDim)
  static constexpr int P_ = 3, G_ = K, Q_ = GEOM ? 4 : 0, S_ = GEOM ? 3 : 0, W0_ = kW0 ? WS::W0 : 0,
                       A_ = kAB ? WS::WA : 0, B_ = kAB ? WS::WB : 0;
  static constexpr int o_p = 0, o_g = o_p + P_, o_q = o_g + G_, o_s = o_q + Q_, o_w0 = o_s + S_,
                       o_a = o_w0 + W0_, o_b = o_a + A_, in_floats = o_b + B_;
  // output regions: d_w0, d_wa, d_wb
  static constexpr int out_floats = WS::W0 + WS::WA + WS::WB;
  static constexpr int o_dw0 = in_floats, o_dwa = o_dw0 + WS::W0, o_dwb = o_dwa + WS::WA;
  static constexpr int floats = in_floats + out_floats;
};

// Raw BF16 rows of the backward's staged colour parameters (bulk-copied,
// then converted into their float areas), in floats per thread.
template <int MODE, int K, int P, int Q, int R, bool GEOM, typename T>
struct BwdRaw {
  using BP = BwdPlan<MODE, K, P, Q, R, GEOM>;
  static constexpr int kHalfs = sizeof(T) == 2 ? BP::W0_ + BP::A_ + BP::B_ : 0;
  static constexpr int kFloats = (kHalfs + 1) / 2;
};

// Stages the block's input rows.  With `acc` (gradients added to what the
// outputs hold) and a full, aligned block, the outputs' current rows are
// bulk-loaded into the block's gradient area in the same transaction, so the
// adjoint adds into them in shared memory and stores them like fresh rows.
// Returns 0 when a bulk copy timed out, 2 when the gradient rows were
// preloaded, else 1.
template <int MODE, int K, int P, int Q, int R, bool GEOM, typename T>
__device__ __forceinline__ int stage_backward(int64_t n, int64_t row0, const float* pws,
                                              const float* rots, const float* scales,
                                              const T* w0, const T* wa, const T* wb,
                                              const float* g_feat, bool acc, const float* d_w0,
                                              const float* d_wa, const float* d_wb, float* sm,
                                              float* raw, uint64_t* bar) {
  using BP = BwdPlan<MODE, K, P, Q, R, GEOM>;
  using WS = WRows<MODE, K, P, Q, R>;
  const int nt = blockDim.x;
  const bool full = row0 + nt <= n;
  bool bulk = full && aligned16(pws + row0 * 3) && aligned16(g_feat + row0 * K);
  if (GEOM) bulk = bulk && aligned16(rots + row0 * 4) && aligned16(scales + row0 * 3);
  if (BP::kW0)
    bulk = bulk && aligned16(w0 + row0 * WS::W0) && (nt * WS::W0 * sizeof(T)) % 16 == 0;
  if (BP::kAB)
    bulk = bulk && aligned16(wa + row0 * WS::WA) && aligned16(wb + row0 * WS::WB) &&
           (nt * WS::WA * sizeof(T)) % 16 == 0 && (nt * WS::WB * sizeof(T)) % 16 == 0;
  const bool raw16 = bulk && sizeof(T) == 2;
  bool pre = bulk && acc && aligned16(d_w0 + row0 * WS::W0) && (nt * WS::W0 * 4) % 16 == 0;
  if (MODE != GSB_WEIGHTS_FULL)
    pre = pre && aligned16(d_wa + row0 * WS::WA) && aligned16(d_wb + row0 * WS::WB) &&
          (nt * WS::WA * 4) % 16 == 0 && (nt * WS::WB * 4) % 16 == 0;
  if (bulk && threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(bar, (uint32_t)(nt * (BP::P_ + BP::G_ + BP::Q_ + BP::S_) * 4 +
                                          nt * (BP::W0_ + BP::A_ + BP::B_) * sizeof(T) +
                                          (pre ? nt * BP::out_floats * 4 : 0)));
  }
  if (pre && threadIdx.x == 0) {
    bulk_load(sm + nt * BP::o_dw0, d_w0 + row0 * WS::W0, (uint32_t)(nt * WS::W0 * 4), bar);
    if constexpr (MODE != GSB_WEIGHTS_FULL) {
      bulk_load(sm + nt * BP::o_dwa, d_wa + row0 * WS::WA, (uint32_t)(nt * WS::WA * 4), bar);
      bulk_load(sm + nt * BP::o_dwb, d_wb + row0 * WS::WB, (uint32_t)(nt * WS::WB * 4), bar);
    }
  }
  stage_rows<3>(pws, row0, n, sm + nt * BP::o_p, bulk, bar);
  stage_rows<K>(g_feat, row0, n, sm + nt * BP::o_g, bulk, bar);
  if constexpr (GEOM) {
    stage_rows<4>(rots, row0, n, sm + nt * BP::o_q, bulk, bar);
    stage_rows<3>(scales, row0, n, sm + nt * BP::o_s, bulk, bar);
  }
  if (raw16) {
    if (threadIdx.x == 0) {
      char* r = (char*)raw;
      if constexpr (BP::kW0) {
        bulk_load(r, w0 + row0 * WS::W0, (uint32_t)(nt * WS::W0 * 2), bar);
        r += nt * WS::W0 * 2;
      }
      if constexpr (BP::kAB) {
        bulk_load(r, wa + row0 * WS::WA, (uint32_t)(nt * WS::WA * 2), bar);
        r += nt * WS::WA * 2;
        bulk_load(r, wb + row0 * WS::WB, (uint32_t)(nt * WS::WB * 2), bar);
      }
    }
  } else {
    if constexpr (BP::kW0) stage_rows<WS::W0>(w0, row0, n, sm + nt * BP::o_w0, bulk, bar);
    if constexpr (BP::kAB) {
      stage_rows<WS::WA>(wa, row0, n, sm + nt * BP::o_a, bulk, bar);
      stage_rows<WS::WB>(wb, row0, n, sm + nt * BP::o_b, bulk, bar);
    }
  }
  __syncthreads();
  if (bulk && !mbar_wait(bar, 0)) {
    if (threadIdx.x == 0) atomicOr(&g_fused_status, kStatusBulkTimeout);
    mbar_wait(bar, 0);  // bounded second wait for copies still in flight
    return 0;
  }
  if constexpr (sizeof(T) == 2) {  // raw BF16 rows -> their float areas
    if (raw16) {
      const __nv_bfloat16* r = (const __nv_bfloat16*)raw;
      if constexpr (BP::kW0) {
        bf16_rows_to_float(r, sm + nt * BP::o_w0, nt * WS::W0);
        r += nt * WS::W0;
      }
      if constexpr (BP::kAB) {
        bf16_rows_to_float(r, sm + nt * BP::o_a, nt * WS::WA);
        bf16_rows_to_float(r + nt * WS::WA, sm + nt * BP::o_b, nt * WS::WB);
      }
    }
    __syncthreads();
  }
  return pre ? 2 : 1;
}

// Writes one gradient array's block span from shared memory: one bulk copy
// for a full, aligned block, else a coalesced per-thread copy.
template <int ROWLEN>
__device__ __forceinline__ void write_rows(float* g, int64_t row0, int64_t n, const float* s) {
  const int nt = blockDim.x;
  if (row0 + nt <= n && aligned16(g + row0 * ROWLEN)) {
    if (threadIdx.x == 0) bulk_store(g + row0 * ROWLEN, s, (uint32_t)(nt * ROWLEN * 4));
  } else {
    stage_out_plain<ROWLEN>(g, row0, n, s);
  }
}

// Adds one gradient array's block span (`rows` rows) from shared memory to
// global memory, coalesced, with kAddBatch loads in flight per thread before
// the adds and stores (one read-add-write at a time would pay a global-memory
// latency per element).  Element e of the span comes from s[src(e)].
constexpr int kAddBatch = 8;
template <int ROWLEN, typename Src>
__device__ __forceinline__ void add_span(float* g, int64_t row0, int64_t rows, Src src) {
  const int total = (int)rows * ROWLEN, nt = blockDim.x;
  float* base = g + row0 * ROWLEN;
  for (int j0 = threadIdx.x; j0 < total; j0 += nt * kAddBatch) {
    float v[kAddBatch];
#pragma unroll
    for (int u = 0; u < kAddBatch; ++u) {
      const int j = j0 + u * nt;
      v[u] = j < total ? base[j] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kAddBatch; ++u) {
      const int j = j0 + u * nt;
      if (j < total) base[j] = v[u] + src(j);
    }
  }
}

template <int ROWLEN>
__device__ __forceinline__ void add_rows(float* g, int64_t row0, int64_t rows, const float* s) {
  add_span<ROWLEN>(g, row0, rows, [s](int j) { return s[j]; });
}

// g_feat [n,K] (dL/dweights), g_u [n,2], g_conic [n,3] come from the
// compositing adjoint, which also writes dL/dalpha directly.  Without GEOM
// (weights-only backward: g_u, g_conic and the geometry outputs unused) only
// the weight-parameter gradients are formed.
template <int MODE, int K, int P, int Q, int R, typename T, bool GEOM>
__global__ void __launch_bounds__(kFuseThreads)
    k_render_backward_pre(int64_t n, CamArgs cam, const float* __restrict__ pws,
                          const float* __restrict__ rots, const float* __restrict__ scales,
                          const T* __restrict__ w0, const T* __restrict__ wa,
                          const T* __restrict__ wb, const float* __restrict__ g_feat,
                          const float* __restrict__ g_u, const float* __restrict__ g_conic,
                          float* __restrict__ d_pws, float* __restrict__ d_rots,
                          float* __restrict__ d_scales, float* __restrict__ d_w0,
                          float* __restrict__ d_wa, float* __restrict__ d_wb, bool acc) {
  pdl_wait();
  using WS = WRows<MODE, K, P, Q, R>;
  using BP = BwdPlan<MODE, K, P, Q, R, GEOM>;
  constexpr int L = WS::L;
  extern __shared__ __align__(16) float sm[];
  __shared__ __align__(8) uint64_t bar;
  const int nt = blockDim.x, t = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * nt;
  float* raw = sm + nt * (BP::floats + PadRows<WS::W0>::kExtra);
  const int staged = stage_backward<MODE, K, P, Q, R, GEOM, T>(
      n, row0, pws, rots, scales, w0, wa, wb, g_feat, acc, d_w0, d_wa, d_wb, sm, raw, &bar);
  if (!staged) return;
  const bool pre = staged == 2;  // the outputs' rows are in the gradient area: add to them
  const auto put = [pre](float* d, float v) { *d = pre ? *d + v : v; };
  const int64_t i = row0 + t;
  // full-SH gradient rows are built at an odd stride past the plan's regions
  // (see PadRows) and packed contiguously before they are stored
  using PR = PadRows<WS::W0>;
  float* o_w0 = PR::kPad ? sm + nt * BP::floats + t * PR::kStride : sm + nt * BP::o_dw0 + t * WS::W0;
  float* o_wa = sm + nt * BP::o_dwa + t * WS::WA;
  float* o_wb = sm + nt * BP::o_dwb + t * WS::WB;
  if (i < n) {
    const float* s_p = sm + nt * BP::o_p + 3 * t;
    const float* s_g = sm + nt * BP::o_g + K * t;
    const float* s_wa = sm + nt * BP::o_a + t * WS::WA;
    const float* s_wb = sm + nt * BP::o_b + t * WS::WB;
    const float3 pw = make_float3(s_p[0], s_p[1], s_p[2]);
    float gw[K];
#pragma unroll
    for (int k = 0; k < K; ++k) gw[k] = s_g[k];
    const CamRegs cr = load_cam(cam);
    float dir[3], nd[3], ninv, Y[16];
    view_direction(pw, make_float3(cr.c[0], cr.c[1], cr.c[2]), dir, nd, &ninv);
    sh_basis(dir, L + 1, Y);
    float dpw[3] = {0.f, 0.f, 0.f}, dq[4] = {0.f, 0.f, 0.f, 0.f}, ds[3] = {0.f, 0.f, 0.f};
    float G[48];
    if constexpr (GEOM) {
      const float* s_q = sm + nt * BP::o_q + 4 * t;
      const float* s_s = sm + nt * BP::o_s + 3 * t;
      const float gu[2] = {g_u[2 * i], g_u[2 * i + 1]};
      const float gq[3] = {g_conic[3 * i], g_conic[3 * i + 1], g_conic[3 * i + 2]};
      const bool any = gu[0] != 0.f || gu[1] != 0.f || gq[0] != 0.f || gq[1] != 0.f || gq[2] != 0.f;
      const float4 q = make_float4(s_q[0], s_q[1], s_q[2], s_q[3]);
      const float3 sc = make_float3(s_s[0], s_s[1], s_s[2]);
      const Projected p = project_point(pw, cr.R, make_float3(cr.t[0], cr.t[1], cr.t[2]), cam.fx,
                                        cam.fy, cam.cx, cam.cy);
      if (any && p.valid) {
        // conic -> cov2d -> (cov3d, pc); u -> pc
        float cov3[6], M3[9], Rq[9], cov2[3], M2[6], xy[2];
        covariance_3d(q, sc, cov3, M3, Rq);
        covariance_2d(cov3, p.x, p.y, p.z, cr.R, cam.fx, cam.fy, cam.tanx, cam.tany, cov2, M2, xy);
        // the chain in FP64 (one per Gaussian: cheap), from the FP32 forward
        // values; d conic / d cov2d with the b^2 / det^2 entries written as
        // such rather than as 1/det - ac/det^2, which cancels
        const double a = cov2[0], b = cov2[1], c = cov2[2];
        const double det = a * c - b * b;
        if (det != 0.0 && !isnan(det)) {
          const double det_inv = 1.0 / det, d2 = det_inv * det_inv;
          const double Ji[9] = {-c * c * d2, 2 * b * c * d2, -b * b * d2,
                                b * c * d2,  -2 * b * b * d2 - det_inv, a * b * d2,
                                -b * b * d2, 2 * a * b * d2, -a * a * d2};
          double dc2[3];
#pragma unroll
          for (int j = 0; j < 3; ++j) dc2[j] = gq[0] * Ji[j] + gq[1] * Ji[3 + j] + gq[2] * Ji[6 + j];
          double c3d[6], M2d[6], Rd[9];
#pragma unroll
          for (int u = 0; u < 6; ++u) { c3d[u] = cov3[u]; M2d[u] = M2[u]; }
#pragma unroll
          for (int u = 0; u < 9; ++u) Rd[u] = cr.R[u];
          double d3[18], dpc_m[9];
          cov2d_jacobians<double>(c3d, M2d, Rd, xy[0], xy[1], p.z, cam.fx, cam.fy, d3, dpc_m);
          double dS[6];
#pragma unroll
          for (int u = 0; u < 6; ++u)
            dS[u] = dc2[0] * d3[u] + dc2[1] * d3[6 + u] + dc2[2] * d3[12 + u];
          double dpc[3];
#pragma unroll
          for (int j = 0; j < 3; ++j)
            dpc[j] = dc2[0] * dpc_m[j] + dc2[1] * dpc_m[3 + j] + dc2[2] * dpc_m[6 + j];
          const double zi = 1.0 / p.z, zi2 = zi * zi;
          dpc[0] += gu[0] * (cam.fx * zi);
          dpc[1] += gu[1] * (cam.fy * zi);
          dpc[2] += gu[0] * (-(p.x * (double)cam.fx) * zi2) + gu[1] * (-(p.y * (double)cam.fy) * zi2);
#pragma unroll
          for (int j = 0; j < 3; ++j)
            dpw[j] += (float)(Rd[j] * dpc[0] + Rd[3 + j] * dpc[1] + Rd[6 + j] * dpc[2]);
          double M3d[9], Rqd[9];
#pragma unroll
          for (int u = 0; u < 9; ++u) { M3d[u] = M3[u]; Rqd[u] = Rq[u]; }
          double jq[24], js[18];
          cov3d_jacobians<double>(q, sc, M3d, Rqd, jq, js);
          double dqd[4] = {0.0, 0.0, 0.0, 0.0}, dsd[3] = {0.0, 0.0, 0.0};
#pragma unroll
          for (int u = 0; u < 6; ++u) {
#pragma unroll
            for (int j = 0; j < 4; ++j) dqd[j] += dS[u] * jq[4 * u + j];
#pragma unroll
            for (int j = 0; j < 3; ++j) dsd[j] += dS[u] * js[3 * u + j];
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) dq[j] += (float)dqd[j];
#pragma unroll
          for (int j = 0; j < 3; ++j) ds[j] += (float)dsd[j];
        }
      }
      sh_basis_grad(dir, L + 1, /*ref_quirk=*/false, G);
    }
    // colour parameters, and (GEOM) the view direction's share of d pws
    float dd[3] = {0.f, 0.f, 0.f};
    if constexpr (MODE == GSB_WEIGHTS_FULL) {
      const float* s_w0 = sm + nt * BP::o_w0 + t * WS::W0;
#pragma unroll
      for (int l = 0; l < 16; ++l)
#pragma unroll
        for (int k = 0; k < K; ++k) {
          o_w0[l * K + k] = gw[k] * Y[l];
          if constexpr (GEOM) {
            if (l > 0) {
              const float cg = gw[k] * s_w0[l * K + k];
              dd[0] += cg * G[3 * l];
              dd[1] += cg * G[3 * l + 1];
              dd[2] += cg * G[3 * l + 2];
            }
          }
        }
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if constexpr (PR::kPad)
          o_w0[k] = gw[k] * SH_C0;  // packed (and added) below
        else
          put(o_w0 + k, gw[k] * SH_C0);
      }
      // dC[p][q] = gw_k Y_{l+1} with g = l*K + k = p*Q + q
#pragma unroll
      for (int pp = 0; pp < P; ++pp) {
        float acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0.f;
#pragma unroll
        for (int qq = 0; qq < Q; ++qq) {
          const int g = pp * Q + qq, k = g % K, l = g / K;
          const float dC = gw[k] * Y[l + 1];
          float coef = 0.f;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            acc[r] += dC * s_wb[r * Q + qq];
            if constexpr (GEOM) coef += s_wa[pp * R + r] * s_wb[r * Q + qq];
          }
          if constexpr (GEOM) {
            const float cg = gw[k] * coef;
            dd[0] += cg * G[3 * (l + 1)];
            dd[1] += cg * G[3 * (l + 1) + 1];
            dd[2] += cg * G[3 * (l + 1) + 2];
          }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) put(o_wa + pp * R + r, acc[r]);
      }
#pragma unroll
      for (int qq = 0; qq < Q; ++qq) {
        float acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = 0.f;
#pragma unroll
        for (int pp = 0; pp < P; ++pp) {
          const int g = pp * Q + qq, k = g % K, l = g / K;
          const float dC = gw[k] * Y[l + 1];
#pragma unroll
          for (int r = 0; r < R; ++r) acc[r] += dC * s_wa[pp * R + r];
        }
#pragma unroll
        for (int r = 0; r < R; ++r) put(o_wb + r * Q + qq, acc[r]);
      }
    }
    if constexpr (GEOM) {
      float Jd[9];
      dir_jacobian(nd, ninv, Jd);
#pragma unroll
      for (int j = 0; j < 3; ++j) dpw[j] += dd[0] * Jd[j] + dd[1] * Jd[3 + j] + dd[2] * Jd[6 + j];
#pragma unroll
      for (int j = 0; j < 3; ++j) d_pws[3 * i + j] = (acc ? d_pws[3 * i + j] : 0.f) + dpw[j];
#pragma unroll
      for (int j = 0; j < 4; ++j) d_rots[4 * i + j] = (acc ? d_rots[4 * i + j] : 0.f) + dq[j];
#pragma unroll
      for (int j = 0; j < 3; ++j) d_scales[3 * i + j] = (acc ? d_scales[3 * i + j] : 0.f) + ds[j];
    }
  }
  // parameter gradients: shared memory -> global, block span by block span;
  // with `acc` and no preloaded rows (a partial or unaligned block), added to
  // what the outputs hold by a coalesced read-add-write
  if (acc && !pre) {
    __syncthreads();
    const int64_t rows = min((int64_t)nt, n - row0);
    if constexpr (PR::kPad) {
      const float* src = sm + nt * BP::floats;
      add_span<WS::W0>(d_w0, row0, rows, [src](int j) {
        const int r = j / WS::W0, c = j - r * WS::W0;
        return src[r * PR::kStride + c];
      });
    } else {
      add_rows<WS::W0>(d_w0, row0, rows, sm + nt * BP::o_dw0);
    }
    if constexpr (MODE != GSB_WEIGHTS_FULL) {
      add_rows<WS::WA>(d_wa, row0, rows, sm + nt * BP::o_dwa);
      add_rows<WS::WB>(d_wb, row0, rows, sm + nt * BP::o_dwb);
    }
    return;
  }
  if constexpr (PR::kPad) {
    __syncthreads();
    float* dst = sm + nt * BP::o_dw0;
    const float* src = sm + nt * BP::floats;
    for (int e = t; e < nt * WS::W0; e += nt) {
      const int r = e / WS::W0, c = e - r * WS::W0;
      dst[e] = pre ? dst[e] + src[r * PR::kStride + c] : src[r * PR::kStride + c];
    }
  }
  fence_proxy_async_shared();
  __syncthreads();
  write_rows<WS::W0>(d_w0, row0, n, sm + nt * BP::o_dw0);
  if constexpr (MODE != GSB_WEIGHTS_FULL) {
    write_rows<WS::WA>(d_wa, row0, n, sm + nt * BP::o_dwa);
    write_rows<WS::WB>(d_wb, row0, n, sm + nt * BP::o_dwb);
  }
  if (threadIdx.x == 0) bulk_store_drain();
}

// ------------------------------------------------------------ dispatch
template <typename Kern>
static int set_smem(Kern kern, int smem) {
  if (smem <= 48 * 1024) return GSB_OK;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return check_launch("render (shared memory attribute)", 0);
  return GSB_OK;
}

template <int MODE, int K, int P, int Q, int R, typename T>
static int launch_fused(const FusedArgs& f, bool backward, cudaStream_t st) {
  using WS = WRows<MODE, K, P, Q, R>;
  const int smem = (WS::INS + FwdExtra<MODE, K, P, Q, R, T>::kRawFloats) * kFuseThreads * 4;
  const int grid = div_up(f.n, kFuseThreads);
  int rc;
  if (!backward) {
    auto kern = f.palette ? k_render_preprocess<MODE, K, P, Q, R, T, true>
                          : k_render_preprocess<MODE, K, P, Q, R, T, false>;
    if ((rc = set_smem(kern, smem))) return rc;
    launch_pdl(kern, dim3(grid), dim3(kFuseThreads), smem, st, f.n, f.gx, f.gy, f.cam, f.palette,
               f.pws, f.rots, f.scales, f.alphas, (const T*)f.w0, (const T*)f.wa, (const T*)f.wb,
               f.st.records, f.st.rects, f.st.dkeys, f.st.counts, f.st.part_sums, f.st.part_max,
               f.depths_out);
    return check_launch("render_preprocess");
  }
  const bool geom = f.g_u != nullptr;
  auto kern = geom ? k_render_backward_pre<MODE, K, P, Q, R, T, true>
                   : k_render_backward_pre<MODE, K, P, Q, R, T, false>;
  const int bsmem = ((geom ? BwdPlan<MODE, K, P, Q, R, true>::floats +
                                 BwdRaw<MODE, K, P, Q, R, true, T>::kFloats
                           : BwdPlan<MODE, K, P, Q, R, false>::floats +
                                 BwdRaw<MODE, K, P, Q, R, false, T>::kFloats) +
                     PadRows<WS::W0>::kExtra) *
                    kFuseThreads * 4;
  if ((rc = set_smem(kern, bsmem))) return rc;
  launch_pdl(kern, dim3(grid), dim3(kFuseThreads), bsmem, st, f.n, f.cam, f.pws, f.rots,
             f.scales, (const T*)f.w0, (const T*)f.wa, (const T*)f.wb, f.g_feat, f.g_u, f.g_conic,
             f.d_pws, f.d_rots, f.d_scales, f.d_w0, f.d_wa, f.d_wb, f.accumulate);
  return check_launch("render_backward");
}

template <typename T>
static int dispatch_fused(int mode, int K, int P, int Q, int R, const FusedArgs& f, bool bwd,
                          cudaStream_t st) {
  if (mode == GSB_WEIGHTS_FULL) {
    switch (K) {
      case 3: return launch_fused<GSB_WEIGHTS_FULL, 3, 0, 0, 0, T>(f, bwd, st);
      case 4: return launch_fused<GSB_WEIGHTS_FULL, 4, 0, 0, 0, T>(f, bwd, st);
      case 5: return launch_fused<GSB_WEIGHTS_FULL, 5, 0, 0, 0, T>(f, bwd, st);
      case 6: return launch_fused<GSB_WEIGHTS_FULL, 6, 0, 0, 0, T>(f, bwd, st);
      case 7: return launch_fused<GSB_WEIGHTS_FULL, 7, 0, 0, 0, T>(f, bwd, st);
      case 8: return launch_fused<GSB_WEIGHTS_FULL, 8, 0, 0, 0, T>(f, bwd, st);
      default: break;
    }
  } else {
#define GSB_FL(KK, PP, QQ, RR)                   \
  if (K == KK && P == PP && Q == QQ && R == RR) \
    return launch_fused<GSB_WEIGHTS_LOWRANK, KK, PP, QQ, RR, T>(f, bwd, st);
    GSB_FL(5, 5, 15, 1) GSB_FL(5, 5, 15, 2) GSB_FL(5, 5, 15, 3) GSB_FL(5, 5, 15, 4)
    GSB_FL(3, 3, 15, 1) GSB_FL(4, 4, 15, 1) GSB_FL(6, 6, 15, 1) GSB_FL(6, 6, 15, 3)
#undef GSB_FL
  }
  set_error("render: unsupported palette parameter shape (mode %d, K=%d, P=%d, Q=%d, rank=%d)",
            mode, K, P, Q, R);
  return GSB_ERR_UNSUPPORTED;
}

int launch_render(int mode, int dtype, int K, int P, int Q, int R, const FusedArgs& f, bool bwd,
                  cudaStream_t st) {
  if (f.n == 0) return GSB_OK;
  return dtype == GSB_DTYPE_BF16 ? dispatch_fused<__nv_bfloat16>(mode, K, P, Q, R, f, bwd, st)
                                 : dispatch_fused<float>(mode, K, P, Q, R, f, bwd, st);
}

const uint32_t* fused_status_word() {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_fused_status) != cudaSuccess) {
    (void)cudaGetLastError();
    return nullptr;
  }
  return (const uint32_t*)p;
}

// Error-path check: one block arms an mbarrier for a 16-byte transaction
// that no copy will ever deliver and waits on it with the given poll limit;
// the wait runs out, the kernel sets the bulk-timeout bit exactly as the
// staging kernels do, and returns.  Nothing is in flight when it exits.
__global__ void k_expire_bulk_wait(uint32_t poll_limit) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_arrive_expect_tx(&bar, 16);
    if (!mbar_wait(&bar, 0, poll_limit)) atomicOr(&g_fused_status, kStatusBulkTimeout);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&bar)) : "memory");
  }
}

int expire_bulk_wait(uint32_t poll_limit, cudaStream_t st) {
  k_expire_bulk_wait<<<1, 32, 0, st>>>(poll_limit);
  return check_launch("debug_expire_bulk_wait");
}

int fused_status(uint32_t* out, bool clear, cudaStream_t st) {
  if (cudaMemcpyFromSymbolAsync(out, g_fused_status, sizeof(uint32_t), 0, cudaMemcpyDeviceToHost,
                                st) != cudaSuccess)
    return check_launch("device_status", 0);
  if (clear) {
    const uint32_t zero = 0;
    if (cudaMemcpyToSymbolAsync(g_fused_status, &zero, sizeof(uint32_t), 0,
                                cudaMemcpyHostToDevice, st) != cudaSuccess)
      return check_launch("device_status", 0);
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return check_launch("device_status", 0);
  return GSB_OK;
}

}  // namespace gsb
