// Tile compositing: forward (draw_weight / draw_color, gsplatcu/kernel.cu:
// 194-372) and its reverse-order adjoint (draw_weight_B / draw_color_B,
// gsplatcu/kernel.cu:1176-1379).
//
// One CTA per 16x16 tile.  In the forward each of the 8 warps owns an 8x4
// block of pixels, one per lane.  In the adjoint each of the 4 warps owns an
// 8x8 block and each lane two pixels of one column, four rows apart, so the
// per-Gaussian loop control and the warp reduction of the gradient terms are
// shared by 64 pixels.  The tile's Gaussian list is staged through shared
// memory in batches of 256 packed records, each thread loading whole records
// (four 16-byte loads for K <= 5) -- the gather measured faster than a
// double-buffered ring filled by per-record 1-D bulk copies or by cp.async
// (the compositing is issue-bound and several blocks per SM already overlap
// one block's staging with the others' compositing).  Within a batch every
// warp first tests 32 records at a time against its pixel block (one record
// per lane, ballot) using the record's conservative support box and then its
// cut ellipse, then walks only the overlapping records in list order, two at
// a time: both records' opacity terms are evaluated before the two blends
// (or, in the adjoint, the two transmittance recoveries) so that their exp()
// chains overlap, and the adjoint sums the two records' gradient vectors in
// one warp reduction.  Per pixel, a record whose Mahalanobis distance exceeds
// its cut is skipped without evaluating exp() -- the reference would skip it
// too (alpha' < 0.002) -- and every other record is evaluated with the
// reference's own FP32 expressions, so skip/stop decisions, contributor
// indices and blended values agree with it.
#include "gsb_geometry.cuh"
#include "gsb_internal.h"

namespace gsb {

constexpr int kBatch = 256;
constexpr int kDrawFwdThreads = 256;  // forward: one pixel per thread, 8x4 pixels per warp
constexpr int kDrawThreads = 128;     // adjoint: two pixels per thread, 8x8 pixels per warp

struct PixelPair {
  int wx, wy;    // warp block origin (8x8)
  int px;        // column
  int py0, py1;  // rows (py1 = py0 + 4)
};

__device__ __forceinline__ PixelPair pixels_of(int tile, int gx) {
  const int tx = tile % gx, ty = tile / gx;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  PixelPair p;
  p.wx = tx * kTile + (w & 1) * 8;
  p.wy = ty * kTile + (w >> 1) * 8;
  p.px = p.wx + (lane & 7);
  p.py0 = p.wy + (lane >> 3);
  p.py1 = p.py0 + 4;
  return p;
}

__device__ __forceinline__ void pixel_of_1px(int tile, int gx, int& wx, int& wy, int& px,
                                             int& py) {
  const int tx = tile % gx, ty = tile / gx;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  wx = tx * kTile + (w & 1) * 8;
  wy = ty * kTile + (w >> 1) * 4;
  px = wx + (lane & 7);
  py = wy + (lane >> 3);
}

// Stage records [first, first+cnt) of the tile list into shared memory,
// vector-major (srec[v * kBatch + slot]) so that per-slot broadcasts and the
// lane-per-slot box test are both conflict-free.
template <int V, int NT>
__device__ __forceinline__ void stage_batch(const int32_t* __restrict__ gsid, int first, int cnt,
                                            const float4* __restrict__ records, float4* srec,
                                            int32_t* sgid) {
  for (int t = threadIdx.x; t < cnt; t += NT) {
    const int g = gsid[first + t];
    const float4* src = records + (int64_t)g * V;
#pragma unroll
    for (int v = 0; v < V; ++v) srec[v * kBatch + t] = __ldg(src + v);
    if (sgid) sgid[t] = g;
  }
}

// First stage of the warp's record test: does the record's support box
// u +- (hx, hy) meet the pixel block [x0, x0+ex] x [y0, y0+ey]?  Written so
// that a non-finite centre passes (as an unbounded box does) and an empty
// box (-inf extents) fails.
__device__ __forceinline__ bool box_meets_block(float4 v0, float4 v2, int x0, int y0, int ex,
                                                int ey) {
  const float hx = 0.5f * (float)ex, hy = 0.5f * (float)ey;
  return !(fabsf(v0.x - ((float)x0 + hx)) > v2.x + hx) &&
         !(fabsf(v0.y - ((float)y0 + hy)) > v2.y + hy);
}

// Second, exact stage of the warp's record test: can the record's cut
// ellipse d^T Q d <= c2 reach the pixel block [x0,x1] x [y0,y1] at all?
// The minimum of the quadratic over the (continuous) block is 0 when the
// centre lies inside, else it is attained on one of the four edges, where it
// is a clamped 1-D quadratic minimum.  The record is dropped only when that
// minimum exceeds c2 (the cut already widened for the rounding of the FP32
// quadratic form): every pixel of the block would then fail the per-pixel
// test, so the results do not change.  Records whose conic is degenerate or
// ill-conditioned carry c2 = +inf and always pass.
__device__ __forceinline__ bool ellipse_meets_block(float4 v0, float4 v1, float4 v2, float x0,
                                                    float y0, float x1, float y1) {
  const float ux = v0.x, uy = v0.y, qa = v0.z, qb = v0.w, qc = v1.x, c2 = v1.y;
  const float ia = v2.z, ic = v2.w;
  if (!(c2 < INFINITY) || !(isfinite(ux) && isfinite(uy)) ||
      (ux >= x0 && ux <= x1 && uy >= y0 && uy <= y1))
    return true;
  float m = INFINITY;
  // vertical edges x = x0, x1: d_x fixed, d_y free in [uy - y1, uy - y0]
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const float dx = ux - (e ? x1 : x0);
    const float dy = fminf(uy - y0, fmaxf(uy - y1, -qb * dx * ic));
    m = fminf(m, qa * dx * dx + dy * (2.f * qb * dx + qc * dy));
  }
  // horizontal edges y = y0, y1
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const float dy = uy - (e ? y1 : y0);
    const float dx = fminf(ux - x0, fmaxf(ux - x1, -qb * dy * ia));
    m = fminf(m, qc * dy * dy + dx * (2.f * qb * dy + qa * dx));
  }
  return !(m > c2);
}

template <int K>
__device__ __forceinline__ void load_feats(const float4* srec, int j, float v2w, float* f) {
  f[0] = v2w;  // channel 0 sits in v1.w
#pragma unroll
  for (int k = 1; k < K; ++k) {
    const int idx = record_channel(k);  // float index inside the record
    const float4 q = srec[(idx >> 2) * kBatch + j];
    f[k] = (idx & 3) == 0 ? q.x : (idx & 3) == 1 ? q.y : (idx & 3) == 2 ? q.z : q.w;
  }
}

// ------------------------------------------------------ tile launch order
// Blocks are launched in blockIdx order, a wave at a time.  Compositing a
// tile costs roughly its list length, which varies by orders of magnitude
// across an image, so launching tiles in raster order leaves the last waves
// waiting on a few long tiles.  The compositing kernels instead take their
// tile from a launch order, longest list first (a largest-first schedule):
// lengths binned at a quarter octave, descending; order within a bin is
// arbitrary.  Measured at 1M Gaussians, 1080p: forward 0.309 -> 0.280 ms,
// adjoint 0.436 -> 0.372 ms (0.220 -> 0.164 and 0.317 -> 0.273 ms for a
// distant view).  The results do not depend on the order.
constexpr int kOrderThreads = 1024, kOrderBins = 128;

__device__ __forceinline__ int order_bin(int2 rg) {
  const uint32_t x = (uint32_t)max(0, rg.y - rg.x) + 1u;   // >= 1
  const int msb = 31 - __clz(x);
  const int frac = msb >= 2 ? (int)((x >> (msb - 2)) & 3u) : (int)((x << (2 - msb)) & 3u);
  return kOrderBins - 1 - min(kOrderBins - 1, 4 * msb + frac);  // longest first
}

__global__ void __launch_bounds__(kOrderThreads)
    k_tile_order(const int2* __restrict__ ranges, int tiles, int32_t* __restrict__ order) {
  pdl_wait();
  __shared__ int cnt[kOrderBins];
  if (threadIdx.x < kOrderBins) cnt[threadIdx.x] = 0;
  __syncthreads();
  for (int t = threadIdx.x; t < tiles; t += kOrderThreads) atomicAdd(&cnt[order_bin(ranges[t])], 1);
  __syncthreads();
  if (threadIdx.x < 32) {  // exclusive scan of the bins, 4 per lane
    const int lane = threadIdx.x;
    int v[kOrderBins / 32], sum = 0;
#pragma unroll
    for (int k = 0; k < kOrderBins / 32; ++k) {
      v[k] = cnt[lane * (kOrderBins / 32) + k];
      sum += v[k];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    int run = incl - sum;
#pragma unroll
    for (int k = 0; k < kOrderBins / 32; ++k) {
      cnt[lane * (kOrderBins / 32) + k] = run;
      run += v[k];
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < tiles; t += kOrderThreads)
    order[atomicAdd(&cnt[order_bin(ranges[t])], 1)] = t;
}

static int launch_tile_order(const int2* ranges, int tiles, int32_t* order, cudaStream_t st) {
  launch_pdl(k_tile_order, dim3(1), dim3(kOrderThreads), 0, st, ranges, tiles, order);
  return check_launch("tile order");
}

// ------------------------------------------------------------- forward
// Composites one 16x16 tile of one image (draw_weight / draw_color,
// gsplatcu/kernel.cu:283-372): ranges/gsid/records of that image's tile
// lists, K channels, final_tau of empty tiles = tau_init, `srec` the block's
// staging buffer (V x kBatch float4s).  Called by all threads of a block; it
// starts with a block barrier, so the buffer may still be in use by the
// block's previous tile when it is called.
template <int K>
__device__ __forceinline__ void draw_tile(int tile, int H, int W, int gx,
                                          const int2* __restrict__ ranges,
                                          const int32_t* __restrict__ gsid,
                                          const float4* __restrict__ records, float tau_init,
                                          float* __restrict__ out, int32_t* __restrict__ contrib,
                                          float* __restrict__ final_tau, float4* srec) {
  constexpr int V = RecordLayout<K>::kVec4;
  int wx, wy, px, py;
  pixel_of_1px(tile, gx, wx, wy, px, py);
  const bool inside = px < W && py < H;
  const int2 rg = ranges[tile];
  const int n = rg.y - rg.x;
  float acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.f;
  float T = 1.f;
  int cont = 0;
  bool done = !inside;
  for (int base = 0; base < n; base += kBatch) {
    const int cnt = min(kBatch, n - base);
    __syncthreads();
    stage_batch<V, kDrawFwdThreads>(gsid, rg.x + base, cnt, records, srec, nullptr);
    __syncthreads();
    if (!__all_sync(0xffffffffu, done)) {
      for (int s = 0; s < cnt; s += 32) {
        const int j = s + (threadIdx.x & 31);
        bool ov = j < cnt && box_meets_block(srec[j], srec[2 * kBatch + j], wx, wy, 7, 3);
        if (ov)
          ov = ellipse_meets_block(srec[j], srec[kBatch + j], srec[2 * kBatch + j], (float)wx,
                                   (float)wy, (float)(wx + 7), (float)(wy + 3));
        unsigned mask = __ballot_sync(0xffffffffu, ov);
        while (mask) {
          const int jj = s + __ffs(mask) - 1;
          mask &= mask - 1;
          if (mask) {
            // two records at once: both opacity terms first, so that their
            // exp() chains overlap, then the two blends in list order
            const int jb = s + __ffs(mask) - 1;
            mask &= mask - 1;
            if (done) continue;
            const float4 a0 = srec[jj], a1 = srec[kBatch + jj];
            const float4 b0 = srec[jb], b1 = srec[kBatch + jb];
            const float dxa = a0.x - (float)px, dya = a0.y - (float)py;
            const float dxb = b0.x - (float)px, dyb = b0.y - (float)py;
            const float ma = fmaxf(0.0f, maha_sq(a0.z, a0.w, a1.x, dxa, dya));
            const float mb = fmaxf(0.0f, maha_sq(b0.z, b0.w, b1.x, dxb, dyb));
            const float apa = fminf(kAlphaMax, a1.z * expf(-0.5f * ma));
            const float apb = fminf(kAlphaMax, b1.z * expf(-0.5f * mb));
            if (!(ma > a1.y) && !(apa < kAlphaMin)) {
              float f[K];
              load_feats<K>(srec, jj, a1.w, f);
#pragma unroll
              for (int k = 0; k < K; ++k) acc[k] += T * apa * f[k];
              cont = base + jj + 1;
              T *= (1.f - apa);
              if (T < kTransMin) done = true;
            }
            if (!done && !(mb > b1.y) && !(apb < kAlphaMin)) {
              float f[K];
              load_feats<K>(srec, jb, b1.w, f);
#pragma unroll
              for (int k = 0; k < K; ++k) acc[k] += T * apb * f[k];
              cont = base + jb + 1;
              T *= (1.f - apb);
              if (T < kTransMin) done = true;
            }
            continue;
          }
          if (done) continue;
          const float4 v0 = srec[jj];           // ux uy qa qb
          const float4 v1 = srec[kBatch + jj];  // qc c2 alpha ch0
          const float dx = v0.x - (float)px, dy = v0.y - (float)py;
          const float maha = fmaxf(0.0f, maha_sq(v0.z, v0.w, v1.x, dx, dy));
          if (maha > v1.y) continue;
          const float ap = fminf(kAlphaMax, v1.z * expf(-0.5f * maha));
          if (ap < kAlphaMin) continue;
          float f[K];
          load_feats<K>(srec, jj, v1.w, f);
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] += T * ap * f[k];
          cont = base + jj + 1;
          T *= (1.f - ap);
          if (T < kTransMin) done = true;
        }
        if (__all_sync(0xffffffffu, done)) break;
      }
    }
    if (!__syncthreads_or(!done)) break;
  }
  if (inside) {
    const int64_t pix = (int64_t)py * W + px, hw = (int64_t)H * W;
#pragma unroll
    for (int k = 0; k < K; ++k) out[k * hw + pix] = acc[k];
    contrib[pix] = cont;
    final_tau[pix] = n > 0 ? T : tau_init;
  }
}

template <int K>
__global__ void __launch_bounds__(kDrawFwdThreads, 4)
    k_draw(int H, int W, int gx, const int2* __restrict__ ranges, const int32_t* __restrict__ gsid,
           const float4* __restrict__ records, const int32_t* __restrict__ order,
           float tau_init, float* __restrict__ out, int32_t* __restrict__ contrib,
           float* __restrict__ final_tau) {
  pdl_wait();
  __shared__ float4 srec[RecordLayout<K>::kVec4 * kBatch];
  draw_tile<K>(order[blockIdx.x], H, W, gx, ranges, gsid, records, tau_init, out, contrib,
               final_tau, srec);
}

// ------------------------------------------------- batched (persistent) draw
// One image of a batch: its packed records, tile lists and outputs, and the
// index of its first tile in the batch's work queue.
struct DrawJob {
  const float4* records;
  const int2* ranges;
  const int32_t* gsid;
  float* out;
  int32_t* contrib;
  float* final_tau;
  int W, H, gx, item0;
  float tau_init;
  int pad[3];
};
static_assert(sizeof(DrawJob) == 80, "DrawJob layout");

// Device work queue of a batch: (image, tile) items numbered 0..total-1
// image by image; `next` is the next unclaimed item (zero at launch).
struct DrawQueue {
  uint32_t njobs, total, next, pad;
  DrawJob jobs[1];  // njobs entries
};

// Persistent compositing of a batch of images (the palette-edit renders of
// several requests): a grid of a few blocks per SM, each block claims the
// next (image, tile) item with one atomic add, composites that tile exactly
// as k_draw does, and claims again until the queue is empty.  The tiles of
// large and small images share the SMs, whatever the images' sizes.
template <int K>
__global__ void __launch_bounds__(kDrawFwdThreads, 4) k_draw_queue(DrawQueue* __restrict__ q) {
  pdl_wait();
  __shared__ float4 srec[RecordLayout<K>::kVec4 * kBatch];
  __shared__ int s_item, s_job;
  const int total = (int)q->total, njobs = (int)q->njobs;
  for (;;) {
    if (threadIdx.x == 0) {
      const int item = (int)atomicAdd(&q->next, 1u);
      int j = 0;
      while (j + 1 < njobs && (int)q->jobs[j + 1].item0 <= item) ++j;
      s_item = item;
      s_job = j;
    }
    __syncthreads();
    const int item = s_item;
    if (item >= total) break;
    const DrawJob& jb = q->jobs[s_job];
    draw_tile<K>(item - jb.item0, jb.H, jb.W, jb.gx, jb.ranges, jb.gsid, jb.records, jb.tau_init,
                 jb.out, jb.contrib, jb.final_tau, srec);
    __syncthreads();  // s_item / s_job are rewritten by the next claim
  }
}

size_t draw_queue_bytes(int max_jobs) {
  return offsetof(DrawQueue, jobs) + (size_t)(max_jobs > 0 ? max_jobs : 1) * sizeof(DrawJob);
}

// Host side: the queue image the caller copies to the device.
int draw_queue_pack(const DrawJobDesc* jobs, int njobs, void* host_table, size_t table_bytes) {
  if (draw_queue_bytes(njobs) > table_bytes) return GSB_ERR_CAPACITY;
  DrawQueue* q = (DrawQueue*)host_table;
  uint32_t item = 0;
  for (int i = 0; i < njobs; ++i) {
    const DrawJobDesc& d = jobs[i];
    const SplatState s = carve_state((void*)d.state, d.n, d.channels, d.height, d.width);
    DrawJob& j = q->jobs[i];
    j.records = s.records;
    j.ranges = (const int2*)d.ranges;
    j.gsid = d.gsid;
    j.out = d.out;
    j.contrib = d.contrib;
    j.final_tau = d.final_tau;
    j.W = d.width;
    j.H = d.height;
    j.gx = div_up(d.width, kTile);
    j.item0 = (int)item;
    j.tau_init = d.tau_init;
    j.pad[0] = j.pad[1] = j.pad[2] = 0;
    item += (uint32_t)(div_up(d.width, kTile) * div_up(d.height, kTile));
  }
  q->njobs = (uint32_t)njobs;
  q->total = item;
  q->next = 0;
  q->pad = 0;
  return GSB_OK;
}

int launch_draw_queue(int channels, const void* dev_table, int grid, cudaStream_t st) {
  DrawQueue* q = (DrawQueue*)dev_table;
  switch (channels) {
#define GSB_K(KK)                                                                          \
  case KK:                                                                                 \
    launch_pdl(k_draw_queue<KK>, dim3(grid), dim3(kDrawFwdThreads), 0, st, q);             \
    break;
    GSB_K(1) GSB_K(2) GSB_K(3) GSB_K(4) GSB_K(5) GSB_K(6) GSB_K(7) GSB_K(8)
#undef GSB_K
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
  return check_launch("draw_queue");
}

// ------------------------------------------------------------- adjoint
// Sum of NV per-lane values over groups of 2*OFF0 lanes (the whole warp for
// OFF0 = 16, each half-warp for OFF0 = 8) with NV-1 + log2(2*OFF0/NV)
// shuffles: each exchange step halves the values a lane carries (lanes with
// the step's bit set keep the upper half), so the totals end up spread over
// the group's lanes.  Returns this lane's total; *idx is the value index it
// holds and *owner is set on exactly one lane per index and group.
template <int NV, int OFF0 = 16>
__device__ __forceinline__ float warp_transpose_sum(float (&x)[NV], int lane, int* idx,
                                                    bool* owner) {
  static_assert(NV >= 1 && NV <= 2 * OFF0 && (NV & (NV - 1)) == 0,
                "NV must be a power of two no larger than the group");
  int id = 0;
  int off = OFF0;
#pragma unroll
  for (int w = NV / 2; w >= 1; w >>= 1, off >>= 1) {
    const bool hi = (lane & off) != 0;
#pragma unroll
    for (int i = 0; i < w; ++i) {
      const float send = hi ? x[i] : x[i + w];
      const float keep = hi ? x[i + w] : x[i];
      x[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
    id += hi ? w : 0;
  }
  float v = x[0];
#pragma unroll
  for (int o = off; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  *idx = id;
  *owner = off == 0 || (lane & (2 * off - 1)) == 0;  // NV == group size: every lane
  return v;
}

template <int NV>
struct Pow2 {
  static constexpr int value = NV <= 1 ? 1 : NV <= 2 ? 2 : NV <= 4 ? 4 : NV <= 8 ? 8 : NV <= 16 ? 16 : 32;
};

// Per-pixel back-to-front state of the adjoint.
template <int K>
struct BwdPixel {
  float dl[K], G[K];
  float T, Tf, dTf;
  int cont;
};

// One contributor of one pixel in the adjoint: recovers T, accumulates the
// pixel's gradient terms into x (x[0..K) features, then alpha, u, conic).
template <int K, bool GEOM, bool DTAU>
__device__ __forceinline__ bool adjoint_pixel(BwdPixel<K>& p, int idx, float m, float4 v0,
                                              float4 v1, float dx, float dy, const float4* srec,
                                              int jj, float* x) {
  if (!(idx < p.cont) || m > v1.y) return false;
  const float g = expf(-0.5f * m);
  const float ap = fminf(kAlphaMax, v1.z * g);
  if (ap < kAlphaMin) return false;
  const float one_m = 1.f - ap;
  p.T = __fdividef(p.T, one_m);
  const float wgt = ap * p.T;
#pragma unroll
  for (int k = 0; k < K; ++k) x[k] += p.dl[k] * wgt;
  if (GEOM) {
    float f[K];
    load_feats<K>(srec, jj, v1.w, f);
    float dap = 0.f;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      dap += p.dl[k] * (p.T * (f[k] - p.G[k]));
      p.G[k] = ap * f[k] + one_m * p.G[k];
    }
    if (DTAU) dap += p.dTf * __fdividef(-p.Tf, one_m);
    x[K] += dap * g;                                    // alpha
    x[K + 1] += dap * ((-v0.z * dx - v0.w * dy) * ap);  // u.x
    x[K + 2] += dap * ((-v0.w * dx - v1.x * dy) * ap);  // u.y
    x[K + 3] += dap * (-0.5f * ap * (dx * dx));         // conic a
    x[K + 4] += dap * (-1.0f * ap * (dx * dy));         // conic b
    x[K + 5] += dap * (-0.5f * ap * (dy * dy));         // conic c
  }
  return true;
}

// Weights-only adjoint of two contributors at once: slot ja lies behind slot
// jb in list order, so it is undone first.  Both records' opacity terms are
// evaluated for both pixels before either transmittance update, so the four
// exp() chains overlap; the skip tests and the T recovery are exactly those
// of adjoint_pixel.  The two gradient vectors are summed together: one
// exchange at offset 16 leaves ja's partial sums on lanes 0-15 and jb's on
// lanes 16-31, then each half-warp transposes its K values (5 + 8 shuffles
// for K = 5, against 2 x 9 for two single reductions).  When at most
// kDirectLanes lanes hit each record, those lanes add their own sums
// directly (at most 2 x kDirectLanes x K atomics instead of about 60
// reduction instructions; 47 % of the records a warp visits have so few hits
// at 1M Gaussians, 1080p).  Measured, near / far view: 4 lanes 0.367 / 0.282
// ms, 8 lanes 0.362 / 0.278, 12 lanes 0.360 / 0.275, 16 lanes 0.361 / 0.278.
constexpr int kDirectLanes = 12;
template <int K>
__device__ __forceinline__ void adjoint_weights_pair(BwdPixel<K> (&p)[2], int base, int ja, int jb,
                                                     const float4* srec, const int32_t* sgid,
                                                     float fx, float fy0, float fy1, int lane,
                                                     float* __restrict__ dfeat) {
  const float4 a0 = srec[ja], a1 = srec[kBatch + ja];
  const float4 b0 = srec[jb], b1 = srec[kBatch + jb];
  const float fy[2] = {fy0, fy1};
  float apa[2], apb[2];
  bool ua[2], ub[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const float dxa = a0.x - fx, dya = a0.y - fy[q];
    const float ma = fmaxf(0.f, maha_sq(a0.z, a0.w, a1.x, dxa, dya));
    apa[q] = fminf(kAlphaMax, a1.z * expf(-0.5f * ma));
    ua[q] = base + ja < p[q].cont && !(ma > a1.y) && !(apa[q] < kAlphaMin);
    const float dxb = b0.x - fx, dyb = b0.y - fy[q];
    const float mb = fmaxf(0.f, maha_sq(b0.z, b0.w, b1.x, dxb, dyb));
    apb[q] = fminf(kAlphaMax, b1.z * expf(-0.5f * mb));
    ub[q] = base + jb < p[q].cont && !(mb > b1.y) && !(apb[q] < kAlphaMin);
  }
  float xa[K], xb[K];
#pragma unroll
  for (int k = 0; k < K; ++k) xa[k] = xb[k] = 0.f;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    if (ua[q]) {
      p[q].T = __fdividef(p[q].T, 1.f - apa[q]);
      const float wgt = apa[q] * p[q].T;
#pragma unroll
      for (int k = 0; k < K; ++k) xa[k] += p[q].dl[k] * wgt;
    }
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    if (ub[q]) {
      p[q].T = __fdividef(p[q].T, 1.f - apb[q]);
      const float wgt = apb[q] * p[q].T;
#pragma unroll
      for (int k = 0; k < K; ++k) xb[k] += p[q].dl[k] * wgt;
    }
  }
  const bool ha = ua[0] || ua[1], hb = ub[0] || ub[1];
  const unsigned ca = __ballot_sync(0xffffffffu, ha), cb = __ballot_sync(0xffffffffu, hb);
  if (!(ca | cb)) return;
  if (__popc(ca) <= kDirectLanes && __popc(cb) <= kDirectLanes) {
    if (ha) {
      const int64_t g = sgid[ja];
#pragma unroll
      for (int k = 0; k < K; ++k) atomicAdd(dfeat + g * K + k, xa[k]);
    }
    if (hb) {
      const int64_t g = sgid[jb];
#pragma unroll
      for (int k = 0; k < K; ++k) atomicAdd(dfeat + g * K + k, xb[k]);
    }
    return;
  }
  constexpr int NV = Pow2<K>::value;
  const bool hi = (lane & 16) != 0;
  float y[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    if (k < K) {
      const float send = hi ? xa[k] : xb[k];
      const float keep = hi ? xb[k] : xa[k];
      y[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    } else {
      y[k] = 0.f;
    }
  }
  int vidx;
  bool owner;
  const float tot = warp_transpose_sum<NV, 8>(y, lane, &vidx, &owner);
  if (owner && vidx < K && (hi ? cb : ca) != 0u) {
    const int64_t g = sgid[hi ? jb : ja];
    atomicAdd(dfeat + g * K + vidx, tot);
  }
}

// Destination of gradient value `v` of Gaussian g: x[0..K) features, then
// alpha, u (2), conic (3).
template <int K>
__device__ __forceinline__ float* grad_slot(int v, int64_t g, float* dfeat, float* dalpha,
                                            float* du, float* dconic) {
  if (v < K) return dfeat + g * K + v;
  if (v == K) return dalpha + g;
  if (v < K + 3) return du + 2 * g + (v - K - 1);
  return dconic + 3 * g + (v - K - 3);
}

// Full adjoint (GEOM) of two contributors at once, slot ja behind slot jb:
// the per-pixel terms are adjoint_pixel's, in the same order (ja then jb for
// each pixel).  The two gradient vectors (K + 6 values each) are summed
// together: one exchange at lane offset 16 leaves ja's partial sums on lanes
// 0-15 and jb's on lanes 16-31, then each half-warp transposes its values
// (K + 6 + 15 shuffles for the pair instead of 2 x 16 for K = 3..8).  When
// at most kDirectLanesGeom lanes hit each record, those lanes add their own
// K + 6 sums directly: at 1M / 1080p 0.776 -> 0.755 ms near, 0.462 -> 0.439
// ms far, against direct atomics for single hits only.
constexpr int kDirectLanesGeom = 8;
template <int K, bool DTAU>
__device__ __forceinline__ void adjoint_geom_pair(BwdPixel<K> (&p)[2], int base, int ja, int jb,
                                                  const float4* srec, const int32_t* sgid,
                                                  float fx, float fy0, float fy1, int lane,
                                                  float* __restrict__ dfeat,
                                                  float* __restrict__ dalpha,
                                                  float* __restrict__ du,
                                                  float* __restrict__ dconic) {
  constexpr int NREAL = K + 6;
  constexpr int NV = Pow2<NREAL>::value;
  static_assert(NV <= 16, "half-warp transposition holds at most 16 values");
  const float4 a0 = srec[ja], a1 = srec[kBatch + ja];
  const float4 b0 = srec[jb], b1 = srec[kBatch + jb];
  float xa[NV], xb[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) xa[v] = xb[v] = 0.f;
  const float dxa = a0.x - fx, dya0 = a0.y - fy0, dya1 = a0.y - fy1;
  const float dxb = b0.x - fx, dyb0 = b0.y - fy0, dyb1 = b0.y - fy1;
  const float ma0 = fmaxf(0.f, maha_sq(a0.z, a0.w, a1.x, dxa, dya0));
  const float ma1 = fmaxf(0.f, maha_sq(a0.z, a0.w, a1.x, dxa, dya1));
  const float mb0 = fmaxf(0.f, maha_sq(b0.z, b0.w, b1.x, dxb, dyb0));
  const float mb1 = fmaxf(0.f, maha_sq(b0.z, b0.w, b1.x, dxb, dyb1));
  bool ha = adjoint_pixel<K, true, DTAU>(p[0], base + ja, ma0, a0, a1, dxa, dya0, srec, ja, xa);
  bool hb = adjoint_pixel<K, true, DTAU>(p[0], base + jb, mb0, b0, b1, dxb, dyb0, srec, jb, xb);
  ha |= adjoint_pixel<K, true, DTAU>(p[1], base + ja, ma1, a0, a1, dxa, dya1, srec, ja, xa);
  hb |= adjoint_pixel<K, true, DTAU>(p[1], base + jb, mb1, b0, b1, dxb, dyb1, srec, jb, xb);
  const unsigned ca = __ballot_sync(0xffffffffu, ha), cb = __ballot_sync(0xffffffffu, hb);
  if (!(ca | cb)) return;
  if (__popc(ca) <= kDirectLanesGeom && __popc(cb) <= kDirectLanesGeom) {
    if (ha) {
      const int64_t g = sgid[ja];
#pragma unroll
      for (int v = 0; v < NREAL; ++v) atomicAdd(grad_slot<K>(v, g, dfeat, dalpha, du, dconic), xa[v]);
    }
    if (hb) {
      const int64_t g = sgid[jb];
#pragma unroll
      for (int v = 0; v < NREAL; ++v) atomicAdd(grad_slot<K>(v, g, dfeat, dalpha, du, dconic), xb[v]);
    }
    return;
  }
  const bool hi = (lane & 16) != 0;
  float y[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    if (v < NREAL) {
      const float send = hi ? xa[v] : xb[v];
      const float keep = hi ? xb[v] : xa[v];
      y[v] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    } else {
      y[v] = 0.f;
    }
  }
  int vidx;
  bool owner;
  const float tot = warp_transpose_sum<NV, 8>(y, lane, &vidx, &owner);
  if (owner && vidx < NREAL && (hi ? cb : ca) != 0u) {
    const int64_t g = sgid[hi ? jb : ja];
    atomicAdd(grad_slot<K>(vidx, g, dfeat, dalpha, du, dconic), tot);
  }
}

// Walks each pixel's contributors back to front from its `contrib` index,
// recovering T by division by (1 - alpha') from the saved final T.  The
// per-pixel skip decisions use the forward's exact expressions, so the walk
// visits exactly the Gaussians the forward blended; T itself is recovered
// with a fast reciprocal division (relative error ~1e-7 per step).  Per
// Gaussian each lane first adds its two pixels' terms, then the warp's 64
// pixels are summed with one transposed reduction and added with one atomic
// per value.  GEOM adds the opacity / centre / conic adjoint (draw_color_B's
// terms, for any channel count); DTAU adds dL/dT_final
// (vanilla_3dgs/gsplatcu/kernel.cu:912-919).  As in the reference, the 0.99
// clamp and max(0, .) are not differentiated.  Weights-only, 8 blocks per SM
// (64 registers, a 12-byte spill): 0.377 -> 0.365 ms at 1M / 1080p against 7
// blocks (72 registers); the full adjoint 6 blocks per SM (80 registers):
// 0.755 -> 0.722 ms near, 1.146 -> 1.112 ms close, 0.437 -> 0.450 ms far.
template <int K, bool GEOM, bool DTAU>
__global__ void __launch_bounds__(kDrawThreads, GEOM ? 6 : 8)
    k_draw_backward(int H, int W, int gx, const int2* __restrict__ ranges,
                    const int32_t* __restrict__ gsid, const float4* __restrict__ records,
                    const int32_t* __restrict__ order,
                    const int32_t* __restrict__ contrib, const float* __restrict__ final_tau,
                    const float* __restrict__ dout, const float* __restrict__ dtau,
                    float* __restrict__ dfeat, float* __restrict__ dalpha,
                    float* __restrict__ du, float* __restrict__ dconic) {
  pdl_wait();
  constexpr int V = RecordLayout<K>::kVec4;
  constexpr int NREAL = GEOM ? K + 6 : K;
  constexpr int NV = Pow2<NREAL>::value;
  __shared__ float4 srec[V * kBatch];
  __shared__ int32_t sgid[kBatch];
  __shared__ unsigned s_maxc;
  const int tile = order[blockIdx.x];
  const PixelPair pp = pixels_of(tile, gx);
  const int lane = threadIdx.x & 31;
  const int2 rg = ranges[tile];
  if (rg.y - rg.x == 0) return;  // uniform per block
  const int64_t hw = (int64_t)H * W;
  BwdPixel<K> p[2];
  const int rows[2] = {pp.py0, pp.py1};
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const bool in = pp.px < W && rows[q] < H;
    const int64_t pix = (int64_t)rows[q] * W + pp.px;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      p[q].dl[k] = in ? dout[k * hw + pix] : 0.f;
      p[q].G[k] = 0.f;
    }
    p[q].Tf = in ? final_tau[pix] : 0.f;
    p[q].T = p[q].Tf;
    p[q].dTf = (DTAU && in) ? dtau[pix] : 0.f;
    p[q].cont = in ? contrib[pix] : 0;
  }
  const int wmax = (int)__reduce_max_sync(0xffffffffu, (unsigned)max(p[0].cont, p[1].cont));
  if (threadIdx.x == 0) s_maxc = 0u;
  __syncthreads();
  if (lane == 0) atomicMax(&s_maxc, (unsigned)wmax);
  __syncthreads();
  // contributor indices never exceed the tile's list (clamped for safety
  // against mismatched inputs)
  const int maxc = min((int)s_maxc, rg.y - rg.x);
  const float fx = (float)pp.px, fy0 = (float)pp.py0, fy1 = (float)pp.py1;
  for (int top = maxc; top > 0; top -= kBatch) {
    const int base = max(0, top - kBatch);
    const int cnt = top - base;
    __syncthreads();
    stage_batch<V, kDrawThreads>(gsid, rg.x + base, cnt, records, srec, sgid);
    __syncthreads();
    const int hi = min(cnt, wmax - base);
    for (int s_hi = hi; s_hi > 0; s_hi -= 32) {
      const int s_lo = max(0, s_hi - 32);
      const int j = s_lo + lane;
      bool ov = j < s_hi && box_meets_block(srec[j], srec[2 * kBatch + j], pp.wx, pp.wy, 7, 7);
      if (ov)
        ov = ellipse_meets_block(srec[j], srec[kBatch + j], srec[2 * kBatch + j], (float)pp.wx,
                                 (float)pp.wy, (float)(pp.wx + 7), (float)(pp.wy + 7));
      unsigned mask = __ballot_sync(0xffffffffu, ov);
      while (mask) {
        const int msb = 31 - __clz(mask);
        mask &= ~(1u << msb);
        if (mask) {
          const int msb2 = 31 - __clz(mask);
          mask &= ~(1u << msb2);
          if constexpr (GEOM)
            adjoint_geom_pair<K, DTAU>(p, base, s_lo + msb, s_lo + msb2, srec, sgid, fx, fy0, fy1,
                                       lane, dfeat, dalpha, du, dconic);
          else
            adjoint_weights_pair<K>(p, base, s_lo + msb, s_lo + msb2, srec, sgid, fx, fy0, fy1,
                                    lane, dfeat);
          continue;
        }
        const int jj = s_lo + msb;
        const int idx = base + jj;
        float x[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) x[v] = 0.f;
        const float4 v0 = srec[jj];
        const float4 v1 = srec[kBatch + jj];
        const float dx = v0.x - fx, dy0 = v0.y - fy0, dy1 = v0.y - fy1;
        const float m0 = fmaxf(0.f, maha_sq(v0.z, v0.w, v1.x, dx, dy0));
        const float m1 = fmaxf(0.f, maha_sq(v0.z, v0.w, v1.x, dx, dy1));
        bool hit = adjoint_pixel<K, GEOM, DTAU>(p[0], idx, m0, v0, v1, dx, dy0, srec, jj, x);
        hit |= adjoint_pixel<K, GEOM, DTAU>(p[1], idx, m1, v0, v1, dx, dy1, srec, jj, x);
        const unsigned cm = __ballot_sync(0xffffffffu, hit);
        if (!cm) continue;
        const int64_t g = sgid[jj];
        if (__popc(cm) == 1) {
          if (hit) {
#pragma unroll
            for (int k = 0; k < K; ++k) atomicAdd(dfeat + g * K + k, x[k]);
            if (GEOM) {
              atomicAdd(dalpha + g, x[K]);
              atomicAdd(du + 2 * g, x[K + 1]);
              atomicAdd(du + 2 * g + 1, x[K + 2]);
              atomicAdd(dconic + 3 * g, x[K + 3]);
              atomicAdd(dconic + 3 * g + 1, x[K + 4]);
              atomicAdd(dconic + 3 * g + 2, x[K + 5]);
            }
          }
          continue;
        }
        int vidx;
        bool owner;
        const float tot = warp_transpose_sum<NV>(x, lane, &vidx, &owner);
        if (owner && vidx < NREAL) {
          float* dst;
          if (vidx < K)
            dst = dfeat + g * K + vidx;
          else if (vidx == K)
            dst = dalpha + g;
          else if (vidx < K + 3)
            dst = du + 2 * g + (vidx - K - 1);
          else
            dst = dconic + 3 * g + (vidx - K - 3);
          atomicAdd(dst, tot);
        }
      }
    }
  }
}

// ------------------------------------------------------------ launchers
int launch_draw(int64_t n, int H, int W, int channels, const int32_t* ranges, const int32_t* gsid,
                const SplatState& s, float tau_init, float* out, int32_t* contrib,
                float* final_tau, cudaStream_t st) {
  (void)n;
  const int gx = div_up(W, kTile), gy = div_up(H, kTile);
  const int tiles = gx * gy;
  if (tiles == 0) return GSB_OK;
  const int2* rg = (const int2*)ranges;
  if (channels < 1 || channels > 8) return GSB_ERR_INVALID_ARGUMENT;
  const int rc = launch_tile_order(rg, tiles, s.tile_order, st);
  if (rc) return rc;
  switch (channels) {
#define GSB_K(KK)                                                                           \
  case KK:                                                                                  \
    launch_pdl(k_draw<KK>, dim3(tiles), dim3(kDrawFwdThreads), 0, st, H, W, gx, rg, gsid,       \
               (const float4*)s.records, (const int32_t*)s.tile_order, tau_init, out, contrib,   \
               final_tau);                                                                      \
    break;
    GSB_K(1) GSB_K(2) GSB_K(3) GSB_K(4) GSB_K(5) GSB_K(6) GSB_K(7) GSB_K(8)
#undef GSB_K
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
  return check_launch("splat_draw");
}

template <int K>
static void draw_bwd_k(int tiles, int H, int W, int gx, const int2* rg, const int32_t* gsid,
                       const float4* rec, const int32_t* order, const int32_t* contrib,
                       const float* ft, const float* dout, const float* dtau, float* dfeat,
                       float* dalpha, float* du, float* dq, cudaStream_t st) {
  const bool geom = dalpha != nullptr;
  auto kern = (geom && dtau) ? k_draw_backward<K, true, true>
              : geom         ? k_draw_backward<K, true, false>
                             : k_draw_backward<K, false, false>;
  launch_pdl(kern, dim3(tiles), dim3(kDrawThreads), 0, st, H, W, gx, rg, gsid, rec, order, contrib,
             ft, dout, dtau, dfeat, dalpha, du, dq);
}

int launch_draw_backward(int64_t n, int H, int W, int channels, const int32_t* ranges,
                         const int32_t* gsid, const SplatState& s, const int32_t* contrib,
                         const float* final_tau, const float* dout, const float* dtau,
                         float* dfeat, float* dalpha, float* du, float* dconic, cudaStream_t st) {
  (void)n;
  const int gx = div_up(W, kTile), gy = div_up(H, kTile);
  const int tiles = gx * gy;
  if (tiles == 0) return GSB_OK;
  const int2* rg = (const int2*)ranges;
  if (channels < 1 || channels > 8) return GSB_ERR_INVALID_ARGUMENT;
  const int rc = launch_tile_order(rg, tiles, s.tile_order, st);
  if (rc) return rc;
  switch (channels) {
#define GSB_K(KK)                                                                              \
  case KK:                                                                                     \
    draw_bwd_k<KK>(tiles, H, W, gx, rg, gsid, s.records, s.tile_order, contrib, final_tau,      \
                   dout, dtau, dfeat, dalpha, du, dconic, st);                                 \
    break;
    GSB_K(1) GSB_K(2) GSB_K(3) GSB_K(4) GSB_K(5) GSB_K(6) GSB_K(7) GSB_K(8)
#undef GSB_K
    default: return GSB_ERR_INVALID_ARGUMENT;
  }
  return check_launch("splat_backward");
}

}  // namespace gsb
