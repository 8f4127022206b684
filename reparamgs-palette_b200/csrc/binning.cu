// Tile binning: per-Gaussian rectangles and patch counts, packed compositing
// records, patch-count scan, key emission, an LSD radix sort over only the
// key bits in use, and per-tile ranges.
//
// Ordering contract (gsplatcu/kernel.cu:96-187, gsplatcu/gausplat.cu:185-226):
// patches are emitted Gaussian by Gaussian (tiles of one Gaussian row-major)
// and sorted STABLY by (tile, uint32(depth*1000)), so each tile's list is
// ordered by quantised depth, then Gaussian id -- the same total order the
// reference's stable 64-bit thrust::sort_by_key produces.  Keys here hold
// only ceil(log2 T) tile bits above the depth-key bits actually used, so the
// sort runs ceil(bits/8) passes instead of eight.
#include <algorithm>

#include "gsb_geometry.cuh"
#include "gsb_internal.h"
#include "gsb_record.cuh"

namespace gsb {

// ----------------------------------------------------------------- state
int record_vec4(int channels) { return ((11 + channels) + 3) / 4; }

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Layout: channel-independent arrays first (so that callers that do not know
// the channel count can locate them), packed records last.
static void state_layout(int64_t n, int channels, int H, int W, size_t* offs) {
  const int64_t nb = (n + kBinBlock - 1) / kBinBlock;
  const int64_t gx = div_up(W, kTile), gy = div_up(H, kTile);
  size_t b = 0;
  offs[0] = b; b += align256((size_t)n * 8);                          // rects
  offs[1] = b; b += align256((size_t)n * 4);                          // dkeys
  offs[2] = b; b += align256((size_t)n * 4);                          // counts
  offs[3] = b; b += align256((size_t)(nb > 0 ? nb : 1) * 4);          // block sums
  offs[4] = b; b += align256(16 * 4);                                 // stats
  offs[5] = b; b += align256((size_t)(gx * gy > 0 ? gx * gy : 1) * 4); // tile launch order
  offs[6] = b; b += align256((size_t)n * record_vec4(channels) * 16); // records
  const int64_t np = (n + kPartBlock - 1) / kPartBlock;
  offs[7] = b; b += 2 * align256((size_t)(np > 0 ? np : 1) * 4);      // part sums, part max
  offs[8] = b;
}

size_t splat_state_bytes(int64_t n, int channels, int H, int W) {
  size_t offs[9];
  state_layout(n, channels, H, W, offs);
  return offs[8];
}

SplatState carve_state(void* base, int64_t n, int channels, int H, int W) {
  size_t o[9];
  state_layout(n, channels, H, W, o);
  char* p = (char*)base;
  SplatState s;
  s.rec_vec4 = record_vec4(channels);
  s.n_blocks = (n + kBinBlock - 1) / kBinBlock;
  s.gx = div_up(W, kTile);
  s.gy = div_up(H, kTile);
  s.rects = (uint2*)(p + o[0]);
  s.dkeys = (uint32_t*)(p + o[1]);
  s.counts = (uint32_t*)(p + o[2]);
  s.block_sums = (uint32_t*)(p + o[3]);
  s.stats = (uint32_t*)(p + o[4]);
  s.tile_order = (int32_t*)(p + o[5]);
  s.records = (float4*)(p + o[6]);
  s.n_parts = (n + kPartBlock - 1) / kPartBlock;
  s.part_sums = (uint32_t*)(p + o[7]);
  s.part_max = s.part_sums + align256((size_t)(s.n_parts > 0 ? s.n_parts : 1) * 4) / 4;
  return s;
}

// --------------------------------------------------------- block helpers
// Exclusive scan of one value per thread over a 256-thread block.
__device__ __forceinline__ uint32_t block_excl_scan256(uint32_t v, uint32_t* warp_tot,
                                                       uint32_t* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  uint32_t base = 0, tot = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t t = warp_tot[k];
    base += (k < w) ? t : 0u;
    tot += t;
  }
  __syncthreads();
  if (total) *total = tot;
  return base + incl - v;
}

// ------------------------------------------------------------------ zero
// Clears up to two word arrays in one launch.  A kernel rather than memset
// nodes, so that it joins the programmatic-dependent-launch chain of the
// kernels around it.
__global__ void k_zero2(uint32_t* __restrict__ a, int64_t na, uint32_t* __restrict__ b,
                        int64_t nb) {
  pdl_wait();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na + nb; i += stride) {
    if (i < na)
      a[i] = 0u;
    else
      b[i - na] = 0u;
  }
}

int launch_zero2(void* a, int64_t na, void* b, int64_t nb, cudaStream_t st) {
  if (!a) na = 0;
  if (!b) nb = 0;
  if (na + nb == 0) return GSB_OK;
  const int64_t blocks = std::min<int64_t>((na + nb + 255) / 256, 148 * 8);
  launch_pdl(k_zero2, dim3((unsigned)blocks), dim3(256), 0, st, (uint32_t*)a, na, (uint32_t*)b,
             nb);
  return check_launch("zero");
}

// ------------------------------------------------------------------ pack
// One thread per Gaussian: tile rectangle and patch count (getRects,
// gsplatcu/kernel.cu:127-162, including its in-place depth/areas updates),
// the quantised depth key, and the packed compositing record (gsb_record.cuh).
template <typename T>
__global__ void __launch_bounds__(kBinBlock)
    k_pack(int64_t n, uint32_t gx, uint32_t gy, int C, int V, const float* __restrict__ us,
           const float* __restrict__ cinv, const float* __restrict__ alphas,
           const T* __restrict__ feats, float* __restrict__ depths, int32_t* __restrict__ areas,
           bool bin, float4* __restrict__ records, uint2* __restrict__ rects,
           uint32_t* __restrict__ dkeys, uint32_t* __restrict__ counts,
           uint32_t* __restrict__ block_sums, uint32_t* __restrict__ stats) {
  pdl_wait();
  __shared__ uint32_t warp_tot[8], warp_max[kBinBlock / 32];
  const int64_t i = (int64_t)blockIdx.x * kBinBlock + threadIdx.x;
  uint32_t cnt = 0, dk = 0;
  if (i < n) {
    const float ux = us[2 * i], uy = us[2 * i + 1];
    if (bin) {
      const float depth = depths[i];
      if (!(depth < kMinDepth)) {
        const float xs = (float)areas[2 * i], ys = (float)areas[2 * i + 1];
        const TileRect r = tile_rect(ux, uy, xs, ys, gx, gy);
        cnt = (r.y1 - r.y0) * (r.x1 - r.x0);
        if (cnt == 0) {
          depths[i] = kBadDepth;
          areas[2 * i] = 0;
          areas[2 * i + 1] = 0;
        } else {
          rects[i] = make_uint2(r.x0 | (r.y0 << 16), r.x1 | (r.y1 << 16));
          dk = __float2uint_rz(depth * 1000);
        }
      }
      counts[i] = cnt;
      dkeys[i] = dk;
    }
    const float qa = cinv[3 * i], qb = cinv[3 * i + 1], qc = cinv[3 * i + 2];
    const float a = alphas[i];
    float f[4 * 5];
    record_head(ux, uy, qa, qb, qc, a, f);
    float4* rec = records + i * V;
#pragma unroll
    for (int k = 0; k < kMaxChannels; ++k)
      if (k < C) f[record_channel(k)] = ld(feats, i * C + k);
#pragma unroll
    for (int v = 0; v < 5; ++v)
      if (v < V) rec[v] = make_float4(f[4 * v], f[4 * v + 1], f[4 * v + 2], f[4 * v + 3]);
  }
  if (!bin) return;
  // block max of the depth keys of binned Gaussians: warp maxima, folded by
  // thread 0 after the scan's barriers, one atomic per block (one per warp
  // would queue ~n/32 atomics on the same word)
  uint32_t m = dk;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = m;
  uint32_t tot;
  block_excl_scan256(cnt, warp_tot, &tot);
  if (threadIdx.x == 0) {
    uint32_t bm = 0;
#pragma unroll
    for (int k = 0; k < kBinBlock / 32; ++k) bm = max(bm, warp_max[k]);
    if (bm) atomicMax(stats + 1, bm);
    block_sums[blockIdx.x] = tot;
  }
}

// Single-block exclusive scan of the per-block patch counts; writes the
// total M (low/high words) into stats[0] / stats[3].  With `psum` (the fused
// preprocess) each block's count is first summed from its kBinBlock /
// kPartBlock parts, and stats[1] (largest depth key) and the other stats
// words are written here too, so that nothing needs zeroing beforehand.
__global__ void __launch_bounds__(1024) k_scan_block_sums(uint32_t* __restrict__ sums, int64_t nb,
                                                          uint32_t* __restrict__ stats,
                                                          const uint32_t* __restrict__ psum,
                                                          const uint32_t* __restrict__ pmax,
                                                          int64_t nparts) {
  pdl_wait();
  constexpr int kPer = kBinBlock / kPartBlock;
  __shared__ uint32_t warp_tot[32];
  __shared__ unsigned long long carry;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0ull;
  if (psum) {
    uint32_t m = 0;
    for (int64_t j = threadIdx.x; j < nparts; j += 1024) m = max(m, pmax[j]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) warp_tot[w] = m;
    __syncthreads();
    if (threadIdx.x < 16) {
      uint32_t mm = 0;
      if (threadIdx.x == 1)
        for (int k = 0; k < 32; ++k) mm = max(mm, warp_tot[k]);
      if (threadIdx.x != 0 && threadIdx.x != 3) stats[threadIdx.x] = mm;  // 1: max; rest 0
    }
  }
  __syncthreads();
  for (int64_t base = 0; base < nb; base += 1024 * 4) {
    uint32_t v[4], s = 0;
    const int64_t j0 = base + (int64_t)threadIdx.x * 4;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (psum) {
        uint32_t t = 0;
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
          const int64_t pj = (j0 + k) * kPer + q;
          t += pj < nparts ? psum[pj] : 0u;
        }
        v[k] = (j0 + k < nb) ? t : 0u;
      } else {
        v[k] = (j0 + k < nb) ? sums[j0 + k] : 0u;
      }
      s += v[k];
    }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    uint32_t wbase = 0, btot = 0;
    for (int k = 0; k < 32; ++k) {
      const uint32_t t = warp_tot[k];
      wbase += (k < w) ? t : 0u;
      btot += t;
    }
    uint32_t run = (uint32_t)carry + wbase + incl - s;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (j0 + k < nb) sums[j0 + k] = run;
      run += v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += btot;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    stats[0] = (uint32_t)carry;
    stats[3] = (uint32_t)(carry >> 32);
  }
}

// Tile index of a sort key (the depth key occupies the low `dkey_bits`).
template <typename KT>
__device__ __forceinline__ uint32_t key_tile(KT k, int dkey_bits) {
  return dkey_bits >= (int)(8 * sizeof(KT)) ? 0u : (uint32_t)(k >> dkey_bits);
}
template <typename KT>
__device__ __forceinline__ KT make_key(uint32_t tile, uint32_t dk, int dkey_bits) {
  return dkey_bits >= (int)(8 * sizeof(KT)) ? (KT)dk : (((KT)tile << dkey_bits) | (KT)dk);
}

// Patch count the sort kernels work on.  `mdev` null: the host-known count
// M.  Otherwise (capacity path, no host read-back) M is a capacity and the
// true count is the device total in mdev (stats words 0 and 3); a count
// above the capacity, or a depth key wider than `dkey_bits`, is an overflow:
// the kernels then stay inside the capacity and k_ranges leaves every range
// empty, so nothing downstream reads the unsorted entries.
__device__ __forceinline__ int64_t device_patches(int64_t M, const uint32_t* mdev) {
  if (!mdev) return M;
  const uint64_t m = (uint64_t)mdev[0] | ((uint64_t)mdev[3] << 32);
  return m > (uint64_t)M ? M : (int64_t)m;
}
__device__ __forceinline__ bool capacity_overflow(int64_t M, const uint32_t* mdev, int dkey_bits) {
  if (!mdev) return false;
  const uint64_t m = (uint64_t)mdev[0] | ((uint64_t)mdev[3] << 32);
  return m > (uint64_t)M || (dkey_bits < 32 && (mdev[1] >> dkey_bits) != 0u);
}

// ------------------------------------------------------------------ emit
// Key emission (createKeys, gsplatcu/kernel.cu:96-124) done cooperatively by
// each warp: the warp's 32 Gaussians own one contiguous run of patch slots,
// and the lanes fill it slot by slot (coalesced), each slot locating its
// Gaussian by binary search over the warp's inclusive counts.
template <typename KT>
__global__ void __launch_bounds__(kBinBlock)
    k_emit(int64_t n, uint32_t gx, int dkey_bits, const uint2* __restrict__ rects,
           const uint32_t* __restrict__ dkeys, const uint32_t* __restrict__ counts,
           const uint32_t* __restrict__ block_offs, KT* __restrict__ keys,
           int32_t* __restrict__ vals, int64_t cap, int2* __restrict__ ranges,
           int64_t n_tiles) {
  pdl_wait();
  // the ranges start empty (getRanges writes only tiles that have patches);
  // cleared here, long before k_ranges writes them
  for (int64_t t = (int64_t)blockIdx.x * kBinBlock + threadIdx.x; t < n_tiles;
       t += (int64_t)gridDim.x * kBinBlock)
    ranges[t] = make_int2(0, 0);
  __shared__ uint32_t warp_tot[8];
  __shared__ uint32_t s_incl[8][32];
  __shared__ uint2 s_rect[8][32];
  __shared__ uint32_t s_dk[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t i = (int64_t)blockIdx.x * kBinBlock + threadIdx.x;
  const uint32_t c = (i < n) ? counts[i] : 0u;
  const uint32_t excl = block_excl_scan256(c, warp_tot, nullptr);
  // inclusive count within the warp
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const uint32_t warp_total = __shfl_sync(0xffffffffu, incl, 31);
  const uint32_t warp_start = block_offs[blockIdx.x] + __shfl_sync(0xffffffffu, excl, 0);
  s_incl[w][lane] = incl;
  s_rect[w][lane] = (c > 0) ? rects[i] : make_uint2(0u, 0u);
  s_dk[w][lane] = (c > 0) ? dkeys[i] : 0u;
  __syncwarp();
  const int64_t first = (int64_t)blockIdx.x * kBinBlock + w * 32;
  for (uint32_t p = lane; p < warp_total; p += 32) {
    int L = 0;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1)
      if (s_incl[w][L + s - 1] <= p) L += s;
    const uint32_t local = p - (L ? s_incl[w][L - 1] : 0u);
    const uint2 r = s_rect[w][L];
    const uint32_t x0 = r.x & 0xffffu, y0 = r.x >> 16, x1 = r.y & 0xffffu;
    const uint32_t wdt = x1 - x0;
    const uint32_t ty = local / wdt, tx = local - ty * wdt;
    const uint32_t tile = (y0 + ty) * gx + (x0 + tx);
    const uint32_t slot = warp_start + p;
    if ((int64_t)slot >= cap) break;  // capacity path overflow (flagged elsewhere)
    keys[slot] = make_key<KT>(tile, s_dk[w][L], dkey_bits);
    vals[slot] = (int32_t)(first + L);
  }
}

// ------------------------------------------------------------ radix sort
constexpr int kSortThreads = 256;
constexpr int kSortItems = 12;  // measured: 8 -> 12 keys per thread, 7 % less sort time
constexpr int kSortTile = kSortThreads * kSortItems;  // keys per block

template <typename KT>
__global__ void __launch_bounds__(kSortThreads)
    k_radix_upsweep(const KT* __restrict__ keys, int64_t M, int shift, uint32_t mask,
                    uint32_t* __restrict__ hist, int64_t nblocks, const uint32_t* __restrict__ mdev) {
  pdl_wait();
  __shared__ uint32_t h[8][kRadixBins];
  M = device_patches(M, mdev);
  const int w = threadIdx.x >> 5;
  for (int k = threadIdx.x; k < 8 * kRadixBins; k += kSortThreads) (&h[0][0])[k] = 0u;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kSortTile;
  // all of the thread's keys in flight before the histogram updates
  KT k[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int64_t idx = base + r * kSortThreads + threadIdx.x;
    k[r] = idx < M ? keys[idx] : (KT)0;
  }
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int64_t idx = base + r * kSortThreads + threadIdx.x;
    if (idx < M) atomicAdd(&h[w][(uint32_t)(k[r] >> shift) & mask], 1u);
  }
  __syncthreads();
  for (uint32_t d = threadIdx.x; d <= mask; d += kSortThreads) {
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += h[k][d];
    hist[(int64_t)d * nblocks + blockIdx.x] = s;
  }
}

// One block per digit: exclusive scan of that digit's per-block counts.
__global__ void __launch_bounds__(256)
    k_radix_scan(uint32_t* __restrict__ hist, int64_t nblocks, uint32_t* __restrict__ digit_tot) {
  pdl_wait();
  __shared__ uint32_t warp_tot[8];
  uint32_t* row = hist + (int64_t)blockIdx.x * nblocks;
  uint32_t carry = 0;
  constexpr int kItems = 8;  // consecutive counts per thread: one block scan per 2048
  for (int64_t base = 0; base < nblocks; base += 256 * kItems) {
    const int64_t j0 = base + (int64_t)threadIdx.x * kItems;
    uint32_t v[kItems], s = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      v[i] = j0 + i < nblocks ? row[j0 + i] : 0u;
      s += v[i];
    }
    uint32_t tot;
    uint32_t run = carry + block_excl_scan256(s, warp_tot, &tot);
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      if (j0 + i < nblocks) row[j0 + i] = run;
      run += v[i];
    }
    carry += tot;
  }
  if (threadIdx.x == 0) digit_tot[blockIdx.x] = carry;
}

// Stable scatter of one digit pass.  Items of a block are ranked in their
// original order (warp w owns items [32 kSortItems w, 32 kSortItems (w+1)),
// lane-minor), staged in
// shared memory in digit order and written out in digit-contiguous runs.
// Thread t owns digits 2t and 2t+1 in the per-digit phases.
template <typename KT>
__global__ void __launch_bounds__(kSortThreads)
    k_radix_downsweep(const KT* __restrict__ kin, const int32_t* __restrict__ vin,
                      KT* __restrict__ kout, int32_t* __restrict__ vout, int64_t M, int shift,
                      uint32_t mask, const uint32_t* __restrict__ hist,
                      const uint32_t* __restrict__ digit_tot, int64_t nblocks,
                      const uint32_t* __restrict__ mdev) {
  pdl_wait();
  static_assert(kRadixBins == 2 * kSortThreads, "two digits per thread");
  M = device_patches(M, mdev);
  if ((int64_t)blockIdx.x * kSortTile >= M) return;  // whole block past the patches
  extern __shared__ __align__(16) unsigned char smem_raw[];
  KT* sk = (KT*)smem_raw;
  int32_t* sv = (int32_t*)(sk + kSortTile);
  uint32_t* wcnt = (uint32_t*)(sv + kSortTile);  // [8][kRadixBins]
  uint32_t* lstart = wcnt + 8 * kRadixBins;      // [kRadixBins]
  uint32_t* gstart = lstart + kRadixBins;        // [kRadixBins]
  uint32_t* warp_tot = gstart + kRadixBins;      // [8]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = threadIdx.x; k < 8 * kRadixBins; k += kSortThreads) wcnt[k] = 0u;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kSortTile + w * (32 * kSortItems);
  KT key[kSortItems];
  int32_t val[kSortItems];
  uint32_t rnk[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int64_t idx = base + r * 32 + lane;
    const bool ok = idx < M;
    key[r] = ok ? kin[idx] : (KT)0;
    val[r] = ok ? vin[idx] : 0;
  }
  const uint32_t lt = (1u << lane) - 1u;
  const int nbits = 32 - __clz(mask);  // digit bits of this pass
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const bool ok = base + r * 32 + lane < M;
    const uint32_t d = ok ? ((uint32_t)(key[r] >> shift) & mask) : 0xffffu;
    // lanes with the same digit: one ballot per digit bit of this pass
    // (faster than __match_any_sync here: 0.181 -> 0.164 ms per sort of
    // 3.5M keys)
    uint32_t peers = __ballot_sync(0xffffffffu, ok);
    if (!ok) peers = ~peers;
    for (int b = 0; b < nbits; ++b) {
      const bool bit = (d >> b) & 1u;
      const uint32_t bm = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? bm : ~bm;
    }
    const uint32_t before = ok ? wcnt[w * kRadixBins + d] : 0u;
    rnk[r] = before + __popc(peers & lt);
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) wcnt[w * kRadixBins + d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per digit: exclusive offsets across warps, block-local start, global start
  const uint32_t d0 = 2 * threadIdx.x, d1 = d0 + 1;
  uint32_t tot0 = 0, tot1 = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t c0 = wcnt[k * kRadixBins + d0], c1 = wcnt[k * kRadixBins + d1];
    wcnt[k * kRadixBins + d0] = tot0;
    wcnt[k * kRadixBins + d1] = tot1;
    tot0 += c0;
    tot1 += c1;
  }
  const uint32_t dt0 = d0 <= mask ? digit_tot[d0] : 0u, dt1 = d1 <= mask ? digit_tot[d1] : 0u;
  const uint32_t ls = block_excl_scan256(tot0 + tot1, warp_tot, nullptr);
  const uint32_t gd = block_excl_scan256(dt0 + dt1, warp_tot, nullptr);
  lstart[d0] = ls;
  lstart[d1] = ls + tot0;
  gstart[d0] = gd + (d0 <= mask ? hist[(int64_t)d0 * nblocks + blockIdx.x] : 0u);
  gstart[d1] = gd + dt0 + (d1 <= mask ? hist[(int64_t)d1 * nblocks + blockIdx.x] : 0u);
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    if (base + r * 32 + lane < M) {
      const uint32_t dd = (uint32_t)(key[r] >> shift) & mask;
      const uint32_t pos = lstart[dd] + wcnt[w * kRadixBins + dd] + rnk[r];
      sk[pos] = key[r];
      sv[pos] = val[r];
    }
  }
  __syncthreads();
  const int64_t rem = M - (int64_t)blockIdx.x * kSortTile;
  const int cnt = rem < kSortTile ? (int)rem : kSortTile;
  for (int j = threadIdx.x; j < cnt; j += kSortThreads) {
    const KT k = sk[j];
    const uint32_t dd = (uint32_t)(k >> shift) & mask;
    const uint32_t g = gstart[dd] + (uint32_t)j - lstart[dd];
    kout[g] = k;
    vout[g] = sv[j];
  }
}

// getRanges (gsplatcu/kernel.cu:165-187) on the sorted keys, with the same
// writes -- including that the end of the only tile is left unset when
// M == 1.  `ranges` is cleared beforehand.
constexpr int kRangeItems = 8;  // keys per thread in k_ranges

template <typename KT>
__global__ void k_ranges(const KT* __restrict__ keys, int64_t M, int dkey_bits,
                         int2* __restrict__ ranges, const uint32_t* __restrict__ mdev) {
  pdl_wait();
  if (capacity_overflow(M, mdev, dkey_bits)) return;
  M = device_patches(M, mdev);
  const int64_t b0 = (int64_t)blockIdx.x * (256 * kRangeItems) + threadIdx.x;
  uint32_t cur[kRangeItems], prv[kRangeItems];
#pragma unroll
  for (int r = 0; r < kRangeItems; ++r) {
    const int64_t p = b0 + r * 256;
    cur[r] = p < M ? key_tile(keys[p], dkey_bits) : 0u;
    prv[r] = p < M ? key_tile(keys[p == 0 ? 0 : p - 1], dkey_bits) : 0u;
  }
#pragma unroll
  for (int r = 0; r < kRangeItems; ++r) {
    const int64_t p = b0 + r * 256;
    if (p >= M) continue;
    if (p == 0)
      ranges[cur[r]].x = 0;
    else if (p == M - 1)
      ranges[cur[r]].y = (int)M;
    if (prv[r] != cur[r]) {
      ranges[prv[r]].y = (int)p;
      ranges[cur[r]].x = (int)p;
    }
  }
}

// Overflow status of a capacity-path sort (bits GSB_STATUS_PATCH_OVERFLOW,
// GSB_STATUS_DEPTH_KEY_OVERFLOW), written for the caller to read later.
__global__ void k_capacity_status(int64_t cap, int dkey_bits, const uint32_t* __restrict__ stats,
                                  uint32_t* __restrict__ status) {
  pdl_wait();
  const uint64_t m = (uint64_t)stats[0] | ((uint64_t)stats[3] << 32);
  uint32_t v = 0;
  if (m > (uint64_t)cap) v |= GSB_STATUS_PATCH_OVERFLOW;
  if (dkey_bits < 32 && (stats[1] >> dkey_bits) != 0u) v |= GSB_STATUS_DEPTH_KEY_OVERFLOW;
  status[0] = v;
  status[1] = stats[0];  // the patch count, low and high words
  status[2] = stats[3];
}

// ------------------------------------------------------------ launchers
template <typename T>
static void pack_t(int64_t n, uint32_t gx, uint32_t gy, int C, const float* us, const float* cinv,
                   const float* alphas, const void* feats, float* depths, int32_t* areas, bool bin,
                   const SplatState& s, cudaStream_t st) {
  launch_pdl(k_pack<T>, dim3((unsigned)s.n_blocks), dim3(kBinBlock), 0, st, n, gx, gy, C,
             s.rec_vec4, us, cinv, alphas, (const T*)feats, depths, areas, bin, s.records, s.rects,
             s.dkeys, s.counts, s.block_sums, s.stats);
}

int launch_pack(int64_t n, int H, int W, int channels, const float* us, const float* cinv,
                const float* alphas, const void* feats, int feat_dtype, float* depths,
                int32_t* areas, bool bin, const SplatState& s, cudaStream_t st) {
  if (bin) {
    const int rc = launch_zero2(s.stats, 16, nullptr, 0, st);
    if (rc) return rc;
  }
  if (n == 0) return GSB_OK;
  const uint32_t gx = (uint32_t)div_up(W, kTile), gy = (uint32_t)div_up(H, kTile);
  if (feat_dtype == GSB_DTYPE_BF16)
    pack_t<__nv_bfloat16>(n, gx, gy, channels, us, cinv, alphas, feats, depths, areas, bin, s, st);
  else
    pack_t<float>(n, gx, gy, channels, us, cinv, alphas, feats, depths, areas, bin, s, st);
  return check_launch("splat_pack");
}

int launch_count_scan(int64_t n, const SplatState& s, cudaStream_t st, bool from_parts) {
  if (n == 0) return from_parts ? launch_zero2(s.stats, 16, nullptr, 0, st) : GSB_OK;
  launch_pdl(k_scan_block_sums, dim3(1), dim3(1024), 0, st, s.block_sums, s.n_blocks, s.stats,
             from_parts ? (const uint32_t*)s.part_sums : nullptr,
             from_parts ? (const uint32_t*)s.part_max : nullptr, s.n_parts);
  return check_launch("splat_scan");
}

static int bit_length(uint64_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

// Radix passes of at most kRadixBits bits each over the key bits in use.
SortPlan make_sort_plan(int64_t n, int H, int W, int64_t M, uint32_t max_dkey) {
  SortPlan p;
  const int64_t gx = div_up(W, kTile), gy = div_up(H, kTile);
  p.n_tiles = gx * gy;
  p.M = M;
  p.tile_bits = bit_length((uint64_t)(p.n_tiles - 1));
  p.dkey_bits = bit_length(max_dkey);
  p.key_bits = p.tile_bits + p.dkey_bits;
  p.wide = p.key_bits > 32;
  p.passes = (p.key_bits + kRadixBits - 1) / kRadixBits;
  p.n_sort_blocks = (M + kSortTile - 1) / kSortTile;
  p.key_bytes = p.wide ? 8 : 4;
  size_t off = 0;
  p.off_keys_a = off;
  off += align256((size_t)M * p.key_bytes);
  p.off_keys_b = off;
  off += align256((size_t)M * p.key_bytes);
  p.off_vals_a = off;
  off += align256((size_t)M * 4);
  p.off_vals_b = off;
  off += align256((size_t)M * 4);
  p.off_hist = off;
  off += align256((size_t)kRadixBins * (p.n_sort_blocks > 0 ? p.n_sort_blocks : 1) * 4);
  p.off_digit_tot = off;
  off += align256(kRadixBins * 4);
  p.bytes_total = off;
  (void)n;
  return p;
}

template <typename KT>
static int sort_t(const SortPlan& p, int64_t n, int W, const SplatState& s, void* ws,
                  int32_t* gsid_out, int32_t* ranges_out, const uint32_t* mdev,
                  cudaStream_t st) {
  char* b = (char*)ws;
  KT* ka = (KT*)(b + p.off_keys_a);
  KT* kb = (KT*)(b + p.off_keys_b);
  int32_t* va = (int32_t*)(b + p.off_vals_a);
  int32_t* vb = (int32_t*)(b + p.off_vals_b);
  uint32_t* hist = (uint32_t*)(b + p.off_hist);
  uint32_t* dtot = (uint32_t*)(b + p.off_digit_tot);
  const uint32_t gx = (uint32_t)div_up(W, kTile);
  launch_pdl(k_emit<KT>, dim3((unsigned)s.n_blocks), dim3(kBinBlock), 0, st, n, gx, p.dkey_bits,
             s.rects, s.dkeys, s.counts, s.block_sums, ka, p.passes == 0 ? gsid_out : va, p.M,
             (int2*)ranges_out, p.n_tiles);
  int rc = check_launch("splat_sort (emit)");
  if (rc) return rc;
  const size_t smem =
      (size_t)kSortTile * (sizeof(KT) + 4) + (8 * kRadixBins + 2 * kRadixBins + 8) * 4;
  if (cudaFuncSetAttribute(k_radix_downsweep<KT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return check_launch("splat_sort (smem attribute)", 0);
  KT* ks = ka;
  KT* kd = kb;
  int32_t* vs = va;
  int32_t* vd = vb;
  const int nbk = (int)p.n_sort_blocks;
  for (int pass = 0; pass < p.passes; ++pass) {
    const int shift = kRadixBits * pass;
    const int bits = (p.key_bits - shift) < kRadixBits ? (p.key_bits - shift) : kRadixBits;
    const uint32_t mask = (1u << bits) - 1u;
    int32_t* vdst = (pass == p.passes - 1) ? gsid_out : vd;
    launch_pdl(k_radix_upsweep<KT>, dim3(nbk), dim3(kSortThreads), 0, st, (const KT*)ks, p.M,
               shift, mask, hist, p.n_sort_blocks, mdev);
    launch_pdl(k_radix_scan, dim3(mask + 1), dim3(256), 0, st, hist, p.n_sort_blocks, dtot);
    launch_pdl(k_radix_downsweep<KT>, dim3(nbk), dim3(kSortThreads), smem, st, (const KT*)ks,
               (const int32_t*)vs, kd, vdst, p.M, shift, mask, (const uint32_t*)hist,
               (const uint32_t*)dtot, p.n_sort_blocks, mdev);
    rc = check_launch("splat_sort (radix pass)", 3);
    if (rc) return rc;
    KT* kt = ks;
    ks = kd;
    kd = kt;
    int32_t* vt = vs;
    vs = vd;
    vd = vt;
  }
  launch_pdl(k_ranges<KT>, dim3((unsigned)div_up(p.M, 256 * kRangeItems)), dim3(256), 0, st,
             (const KT*)ks, p.M,
             p.dkey_bits, (int2*)ranges_out, mdev);
  return check_launch("splat_sort (ranges)");
}

int launch_sort(const SortPlan& p, int64_t n, int H, int W, const SplatState& s, void* ws,
                int32_t* gsid_out, int32_t* ranges_out, cudaStream_t st) {
  (void)H;
  if (p.M == 0)  // no emission to clear the ranges
    return launch_zero2(ranges_out, p.n_tiles * 2, nullptr, 0, st);
  return p.wide ? sort_t<uint64_t>(p, n, W, s, ws, gsid_out, ranges_out, nullptr, st)
                : sort_t<uint32_t>(p, n, W, s, ws, gsid_out, ranges_out, nullptr, st);
}

int launch_patch_status(const SortPlan& p, const SplatState& s, uint32_t* status,
                        cudaStream_t st) {
  launch_pdl(k_capacity_status, dim3(1), dim3(1), 0, st, p.M, p.dkey_bits,
             (const uint32_t*)s.stats, status);
  return check_launch("splat_patch_status");
}

int launch_sort_capacity(const SortPlan& p, int64_t n, int H, int W, const SplatState& s,
                         void* ws, int32_t* gsid_out, int32_t* ranges_out, uint32_t* status,
                         cudaStream_t st) {
  (void)H;
  if (status) {  // (callers that read the status through gsb_splat_patch_status pass null)
    launch_pdl(k_capacity_status, dim3(1), dim3(1), 0, st, p.M, p.dkey_bits,
               (const uint32_t*)s.stats, status);
    const int rc = check_launch("splat_sort_capacity (status)");
    if (rc) return rc;
  }
  if (p.M == 0 || n == 0) return launch_zero2(ranges_out, p.n_tiles * 2, nullptr, 0, st);
  return p.wide ? sort_t<uint64_t>(p, n, W, s, ws, gsid_out, ranges_out, s.stats, st)
                : sort_t<uint32_t>(p, n, W, s, ws, gsid_out, ranges_out, s.stats, st);
}

}  // namespace gsb
