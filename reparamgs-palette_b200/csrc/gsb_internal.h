// Internal launcher declarations shared by the .cu files of the library.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "gsplat_b200.h"

namespace gsb {

// preprocess.cu
int launch_project(int64_t n, const float* pws, const float* Rcw, const float* tcw, float fx,
                   float fy, float cx, float cy, float* us, float* pcs, float* depths, float* du,
                   cudaStream_t st);
int launch_cov3d(int64_t n, const float* rots, const float* scales, const float* depths,
                 float* cov3ds, float* dq, float* ds, cudaStream_t st);
int launch_cov2d(int64_t n, const float* cov3ds, const float* pcs, const float* Rcw,
                 const float* depths, float fx, float fy, float tanx, float tany, float* cov2ds,
                 float* d3, float* dp, cudaStream_t st);
int launch_inverse_cov2d(int64_t n, const float* cov2ds, float* depths, float* cinv, int* areas,
                         float* dcinv, cudaStream_t st);
int launch_sh2feat(int64_t n, const void* shs, int dtype, int nb, int K, const float* pws,
                   const float* twc, float* feat, float* dshs, float* dpws, cudaStream_t st);
int launch_sh2weight_lowrank(int64_t n, const void* dc, const void* A, const void* B, int dtype,
                             int K, int P, int Q, int rank, int L, const float* pws,
                             const float* twc, float* w, float* ddc, float* ylm, cudaStream_t st);
int launch_sh2weight_lowrank_b(int64_t n, const void* A, const void* B, int dtype,
                               const float* ylm, const float* dw, int K, int P, int Q, int rank,
                               int L, float* dA, float* dB, cudaStream_t st);
int launch_lab2rgb(int H, int W, const float* lab, float* rgb, cudaStream_t st);
int lowrank_status(uint32_t* out, bool clear, cudaStream_t st);
// Device address of this file's status word (cudaGetSymbolAddress, with the
// current device and context), null on failure.
const uint32_t* lowrank_status_word();

// loss.cu
int launch_palette_l1(int K, int H, int W, const float* layer, const float* palette,
                      const float* target, float* image, float* loss, float* dlayer, float* dpal,
                      cudaStream_t st);
int launch_palette_geo_loss(int KC, int H, int W, const float* layer, const float* target,
                            const float* chroma, int clamp, int kind, float lambda_pos,
                            float* wbary, float* loss, float* dlayer, float* dchroma,
                            cudaStream_t st);

// ssim.cu
int launch_palette_l1_ssim(int K, int H, int W, const float* layer, const float* palette,
                           const float* target, float lambda_ssim, float lambda_pos,
                           float data_range, float* image, float* loss, float* dlayer,
                           float* dpal, cudaStream_t st);

// sort_static.cu -- process-unique id of the calling thread's current CUDA
// context (0 if unknown).
unsigned long long current_context_id();

// binning.cu -- clears a[0, na) and b[0, nb) (32-bit words; either may be
// null) in one kernel launched in the programmatic-dependent-launch chain.
int launch_zero2(void* a, int64_t na, void* b, int64_t nb, cudaStream_t st);

// binning.cu -- per-Gaussian binning state carved out of one caller buffer.
struct SplatState {
  float4* records;       // [n * rec_vec4]
  uint2* rects;          // [n] packed 16-bit x0 | y0 << 16, x1 | y1 << 16
  uint32_t* dkeys;       // [n] uint32(depth * 1000)
  uint32_t* counts;      // [n] patches per Gaussian
  uint32_t* block_sums;  // [n_blocks] -> exclusive block offsets after the scan
  uint32_t* stats;       // [16]: 0/3 = M low/high, 1 = max depth key
  int32_t* tile_order;   // [gx * gy] launch order of the compositing tiles
  uint32_t* part_sums;   // [n_parts] patches per kPartBlock Gaussians (fused preprocess)
  uint32_t* part_max;    // [n_parts] their largest depth key
  int rec_vec4;          // float4 vectors per record
  int64_t n_blocks, n_parts;
  int gx, gy;
};
constexpr int kBinBlock = 256;      // Gaussians per binning block
constexpr int kPartBlock = 64;      // Gaussians per fused-preprocess block (a quarter binning block)
constexpr int kRadixBits = 9;                  // digit width of one radix pass
constexpr int kRadixBins = 1 << kRadixBits;  // digits per pass
int record_vec4(int channels);
size_t splat_state_bytes(int64_t n, int channels, int H, int W);
SplatState carve_state(void* base, int64_t n, int channels, int H, int W);

int launch_pack(int64_t n, int H, int W, int channels, const float* us, const float* cinv,
                const float* alphas, const void* feats, int feat_dtype, float* depths,
                int32_t* areas, bool bin, const SplatState& s, cudaStream_t st);
// from_parts: the block sums and the largest depth key are formed from the
// fused preprocess's per-part values (nothing needs zeroing beforehand).
int launch_count_scan(int64_t n, const SplatState& s, cudaStream_t st, bool from_parts = false);

struct SortPlan {
  int tile_bits, dkey_bits, key_bits, passes;
  bool wide;  // 64-bit keys
  int64_t M, n_tiles, n_sort_blocks;
  size_t key_bytes, bytes_total;
  size_t off_keys_a, off_keys_b, off_vals_a, off_vals_b, off_hist, off_digit_tot;
};
SortPlan make_sort_plan(int64_t n, int H, int W, int64_t M, uint32_t max_dkey);
int launch_sort(const SortPlan& p, int64_t n, int H, int W, const SplatState& s, void* ws,
                int32_t* gsid_out, int32_t* ranges_out, cudaStream_t st);
// Capacity path: p.M is a patch capacity, the true count stays on the device
// (s.stats); `status` (device) receives the overflow bits.  No host sync.
int launch_patch_status(const SortPlan& p, const SplatState& s, uint32_t* status,
                        cudaStream_t st);
int launch_sort_capacity(const SortPlan& p, int64_t n, int H, int W, const SplatState& s,
                         void* ws, int32_t* gsid_out, int32_t* ranges_out, uint32_t* status,
                         cudaStream_t st);

// raster.cu
int launch_draw(int64_t n, int H, int W, int channels, const int32_t* ranges, const int32_t* gsid,
                const SplatState& s, float tau_init, float* out, int32_t* contrib,
                float* final_tau, cudaStream_t st);
// Batched compositing (raster.cu): one image of a batch as the host
// describes it (gsb_draw_job of the C ABI).
using DrawJobDesc = gsb_draw_job;
size_t draw_queue_bytes(int max_jobs);
int draw_queue_pack(const DrawJobDesc* jobs, int njobs, void* host_table, size_t table_bytes);
int launch_draw_queue(int channels, const void* dev_table, int grid, cudaStream_t st);
int launch_draw_backward(int64_t n, int H, int W, int channels, const int32_t* ranges,
                         const int32_t* gsid, const SplatState& s, const int32_t* contrib,
                         const float* final_tau, const float* dout, const float* dtau,
                         float* dfeat, float* dalpha, float* du, float* dconic, cudaStream_t st);


// fused.cu -- per-Gaussian preprocess and its adjoint in one kernel each.
struct CamArgs {
  const float* R;  // device [3,3] Rcw
  const float* t;  // device [3] tcw
  const float* c;  // device [3] twc
  float fx, fy, cx, cy, tanx, tany;
};
struct FusedArgs {
  int64_t n;
  uint32_t gx, gy;
  CamArgs cam;
  const float *pws, *rots, *scales, *alphas;
  const void *w0, *wa, *wb;  // shs or dc; A; B (storage dtype)
  SplatState st;             // forward: filled like gsb_splat_pack + count
  float* depths_out;         // forward, may be null
  const float* palette;      // forward, may be null: [K,3] -> colour records
  const float *g_feat, *g_u, *g_conic;  // backward: screen-space gradients (g_u null: weights only)
  float *d_pws, *d_rots, *d_scales, *d_w0, *d_wa, *d_wb;
  bool accumulate;  // backward: add to the d_* outputs instead of overwriting them
};
int launch_render(int mode, int dtype, int K, int P, int Q, int R, const FusedArgs& f, bool backward,
                  cudaStream_t st);
int fused_status(uint32_t* out, bool clear, cudaStream_t st);
const uint32_t* fused_status_word();
int expire_bulk_wait(uint32_t poll_limit, cudaStream_t st);

}  // namespace gsb
