/*
 * gsplat_b200.h -- C ABI of the B200 (sm_100a) palette-weight Gaussian
 * rasterizer.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (cudaStream_t passed as void*; NULL is the legacy default stream), enqueues
 * its kernels on that stream and returns a status code (GSB_OK == 0).  No
 * entry point allocates device memory: callers pass every output buffer and
 * every scratch buffer, sized with the *_bytes() queries (gsb_splat_state_bytes,
 * gsb_splat_sort_bytes, ...), except gsb_splat_sort_static, which sorts in a
 * fixed file-scope device array.  On error
 * gsb_last_error() returns a message for the calling thread.
 *
 * The functions under "reference operators" are the kernels behind the 13
 * Python ops of the reference extension `gsplatcu` (ReparamGS-Palette,
 * gsplatcu/ext.cpp:125-139); each comment names the reference host function
 * (gsplatcu/gausplat.cu) it replaces.  Unless stated, outputs have the shapes
 * and layouts of the reference's output tensors, FP32 row-major.
 */
#ifndef GSPLAT_B200_H_
#define GSPLAT_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------- status codes */
#define GSB_OK 0
#define GSB_ERR_INVALID_ARGUMENT 1 /* bad size, pointer or mode            */
#define GSB_ERR_CUDA 2             /* a CUDA runtime call or launch failed */
#define GSB_ERR_UNSUPPORTED 3      /* valid but unsupported configuration  */
#define GSB_ERR_CAPACITY 4         /* patch count exceeded a capacity      */
#define GSB_ERR_DEVICE_TIMEOUT 5   /* a bounded device-side wait expired   */

/* Storage type of per-Gaussian colour parameters (SH weights, factors). */
#define GSB_DTYPE_F32 0
#define GSB_DTYPE_BF16 1

/* Maximum channels composited per pixel (MAX_SPLAT_DIM, gsplatcu/kernel.cu:12). */
#define GSB_MAX_CHANNELS 8

/* Message describing the last error on this thread ("" if none). */
const char* gsb_last_error(void);
/* Library ABI version, major * 100 + minor. */
int gsb_version(void);
/* Device-side status word of the library's kernels on the current device:
 * bit 0 (GSB_STATUS_BULK_TIMEOUT) -- a bounded wait for a bulk (TMA) copy gave
 * up and the kernel returned without results.  Synchronises `stream`;
 * clears the word when `clear` is non-zero. */
#define GSB_STATUS_BULK_TIMEOUT 1u
/* Bits gsb_splat_sort_capacity writes to its status word. */
#define GSB_STATUS_PATCH_OVERFLOW 2u     /* more patches than the capacity       */
#define GSB_STATUS_DEPTH_KEY_OVERFLOW 4u /* a depth key above max_depth_key      */
int gsb_device_status(uint32_t* status, int clear, void* stream);
/* Asynchronous form: enqueues on `stream` one-thread kernels that OR the
 * device status bits into *out (device memory, or pinned host memory mapped
 * into the device's address space) without synchronising or clearing; the
 * caller reads *out once the stream has passed that point.  Callers enqueue
 * it after the entry points whose kernels stage through bounded bulk-copy
 * waits (gsb_sh2weight_fast, gsb_sh2weight_fast_backward,
 * gsb_render_preprocess, gsb_render_backward(_accumulate)) and raise
 * GSB_ERR_DEVICE_TIMEOUT when a bit is set.  No counterpart in the
 * reference, whose CUDA errors are printed and ignored
 * (gsplatcu/common.cuh:19-25). */
int gsb_device_status_fetch(uint32_t* out, void* stream);
/* Test hook for that error path: launches one block that arms an mbarrier
 * for a transaction no copy delivers and waits on it at most `poll_limit`
 * times (1..65536); the wait runs out and GSB_STATUS_BULK_TIMEOUT is set, as
 * when a real bulk copy never completes.  No copy is in flight when the
 * kernel returns, so the context stays usable.  No counterpart in the
 * reference. */
int gsb_debug_expire_bulk_wait(uint32_t poll_limit, void* stream);
/* Number of kernels this library has launched in the process so far
 * (diagnostic; used to report how many of the library's kernels a timed
 * region ran). */
unsigned long long gsb_launch_count(void);

/* ===================================================== reference operators */

/* project (gsplatcu/gausplat.cu:381-419).  pc = Rcw pw + tcw; depth = -1 and
 * zero us/pcs when z < 0.2; u = (fx x/z + cx, fy y/z + cy).  du_dpcs [n,2,3]
 * may be NULL (calc_J false).  Rcw [3,3] and tcw [3] are device pointers. */
int gsb_project(int64_t n, const float* pws, const float* Rcw, const float* tcw, float fx,
                float fy, float cx, float cy, float* us, float* pcs, float* depths,
                float* du_dpcs, void* stream);

/* computeCov3D (gsplatcu/gausplat.cu:298-331).  Sigma = (R(q) S)(R(q) S)^T as
 * 6 upper entries; zero where depth < 0.2.  Jacobians [n,6,4] and [n,6,3] may
 * both be NULL. */
int gsb_compute_cov3d(int64_t n, const float* rots, const float* scales, const float* depths,
                      float* cov3ds, float* dcov3d_drots, float* dcov3d_dscales, void* stream);

/* computeCov2D (gsplatcu/gausplat.cu:333-379).  width/height are used only to
 * form tan_fov = width/(2 fx), height/(2 fy) as the reference does.
 * Jacobians [n,3,6] and [n,3,3] may both be NULL. */
int gsb_compute_cov2d(int64_t n, const float* cov3ds, const float* pcs, const float* Rcw,
                      const float* depths, float fx, float fy, float width, float height,
                      float* cov2ds, float* dcov2d_dcov3ds, float* dcov2d_dpcs, void* stream);

/* inverseCov2D (gsplatcu/gausplat.cu:590-617).  conic = adj/det with no
 * epsilon; a NaN 1/det sets depth := -1 IN PLACE.  areas (int32 [n,2]) =
 * ceil(3 sqrt|diag|).  dcinv2d_dcov2ds [n,3,3] may be NULL. */
int gsb_inverse_cov2d(int64_t n, const float* cov2ds, float* depths, float* cinv2ds,
                      int32_t* areas, float* dcinv2d_dcov2ds, void* stream);

/* sh2Weight (gsplatcu/gausplat.cu:425-462).  shs [n, sh_dim*K] band-major in
 * FP32 or BF16 (shs_dtype), sh_dim in {1,4,9,16}, 1 <= K <= 8.  weights [n,K];
 * dweight_dshs [n,1,sh_dim] and dweight_dpws [n,K,3] may both be NULL. */
int gsb_sh2weight(int64_t n, const void* shs, int shs_dtype, int sh_dim, int K, const float* pws,
                  const float* twc, float* weights, float* dweight_dshs, float* dweight_dpws,
                  void* stream);

/* sh2Weight_fast (gsplatcu/gausplat.cu:469-509), generalised to rank r.
 * shs_dc [n,K]; shs_A [n,P,r]; shs_B [n,r,Q] (rank 1 is the reference's 2-D
 * [n,P], [n,Q]); L = P*Q/K must be 0, 3, 8 or 15.  dweight_ddc [n,K] and
 * ylm [n,L] may both be NULL (calc_J false). */
int gsb_sh2weight_fast(int64_t n, const void* shs_dc, const void* shs_A, const void* shs_B,
                       int dtype, int K, int P, int Q, int rank, const float* pws,
                       const float* twc, float* weights, float* dweight_ddc, float* ylm,
                       void* stream);

/* sh2Weight_fast_B (gsplatcu/gausplat.cu:512-541), rank r.  dA [n,P,r] and
 * dB [n,r,Q] are overwritten (no atomics; one thread owns one Gaussian). */
int gsb_sh2weight_fast_backward(int64_t n, const void* shs_A, const void* shs_B, int dtype,
                                const float* ylm, const float* dloss_dw, int K, int P, int Q,
                                int rank, float* dA, float* dB, void* stream);

/* sh2Color (gsplatcu/gausplat.cu:551-584).  shs [n, sh_dim*3]; colors [n,3];
 * dcolor_dshs [n,1,sh_dim] and dcolor_dpws [n,3,3] may both be NULL. */
int gsb_sh2color(int64_t n, const void* shs, int shs_dtype, int sh_dim, const float* pws,
                 const float* twc, float* colors, float* dcolor_dshs, float* dcolor_dpws,
                 void* stream);

/* lab2rgb (gsplatcu/gausplat.cu:623-641).  lab, rgb: [3,H,W]. */
int gsb_lab2rgb(int height, int width, const float* lab, float* rgb, void* stream);

/* ------------------------------------------------------ splatting pipeline
 * splat_weight / splat_color (gsplatcu/gausplat.cu:161-249, 25-109) run as
 * four calls so that the caller owns every allocation:
 *
 *   1. gsb_splat_pack      -- per-Gaussian tile rectangles and patch counts
 *                             (getRects, gsplatcu/kernel.cu:127-162, updating
 *                             depths/areas in place like the reference), the
 *                             packed compositing records and the patch-count
 *                             prefix sum.  Needs `state` of
 *                             gsb_splat_state_bytes(...) bytes.
 *   2. gsb_splat_counts    -- copies the sizes the next step needs into a
 *                             gsb_splat_plan (synchronises `stream`, as the
 *                             reference reads its patch count back).
 *   3. gsb_splat_sort      -- key emission, sort and per-tile ranges
 *                             (createKeys / sort_by_key / getRanges).  Needs
 *                             `sort_ws` of gsb_splat_sort_bytes(plan) bytes.
 *   4. gsb_splat_draw      -- front-to-back compositing (draw_weight /
 *                             draw_color, gsplatcu/kernel.cu:194-372).
 *                             It (and the adjoint) first writes a launch
 *                             order of the tiles, longest list first, into
 *                             `state`; so a state buffer serves one draw or
 *                             adjoint at a time.
 *
 * Tile lists and ranges are bit-identical to the reference's given identical
 * us/areas/depths: keys (tile << b | uint32(depth*1000)) are emitted in
 * Gaussian order and sorted stably, b being the bit length of the largest
 * depth key, so each tile's list is ordered by (depth key, Gaussian id) as
 * the reference's stable 64-bit sort orders it; the LSD radix sort runs
 * ceil(key bits / 9) passes.  `channels` is K for weights, 3 for colours. */
typedef struct gsb_splat_plan {
  int64_t patches;        /* M, total (tile, Gaussian) patches          */
  uint32_t max_depth_key; /* max uint32(depth*1000) of binned Gaussians */
  uint32_t reserved;      /* zero                                       */
} gsb_splat_plan;

size_t gsb_splat_state_bytes(int64_t n, int channels, int height, int width);

int gsb_splat_pack(int64_t n, int height, int width, int channels, const float* us,
                   const float* cinv2ds, const float* alphas, const void* feats, int feat_dtype,
                   float* depths, int32_t* areas, void* state, void* stream);

/* Fills *plan; blocks until `stream` has finished step 1. */
int gsb_splat_counts(int64_t n, int height, int width, const void* state, gsb_splat_plan* plan,
                     void* stream);

size_t gsb_splat_sort_bytes(int64_t n, int height, int width, const gsb_splat_plan* plan);

/* gsid_out [patches] (int32) receives the sorted Gaussian ids; ranges_out
 * [tiles,2] (int32) the per-tile [start,end) -- (0,0) for empty tiles and,
 * as in the reference's getRanges, (0,0) for the single tile when M == 1. */
int gsb_splat_sort(int64_t n, int height, int width, const gsb_splat_plan* plan,
                   const void* state, void* sort_ws, int32_t* gsid_out, int32_t* ranges_out,
                   void* stream);

/* gsb_splat_sort without the caller workspace; no counterpart in the
 * reference extension.  For callers that cannot allocate device memory where
 * they render (device memory owned by another runtime's pool, a plug-in
 * handed only its input and output buffers, a fixed start-up footprint):
 * the sort's temporaries live in one device array inside this library, of
 * gsb_splat_sort_static_max_bytes() bytes (32 MiB: about 2.0M patches with
 * 32-bit keys, 1.3M with 64-bit keys), which every GPU that loads the library
 * holds until the process exits.  Plans needing more return GSB_ERR_CAPACITY
 * with a message; use gsb_splat_sort then.  Allocates nothing; the first
 * call on each device looks up the array's device address (once per device
 * and CUDA context, with that device current: after a device reset or a
 * re-created primary context the next call looks it up again), so make the
 * first call in each context before any stream capture.  All
 * calls on a device share the array and it keeps the last call's contents
 * (nothing needs to start at zero), so calls that overlap on the GPU race:
 * order them on one stream.  Inputs, outputs and results as gsb_splat_sort. */
size_t gsb_splat_sort_static_max_bytes(void);
int gsb_splat_sort_static(int64_t n, int height, int width, const gsb_splat_plan* plan,
                          const void* state, int32_t* gsid_out, int32_t* ranges_out,
                          void* stream);

/* Step 3 without the host read-back of step 2, for callers that keep the
 * whole render on the device (CUDA-graph capture, serving): the sort is
 * sized for `patch_capacity` patches and depth keys up to `max_depth_key`
 * (uint32(depth*1000)); the true patch count stays on the device.  Needs
 * `sort_ws` of gsb_splat_sort_capacity_bytes(...) bytes and gsid_out of
 * patch_capacity entries.  status (device uint32[3]) receives the overflow
 * bits GSB_STATUS_PATCH_OVERFLOW / GSB_STATUS_DEPTH_KEY_OVERFLOW (or 0) and
 * the true patch count (low, high word); it may be NULL when the caller
 * reads the same words through gsb_splat_patch_status.  On an
 * overflow every range is left empty (the image then shows nothing) and the
 * caller re-renders with a larger capacity.  Without overflow the results
 * equal gsb_splat_sort's.  No counterpart in the reference, which always
 * reads the patch count back (gsplatcu/gausplat.cu:199-201). */
size_t gsb_splat_sort_capacity_bytes(int64_t n, int height, int width, int64_t patch_capacity,
                                     uint32_t max_depth_key);
/* Writes only the status words of gsb_splat_sort_capacity (overflow bits and
 * the true patch count, status = device uint32[3]) for `state`, so that a
 * caller can copy them to the host and learn the patch count while the sort
 * and compositing already run. */
int gsb_splat_patch_status(int64_t n, int height, int width, int64_t patch_capacity,
                           uint32_t max_depth_key, const void* state, uint32_t* status,
                           void* stream);
int gsb_splat_sort_capacity(int64_t n, int height, int width, int64_t patch_capacity,
                            uint32_t max_depth_key, const void* state, void* sort_ws,
                            int32_t* gsid_out, int32_t* ranges_out, uint32_t* status,
                            void* stream);

/* out [channels,H,W], contrib [H,W] (1-based index of the last blended
 * Gaussian in the tile list), final_tau [H,W].  Pixels of tiles without
 * patches are set to 0 / 0 / tau_init (0 for weights, 1 for colours, as
 * gsplatcu/gausplat.cu:178 and :39 initialise them). */
int gsb_splat_draw(int64_t n, int height, int width, int channels, const int32_t* ranges,
                   const int32_t* gsid, const void* state, float tau_init, float* out,
                   int32_t* contrib, float* final_tau, void* stream);

/* splat_weight_B / splat_color_B (gsplatcu/gausplat.cu:252-292, 111-155):
 * reverse-order adjoint of the compositing.  Re-packs the records into
 * `state` (gsb_splat_state_bytes(n, channels, height, width) bytes) from the
 * forward's inputs.  Outputs are
 * ACCUMULATED (+=) and may be NULL:
 *   dfeats [n,channels]  -- dL/dweights (splat_weight_B) / dL/dcolors
 *   dalphas [n], dus [n,2], dcinv2ds [n,3]  -- the geometry/opacity adjoint of
 *   draw_color_B (gsplatcu/kernel.cu:1176-1284), here for any channel count.
 * dloss_dtau [H,W] (may be NULL) adds the final-transmittance term of
 * vanilla_3dgs/gsplatcu/kernel.cu:912-919. */
int gsb_splat_backward(int64_t n, int height, int width, int channels, const float* us,
                       const float* cinv2ds, const float* alphas, const void* feats,
                       int feat_dtype, const int32_t* ranges, const int32_t* gsid,
                       const int32_t* contrib, const float* final_tau, const float* dloss_dout,
                       const float* dloss_dtau, void* state, float* dfeats, float* dalphas,
                       float* dus, float* dcinv2ds, void* stream);

/* The same adjoint on records already packed into `state` by gsb_splat_pack
 * for these inputs (no re-pack).  Used when the forward's state is kept. */
int gsb_splat_backward_packed(int64_t n, int height, int width, int channels,
                              const int32_t* ranges, const int32_t* gsid, const int32_t* contrib,
                              const float* final_tau, const float* dloss_dout,
                              const float* dloss_dtau, const void* state, float* dfeats,
                              float* dalphas, float* dus, float* dcinv2ds, void* stream);

/* ------------------------------------------------------------- loss side
 * Palette colour composite and L1 loss in one pass (no counterpart in the
 * reference extension, whose callers compute the loss in torch,
 * finetune.py:356-389):
 *   image[c] = sum_k palette[k][c] layer[k]   (palette [K,3], layer [K,H,W]);
 *   *loss = mean |image - target| over the 3*H*W values (target [3,H,W]);
 *   dlayer[k] = sum_c palette[k][c] sign(image[c] - target[c]) / (3HW);
 *   dpalette[k][c] = sum_pixels layer[k] sign(image[c] - target[c]) / (3HW).
 * image, dlayer and dpalette may be NULL; loss and dpalette are overwritten. */
int gsb_palette_l1(int K, int height, int width, const float* layer, const float* palette,
                   const float* target, float* image, float* loss, float* dlayer,
                   float* dpalette, void* stream);

/* The finetune step's loss on the rendered weights (finetune.py:356-389, the
 * target by gsplat/gsmodel.py:219-285), one pass over the image: the
 * barycentric target W of the colour image `target` [3,H,W] in the palette
 * {black, white, chroma [chroma_count,3]} (optionally clamped to >= 0 and
 * renormalised, `clamp`), then loss[0] = loss[1] + loss[2] with
 * loss[1] = mean((layer - W)^2) (GSB_LOSS_MSE) or mean|layer - W| (GSB_LOSS_L1)
 * over the K = chroma_count + 2 channels, loss[2] = lambda_pos *
 * mean(relu(-layer)).  dlayer [K,H,W] (overwritten) and dchroma
 * [chroma_count,3] (overwritten) are the loss gradients, the latter through
 * the target; target_weights [K,H,W] receives W.  Outputs other than loss may
 * be NULL. */
#define GSB_LOSS_MSE 0
#define GSB_LOSS_L1 1
int gsb_palette_geo_loss(int chroma_count, int height, int width, const float* layer,
                         const float* target, const float* chroma, int clamp, int kind,
                         float lambda_pos, float* target_weights, float* loss, float* dlayer,
                         float* dchroma, void* stream);

/* The differentiation workload's loss, one launch (plus a one-block init): the
 * colour image img_c = sum_k palette[k][c] layer_k and
 *   loss[0] = (1 - lambda_ssim) loss[1] + lambda_ssim (1 - loss[2]) + loss[3],
 *   loss[1] = mean |img - target|, loss[2] = mean SSIM(img, target),
 *   loss[3] = lambda_pos mean(relu(-layer)),
 * i.e. gau_loss (vanilla_3dgs/gsplat/pytorch_ssim.py:26-67: 11x11 Gaussian
 * window, sigma 1.5, zero padding, C1 = (0.01 data_range)^2, C2 =
 * (0.03 data_range)^2; data_range 1 there) plus the negative-weight penalty of
 * finetune.py:375,381, with dlayer [K,H,W] and dpalette [K,3] its gradients
 * (overwritten; either may be NULL) and image [3,H,W] (may be NULL) the colour
 * image.  With palette NULL, layer is the colour image itself (K must be 3) and
 * dlayer the image gradient: gau_loss alone when lambda_pos is 0. */
int gsb_palette_l1_ssim(int K, int height, int width, const float* layer, const float* palette,
                        const float* target, float lambda_ssim, float lambda_pos,
                        float data_range, float* image, float* loss, float* dlayer,
                        float* dpalette, void* stream);

/* ============================================================ fused path
 * One view of the palette-weight rasterizer with the per-Gaussian work of
 * project / computeCov3D / computeCov2D / sh2Weight(_fast) / inverseCov2D /
 * getRects done in one kernel (gsb_render_preprocess, filling the same
 * `state` as gsb_splat_pack and its count step); then gsb_splat_counts /
 * gsb_splat_sort / gsb_splat_draw as for splat_weight (gsplat/gsmodel.py:
 * 107-118, 155-170).  gsb_render_backward is the adjoint of the whole view:
 * compositing and the per-Gaussian chain to every parameter
 * (vanilla_3dgs/gsplat/gsmodel.py:65-75 is the reference's chain for the
 * geometry, gsplat/gsmodel.py:120-130, 172-200 for the weights). */
#define GSB_WEIGHTS_FULL 0    /* shs [n,16K], SH order 3, band-major          */
#define GSB_WEIGHTS_LOWRANK 1 /* dc [n,K], A [n,P,rank], B [n,rank,Q]         */

typedef struct gsb_camera {
  const float* Rcw; /* device [3,3] row-major world -> camera rotation  */
  const float* tcw; /* device [3] translation                          */
  const float* twc; /* device [3] camera centre in world coordinates    */
  float fx, fy, cx, cy;
  int width, height;
} gsb_camera;

typedef struct gsb_palette_params {
  int mode;       /* GSB_WEIGHTS_FULL or GSB_WEIGHTS_LOWRANK              */
  int dtype;      /* GSB_DTYPE_F32 or GSB_DTYPE_BF16 (FP32 arithmetic)    */
  int K;          /* palette entries = channels composited               */
  int P, Q, rank; /* low-rank factor shape                                */
  const void* w0; /* full: shs [n,16K]; low-rank: dc [n,K]               */
  const void* A;  /* low-rank: [n,P,rank]                                 */
  const void* B;  /* low-rank: [n,rank,Q]                                 */
  const float* palette; /* NULL: records carry the K weights.  Else device
                         * [K,3] RGB palette: records carry each Gaussian's
                         * colour sum_k w_k palette[k] (3 channels; state of
                         * gsb_splat_state_bytes(n, 3, H, W)), the palette-edit
                         * render of gsplat/gsmodel.py:488-509 + 14-26. */
} gsb_palette_params;

/* pws [n,3], rots [n,4] (w,x,y,z), scales [n,3], alphas [n]; `state` of
 * gsb_splat_state_bytes(n, K (3 with a palette), height, width) bytes,
 * 256-byte aligned;
 * depths_out [n] (may be NULL) receives the camera depth, or -1 for
 * Gaussians dropped by the depth, conic or tile tests (the reference's
 * depths after its in-place updates).  Supported shapes: full K in 3..8;
 * low-rank (K,P,Q,rank) in {(5,5,15,1..4), (3,3,15,1), (4,4,15,1),
 * (6,6,15,1), (6,6,15,3)}. */
int gsb_render_preprocess(int64_t n, const gsb_camera* cam, const float* pws, const float* rots,
                          const float* scales, const float* alphas,
                          const gsb_palette_params* params, void* state, float* depths_out,
                          void* stream);

/* The weight-parameter half of the reference backward in one kernel: from
 * dloss_dweights [n,K] (splat_weight_B's output) to dw0 (shs [n,16K] for
 * full weights, dc [n,K] for low-rank) and dA [n,P,rank], dB [n,rank,Q]
 * (FP32, overwritten), recomputing the view direction and SH basis from
 * pws and cam->twc.  Replaces, on the GPU, the reference backward's
 * batched outer product dW x dweight_dshs (gsplat/gsmodel.py:140-143) and
 * its dW * dweight_ddc + sh2Weight_fast_B pair (gsmodel.py:194-198), so the
 * forward needs no Jacobian outputs.  Shapes as gsb_render_preprocess. */
int gsb_palette_weights_backward(int64_t n, const gsb_camera* cam, const float* pws,
                                 const gsb_palette_params* params, const float* dloss_dweights,
                                 float* dw0, float* dA, float* dB, void* stream);

/* ------------------------------------------------ batched compositing
 * Several images' compositing in one persistent kernel (the serving loop's
 * batches of palette-edit renders; no counterpart in the reference, which
 * renders one request per call).  Each image is described by its packed
 * state (gsb_render_preprocess or gsb_splat_pack), sorted tile lists and
 * output buffers; all images of a batch carry the same channel count.  The
 * caller packs a batch into a host table (gsb_draw_batch_pack, host code
 * only), copies it to a device buffer of gsb_draw_batch_bytes(max_jobs)
 * bytes (16-byte aligned) and launches gsb_draw_batch on that buffer.  The
 * kernel's blocks claim (image, tile) items from the table's queue with an
 * atomic counter, so tiles of large and small images share the SMs; each
 * tile is composited exactly as gsb_splat_draw composites it (results are
 * bit-identical to rendering the images one by one).  The copy and the
 * launch can be captured in a CUDA graph: replaying the graph copies the
 * host table's current contents.  A device buffer must not be reused for
 * another batch before the kernel reading it has finished. */
typedef struct gsb_draw_job {
  const void* state;      /* packed state: gsb_splat_state_bytes(n, channels, height, width) */
  int64_t n;              /* Gaussians of the image                                        */
  int height, width;
  int channels;           /* record channels (equal for every job of a batch)              */
  const int32_t* ranges;  /* [tiles,2] tile ranges of the sorted lists                     */
  const int32_t* gsid;    /* sorted Gaussian ids                                           */
  float tau_init;         /* final_tau of empty tiles: 0 (weights) or 1 (colours)          */
  float* out;             /* [channels,height,width]                                       */
  int32_t* contrib;       /* [height,width]                                                */
  float* final_tau;       /* [height,width]                                                */
} gsb_draw_job;
size_t gsb_draw_batch_bytes(int max_jobs);
int gsb_draw_batch_pack(const gsb_draw_job* jobs, int njobs, void* host_table,
                        size_t table_bytes);
int gsb_draw_batch(const void* dev_table, int channels, void* stream);

/* Scratch bytes gsb_render_backward needs for the per-Gaussian screen-space
 * gradients. */
size_t gsb_render_backward_bytes(int64_t n, int K);

/* dloss_dout [K,H,W]; dloss_dtau [H,W] may be NULL.  Outputs (FP32,
 * overwritten): dw0 (shs [n,16K] or dc [n,K]), dA [n,P,rank], dB [n,rank,Q]
 * always; the geometry gradients dpws [n,3], drots [n,4], dscales [n,3],
 * dalphas [n] either all four or none.  With none (the reference backward's
 * scope) only the weight gradients are computed and dloss_dtau, which
 * reaches only geometry and opacity, is ignored. */
int gsb_render_backward(int64_t n, const gsb_camera* cam, const float* pws, const float* rots,
                        const float* scales, const float* alphas,
                        const gsb_palette_params* params, const void* state,
                        const int32_t* ranges, const int32_t* gsid, const int32_t* contrib,
                        const float* final_tau, const float* dloss_dout, const float* dloss_dtau,
                        void* scratch, float* dpws, float* drots, float* dscales, float* dalphas,
                        float* dw0, float* dA, float* dB, void* stream);

/* gsb_render_backward for several views of one scene: the same arguments and
 * gradients, but ADDED to what dw0, dA, dB (and, when given, dpws, drots,
 * dscales, dalphas) already hold instead of overwriting them.  A training
 * step over a batch of views calls gsb_render_backward for its first view and
 * this entry for the others, so the views' gradients are summed in FP32 in the
 * output buffers, whatever the storage dtype of the parameters.  The reference
 * has no counterpart: its backward handles one view per call, and a batch of
 * views is summed by torch autograd in the parameters' dtype. */
int gsb_render_backward_accumulate(int64_t n, const gsb_camera* cam, const float* pws,
                                   const float* rots, const float* scales, const float* alphas,
                                   const gsb_palette_params* params, const void* state,
                                   const int32_t* ranges, const int32_t* gsid,
                                   const int32_t* contrib, const float* final_tau,
                                   const float* dloss_dout, const float* dloss_dtau,
                                   void* scratch, float* dpws, float* drots, float* dscales,
                                   float* dalphas, float* dw0, float* dA, float* dB, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GSPLAT_B200_H_ */
