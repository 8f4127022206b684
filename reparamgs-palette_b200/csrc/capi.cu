// extern "C" entry points of libgsplat_b200.so (declared in gsplat_b200.h):
// argument validation, workspace carving and kernel launches.  No entry point
// allocates device memory or synchronises, except gsb_splat_counts, which
// must return the patch count to the host.
#include <mutex>
#include <cmath>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "gsb_common.cuh"
#include "gsb_internal.h"

namespace gsb {

static thread_local char g_err[512] = {0};
static std::atomic<unsigned long long> g_launches{0};

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int check_launch(const char* what, int launches) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return GSB_ERR_CUDA;
  }
  g_launches.fetch_add((unsigned long long)launches, std::memory_order_relaxed);
  return GSB_OK;
}

// lab2rgb -- gsplatcu/kernel.cu:1385-1428: CIE L*a*b* (L in [0,1]) -> sRGB.
__device__ __forceinline__ float lab_finv(float t) {
  const float delta = 6.0f / 29.0f;
  return (t > delta) ? t * t * t : 3.f * delta * delta * (t - 4.f / 29.f);
}
__device__ __forceinline__ float srgb_gamma(float c) {
  return (c <= 0.0031308f) ? 12.92f * c : 1.055f * powf(c, 1.f / 2.4f) - 0.055f;
}
__global__ void k_lab2rgb(int H, int W, const float* __restrict__ lab, float* __restrict__ rgb) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= W || py >= H) return;
  const int64_t p = (int64_t)py * W + px, P = (int64_t)H * W;
  const float L = lab[p] * 100.f, a = lab[P + p], b = lab[2 * P + p];
  const float fy = (L + 16.f) / 116.f, fx = a / 500.f + fy, fz = fy - b / 200.f;
  const float X = 0.95047f * lab_finv(fx), Y = 1.00000f * lab_finv(fy), Z = 1.08883f * lab_finv(fz);
  const float r = fmaxf(0.f, fminf(1.f, 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z));
  const float g = fmaxf(0.f, fminf(1.f, -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z));
  const float bl = fmaxf(0.f, fminf(1.f, 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z));
  rgb[p] = srgb_gamma(r);
  rgb[P + p] = srgb_gamma(g);
  rgb[2 * P + p] = srgb_gamma(bl);
}

int launch_lab2rgb(int H, int W, const float* lab, float* rgb, cudaStream_t st) {
  if (H == 0 || W == 0) return GSB_OK;
  dim3 block(16, 16), grid(div_up(W, 16), div_up(H, 16));
  k_lab2rgb<<<grid, block, 0, st>>>(H, W, lab, rgb);
  return check_launch("lab2rgb");
}

static bool valid_sh_dim(int nb) { return nb == 1 || nb == 4 || nb == 9 || nb == 16; }
static bool valid_dtype(int d) { return d == GSB_DTYPE_F32 || d == GSB_DTYPE_BF16; }

}  // namespace gsb

using namespace gsb;

#define ST(s) ((cudaStream_t)(s))
#define GSB_API extern "C" __attribute__((visibility("default")))

GSB_API const char* gsb_last_error(void) { return g_err; }
GSB_API int gsb_version(void) { return 100; }
GSB_API int gsb_device_status(uint32_t* status, int clear, void* stream) {
  GSB_CHECK_ARG(status, "device_status: null pointer");
  uint32_t a = 0, b = 0;
  int rc = lowrank_status(&a, clear != 0, ST(stream));
  if (rc) return rc;
  rc = fused_status(&b, clear != 0, ST(stream));
  if (rc) return rc;
  *status = a | b;
  return GSB_OK;
}

// The device addresses of the status words of the files whose kernels wait
// on bulk copies (low-rank weights, fused preprocess / adjoint), looked up
// once per device and CUDA context.
struct StatusWords {
  unsigned long long ctx;
  const uint32_t* w[2];
};
static StatusWords g_status_words[64];
static std::mutex g_status_mutex;

static int status_words(const uint32_t** w) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("device_status_fetch", 0);
  if (dev < 0 || dev >= 64) {
    set_error("device_status_fetch: device %d beyond the 64 supported", dev);
    return GSB_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_status_mutex);
  const unsigned long long ctx = current_context_id();
  StatusWords& e = g_status_words[dev];
  if (!e.w[0] || ctx == 0 || e.ctx != ctx) {
    e.w[0] = lowrank_status_word();
    e.w[1] = fused_status_word();
    e.ctx = ctx;
    if (!e.w[0] || !e.w[1]) {
      e.w[0] = nullptr;
      set_error("device_status_fetch: cudaGetSymbolAddress failed on device %d", dev);
      return GSB_ERR_CUDA;
    }
  }
  for (int k = 0; k < 2; ++k) w[k] = e.w[k];
  return GSB_OK;
}

// ORs the status words into *out (device memory or mapped host memory; one
// thread, so the read-modify-write of *out is not shared).  The words
// themselves are left set: only gsb_device_status clears them.
__global__ void k_status_fetch(const uint32_t* a, const uint32_t* b, uint32_t* out) {
  pdl_wait();
  const uint32_t v = *(const volatile uint32_t*)a | *(const volatile uint32_t*)b;
  if (v) *(volatile uint32_t*)out |= v;
}

GSB_API int gsb_device_status_fetch(uint32_t* out, void* stream) {
  GSB_CHECK_ARG(out, "device_status_fetch: null pointer");
  const uint32_t* w[2];
  const int rc = status_words(w);
  if (rc) return rc;
  launch_pdl(k_status_fetch, dim3(1), dim3(1), 0, ST(stream), w[0], w[1], out);
  return check_launch("device_status_fetch");
}

GSB_API int gsb_debug_expire_bulk_wait(uint32_t poll_limit, void* stream) {
  GSB_CHECK_ARG(poll_limit >= 1 && poll_limit <= (1u << 16),
                "debug_expire_bulk_wait: poll_limit must be in [1, 65536]");
  return expire_bulk_wait(poll_limit, ST(stream));
}

GSB_API unsigned long long gsb_launch_count(void) {
  return g_launches.load(std::memory_order_relaxed);
}

GSB_API int gsb_project(int64_t n, const float* pws, const float* Rcw, const float* tcw, float fx,
                        float fy, float cx, float cy, float* us, float* pcs, float* depths,
                        float* du_dpcs, void* stream) {
  GSB_CHECK_ARG(n >= 0, "project: n < 0");
  GSB_CHECK_ARG(n == 0 || (pws && Rcw && tcw && us && pcs && depths), "project: null pointer");
  return launch_project(n, pws, Rcw, tcw, fx, fy, cx, cy, us, pcs, depths, du_dpcs, ST(stream));
}

GSB_API int gsb_compute_cov3d(int64_t n, const float* rots, const float* scales,
                              const float* depths, float* cov3ds, float* dq, float* ds,
                              void* stream) {
  GSB_CHECK_ARG(n >= 0, "computeCov3D: n < 0");
  GSB_CHECK_ARG(n == 0 || (rots && scales && depths && cov3ds), "computeCov3D: null pointer");
  GSB_CHECK_ARG((dq == nullptr) == (ds == nullptr), "computeCov3D: pass both Jacobians or none");
  GSB_CHECK_ARG(((uintptr_t)rots & 15) == 0, "computeCov3D: rots must be 16-byte aligned");
  return launch_cov3d(n, rots, scales, depths, cov3ds, dq, ds, ST(stream));
}

GSB_API int gsb_compute_cov2d(int64_t n, const float* cov3ds, const float* pcs, const float* Rcw,
                              const float* depths, float fx, float fy, float width, float height,
                              float* cov2ds, float* d3, float* dp, void* stream) {
  GSB_CHECK_ARG(n >= 0, "computeCov2D: n < 0");
  GSB_CHECK_ARG(n == 0 || (cov3ds && pcs && Rcw && depths && cov2ds), "computeCov2D: null pointer");
  GSB_CHECK_ARG((d3 == nullptr) == (dp == nullptr), "computeCov2D: pass both Jacobians or none");
  // tan of the half field of view, formed in FP32 as gsplatcu/gausplat.cu:357-358
  const float tanx = width / (2 * fx);
  const float tany = height / (2 * fy);
  return launch_cov2d(n, cov3ds, pcs, Rcw, depths, fx, fy, tanx, tany, cov2ds, d3, dp, ST(stream));
}

GSB_API int gsb_inverse_cov2d(int64_t n, const float* cov2ds, float* depths, float* cinv2ds,
                              int32_t* areas, float* dcinv, void* stream) {
  GSB_CHECK_ARG(n >= 0, "inverseCov2D: n < 0");
  GSB_CHECK_ARG(n == 0 || (cov2ds && depths && cinv2ds && areas), "inverseCov2D: null pointer");
  return launch_inverse_cov2d(n, cov2ds, depths, cinv2ds, areas, dcinv, ST(stream));
}

GSB_API int gsb_sh2weight(int64_t n, const void* shs, int shs_dtype, int sh_dim, int K,
                          const float* pws, const float* twc, float* weights, float* dshs,
                          float* dpws, void* stream) {
  GSB_CHECK_ARG(n >= 0, "sh2Weight: n < 0");
  GSB_CHECK_ARG(K >= 1 && K <= GSB_MAX_CHANNELS, "sh2Weight: num_palette must be in [1, %d], got %d",
                GSB_MAX_CHANNELS, K);
  GSB_CHECK_ARG(valid_sh_dim(sh_dim), "sh2Weight: SH bands per channel must be 1, 4, 9 or 16, got %d",
                sh_dim);
  GSB_CHECK_ARG(valid_dtype(shs_dtype), "sh2Weight: unsupported shs dtype %d", shs_dtype);
  GSB_CHECK_ARG(n == 0 || (shs && pws && twc && weights), "sh2Weight: null pointer");
  GSB_CHECK_ARG((dshs == nullptr) == (dpws == nullptr), "sh2Weight: pass both Jacobians or none");
  return launch_sh2feat(n, shs, shs_dtype, sh_dim, K, pws, twc, weights, dshs, dpws, ST(stream));
}

GSB_API int gsb_sh2color(int64_t n, const void* shs, int shs_dtype, int sh_dim, const float* pws,
                         const float* twc, float* colors, float* dshs, float* dpws, void* stream) {
  GSB_CHECK_ARG(n >= 0, "sh2Color: n < 0");
  GSB_CHECK_ARG(valid_sh_dim(sh_dim), "sh2Color: SH bands must be 1, 4, 9 or 16, got %d", sh_dim);
  GSB_CHECK_ARG(valid_dtype(shs_dtype), "sh2Color: unsupported shs dtype %d", shs_dtype);
  GSB_CHECK_ARG(n == 0 || (shs && pws && twc && colors), "sh2Color: null pointer");
  GSB_CHECK_ARG((dshs == nullptr) == (dpws == nullptr), "sh2Color: pass both Jacobians or none");
  return launch_sh2feat(n, shs, shs_dtype, sh_dim, 3, pws, twc, colors, dshs, dpws, ST(stream));
}

static int check_lowrank(const char* op, int K, int P, int Q, int rank, int dtype, int* L) {
  GSB_CHECK_ARG(K >= 1 && K <= GSB_MAX_CHANNELS, "%s: num_palette must be in [1, %d], got %d", op,
                GSB_MAX_CHANNELS, K);
  GSB_CHECK_ARG(P >= 1 && Q >= 1 && rank >= 1, "%s: P, Q and rank must be positive", op);
  GSB_CHECK_ARG((P * Q) % K == 0, "%s: P*Q (%d) must be a multiple of num_palette (%d)", op, P * Q, K);
  *L = P * Q / K;
  GSB_CHECK_ARG(*L == 0 || *L == 3 || *L == 8 || *L == 15,
                "%s: P*Q/K = %d higher-order SH coefficients; must be 3, 8 or 15", op, *L);
  GSB_CHECK_ARG(valid_dtype(dtype), "%s: unsupported dtype %d", op, dtype);
  return GSB_OK;
}

GSB_API int gsb_sh2weight_fast(int64_t n, const void* dc, const void* A, const void* B, int dtype,
                               int K, int P, int Q, int rank, const float* pws, const float* twc,
                               float* weights, float* ddc, float* ylm, void* stream) {
  int L = 0;
  int rc = check_lowrank("sh2Weight_fast", K, P, Q, rank, dtype, &L);
  if (rc) return rc;
  GSB_CHECK_ARG(n >= 0, "sh2Weight_fast: n < 0");
  GSB_CHECK_ARG(n == 0 || (dc && A && B && pws && twc && weights), "sh2Weight_fast: null pointer");
  return launch_sh2weight_lowrank(n, dc, A, B, dtype, K, P, Q, rank, L, pws, twc, weights, ddc,
                                  L > 0 ? ylm : nullptr, ST(stream));
}

GSB_API int gsb_sh2weight_fast_backward(int64_t n, const void* A, const void* B, int dtype,
                                        const float* ylm, const float* dw, int K, int P, int Q,
                                        int rank, float* dA, float* dB, void* stream) {
  int L = 0;
  int rc = check_lowrank("sh2Weight_fast_B", K, P, Q, rank, dtype, &L);
  if (rc) return rc;
  GSB_CHECK_ARG(n >= 0, "sh2Weight_fast_B: n < 0");
  GSB_CHECK_ARG(n == 0 || (A && B && dw && dA && dB && (L == 0 || ylm)),
                "sh2Weight_fast_B: null pointer");
  return launch_sh2weight_lowrank_b(n, A, B, dtype, ylm, dw, K, P, Q, rank, L, dA, dB, ST(stream));
}

GSB_API int gsb_lab2rgb(int height, int width, const float* lab, float* rgb, void* stream) {
  GSB_CHECK_ARG(height >= 0 && width >= 0, "lab2rgb: negative size");
  GSB_CHECK_ARG((height == 0 || width == 0) || (lab && rgb), "lab2rgb: null pointer");
  return launch_lab2rgb(height, width, lab, rgb, ST(stream));
}

// ----------------------------------------------------------------- splat
static int check_image(const char* op, int64_t n, int H, int W, int C) {
  GSB_CHECK_ARG(n >= 0 && n < (int64_t)INT32_MAX, "%s: Gaussian count %lld out of range", op,
                (long long)n);
  GSB_CHECK_ARG(H >= 0 && W >= 0, "%s: negative image size", op);
  GSB_CHECK_ARG((int64_t)div_up(W, kTile) < 65536 && (int64_t)div_up(H, kTile) < 65536,
                "%s: image too large (%d x %d)", op, W, H);
  GSB_CHECK_ARG(C >= 1 && C <= GSB_MAX_CHANNELS, "%s: channels must be in [1, %d], got %d", op,
                GSB_MAX_CHANNELS, C);
  return GSB_OK;
}

GSB_API size_t gsb_splat_state_bytes(int64_t n, int channels, int height, int width) {
  if (n < 0 || channels < 1 || channels > GSB_MAX_CHANNELS || height < 0 || width < 0) return 0;
  return splat_state_bytes(n, channels, height, width);
}

GSB_API int gsb_splat_pack(int64_t n, int height, int width, int channels, const float* us,
                           const float* cinv2ds, const float* alphas, const void* feats,
                           int feat_dtype, float* depths, int32_t* areas, void* state,
                           void* stream) {
  int rc = check_image("splat_pack", n, height, width, channels);
  if (rc) return rc;
  GSB_CHECK_ARG(valid_dtype(feat_dtype), "splat_pack: unsupported feature dtype %d", feat_dtype);
  GSB_CHECK_ARG(state && ((uintptr_t)state & 255) == 0, "splat_pack: state must be 256-byte aligned");
  GSB_CHECK_ARG(n == 0 || (us && cinv2ds && alphas && feats && depths && areas),
                "splat_pack: null pointer");
  const SplatState s = carve_state(state, n, channels, height, width);
  rc = launch_pack(n, height, width, channels, us, cinv2ds, alphas, feats, feat_dtype, depths,
                   areas, true, s, ST(stream));
  if (rc) return rc;
  return launch_count_scan(n, s, ST(stream));
}

GSB_API int gsb_splat_counts(int64_t n, int height, int width, const void* state,
                             gsb_splat_plan* plan, void* stream) {
  GSB_CHECK_ARG(n >= 0 && height >= 0 && width >= 0 && state && plan,
                "splat_counts: bad argument");
  const SplatState s = carve_state((void*)state, n, 1, height, width);
  uint32_t v[4];
  if (cudaMemcpyAsync(v, s.stats, sizeof(v), cudaMemcpyDeviceToHost, ST(stream)) != cudaSuccess ||
      cudaStreamSynchronize(ST(stream)) != cudaSuccess)
    return check_launch("splat_counts", 0);
  GSB_CHECK_ARG(v[3] == 0 && v[0] < (uint32_t)INT32_MAX,
                "splat_counts: patch count exceeds the int32 index range");
  plan->patches = v[0];
  plan->max_depth_key = v[1];
  return GSB_OK;
}

GSB_API size_t gsb_splat_sort_bytes(int64_t n, int height, int width, const gsb_splat_plan* plan) {
  if (n < 0 || height < 0 || width < 0 || !plan || plan->patches < 0) return 0;
  return make_sort_plan(n, height, width, plan->patches, plan->max_depth_key).bytes_total;
}

GSB_API int gsb_splat_sort(int64_t n, int height, int width, const gsb_splat_plan* plan,
                           const void* state, void* sort_ws, int32_t* gsid_out,
                           int32_t* ranges_out, void* stream) {
  int rc = check_image("splat_sort", n, height, width, 1);
  if (rc) return rc;
  GSB_CHECK_ARG(plan && plan->patches >= 0 && plan->patches < (int64_t)INT32_MAX,
                "splat_sort: bad plan");
  GSB_CHECK_ARG(state && ranges_out, "splat_sort: null pointer");
  GSB_CHECK_ARG(plan->patches == 0 || (sort_ws && gsid_out), "splat_sort: null workspace/output");
  const SortPlan p = make_sort_plan(n, height, width, plan->patches, plan->max_depth_key);
  const SplatState s = carve_state((void*)state, n, 1, height, width);
  return launch_sort(p, n, height, width, s, sort_ws, gsid_out, ranges_out, ST(stream));
}

GSB_API size_t gsb_splat_sort_capacity_bytes(int64_t n, int height, int width,
                                             int64_t patch_capacity, uint32_t max_depth_key) {
  if (n < 0 || height < 0 || width < 0 || patch_capacity < 0) return 0;
  return make_sort_plan(n, height, width, patch_capacity, max_depth_key).bytes_total;
}

GSB_API int gsb_splat_patch_status(int64_t n, int height, int width, int64_t patch_capacity,
                                   uint32_t max_depth_key, const void* state, uint32_t* status,
                                   void* stream) {
  int rc = check_image("splat_patch_status", n, height, width, 1);
  if (rc) return rc;
  GSB_CHECK_ARG(state && status, "splat_patch_status: null pointer");
  const SortPlan p = make_sort_plan(n, height, width, patch_capacity, max_depth_key);
  const SplatState s = carve_state((void*)state, n, 1, height, width);
  return launch_patch_status(p, s, status, ST(stream));
}

GSB_API int gsb_splat_sort_capacity(int64_t n, int height, int width, int64_t patch_capacity,
                                    uint32_t max_depth_key, const void* state, void* sort_ws,
                                    int32_t* gsid_out, int32_t* ranges_out, uint32_t* status,
                                    void* stream) {
  int rc = check_image("splat_sort_capacity", n, height, width, 1);
  if (rc) return rc;
  GSB_CHECK_ARG(patch_capacity >= 0 && patch_capacity < (int64_t)INT32_MAX,
                "splat_sort_capacity: capacity out of range");
  GSB_CHECK_ARG(state && ranges_out, "splat_sort_capacity: null pointer");
  GSB_CHECK_ARG(patch_capacity == 0 || (sort_ws && gsid_out),
                "splat_sort_capacity: null workspace/output");
  const SortPlan p = make_sort_plan(n, height, width, patch_capacity, max_depth_key);
  const SplatState s = carve_state((void*)state, n, 1, height, width);
  return launch_sort_capacity(p, n, height, width, s, sort_ws, gsid_out, ranges_out, status,
                              ST(stream));
}

GSB_API int gsb_splat_draw(int64_t n, int height, int width, int channels, const int32_t* ranges,
                           const int32_t* gsid, const void* state, float tau_init, float* out,
                           int32_t* contrib, float* final_tau, void* stream) {
  int rc = check_image("splat_draw", n, height, width, channels);
  if (rc) return rc;
  GSB_CHECK_ARG(ranges && state && out && contrib && final_tau, "splat_draw: null pointer");
  const SplatState s = carve_state((void*)state, n, channels, height, width);
  return launch_draw(n, height, width, channels, ranges, gsid, s, tau_init, out, contrib,
                     final_tau, ST(stream));
}

GSB_API int gsb_splat_backward(int64_t n, int height, int width, int channels, const float* us,
                               const float* cinv2ds, const float* alphas, const void* feats,
                               int feat_dtype, const int32_t* ranges, const int32_t* gsid,
                               const int32_t* contrib, const float* final_tau,
                               const float* dloss_dout, const float* dloss_dtau, void* state,
                               float* dfeats, float* dalphas, float* dus, float* dcinv2ds,
                               void* stream) {
  int rc = check_image("splat_backward", n, height, width, channels);
  if (rc) return rc;
  GSB_CHECK_ARG(valid_dtype(feat_dtype), "splat_backward: unsupported feature dtype %d", feat_dtype);
  GSB_CHECK_ARG(state && ((uintptr_t)state & 255) == 0,
                "splat_backward: state must be 256-byte aligned");
  GSB_CHECK_ARG(ranges && contrib && final_tau && dloss_dout && dfeats, "splat_backward: null pointer");
  const bool geom = dalphas || dus || dcinv2ds;
  GSB_CHECK_ARG(!geom || (dalphas && dus && dcinv2ds),
                "splat_backward: pass all of dalphas/dus/dcinv2ds or none");
  GSB_CHECK_ARG(!dloss_dtau || geom, "splat_backward: dloss_dtau needs the geometry outputs");
  GSB_CHECK_ARG(n == 0 || (us && cinv2ds && alphas && feats), "splat_backward: null input");
  const SplatState s = carve_state(state, n, channels, height, width);
  rc = launch_pack(n, height, width, channels, us, cinv2ds, alphas, feats, feat_dtype, nullptr,
                   nullptr, false, s, ST(stream));
  if (rc) return rc;
  return launch_draw_backward(n, height, width, channels, ranges, gsid, s, contrib, final_tau,
                              dloss_dout, dloss_dtau, dfeats, dalphas, dus, dcinv2ds, ST(stream));
}

GSB_API int gsb_splat_backward_packed(int64_t n, int height, int width, int channels,
                                      const int32_t* ranges, const int32_t* gsid,
                                      const int32_t* contrib, const float* final_tau,
                                      const float* dloss_dout, const float* dloss_dtau,
                                      const void* state, float* dfeats, float* dalphas, float* dus,
                                      float* dcinv2ds, void* stream) {
  int rc = check_image("splat_backward_packed", n, height, width, channels);
  if (rc) return rc;
  GSB_CHECK_ARG(state && ranges && contrib && final_tau && dloss_dout && dfeats,
                "splat_backward_packed: null pointer");
  const bool geom = dalphas || dus || dcinv2ds;
  GSB_CHECK_ARG(!geom || (dalphas && dus && dcinv2ds),
                "splat_backward_packed: pass all of dalphas/dus/dcinv2ds or none");
  GSB_CHECK_ARG(!dloss_dtau || geom, "splat_backward_packed: dloss_dtau needs the geometry outputs");
  const SplatState s = carve_state((void*)state, n, channels, height, width);
  return launch_draw_backward(n, height, width, channels, ranges, gsid, s, contrib, final_tau,
                              dloss_dout, dloss_dtau, dfeats, dalphas, dus, dcinv2ds, ST(stream));
}

GSB_API int gsb_palette_l1(int K, int height, int width, const float* layer,
                           const float* palette, const float* target, float* image, float* loss,
                           float* dlayer, float* dpalette, void* stream) {
  GSB_CHECK_ARG(K >= 1 && K <= GSB_MAX_CHANNELS, "palette_l1: channels must be in [1, %d]",
                GSB_MAX_CHANNELS);
  GSB_CHECK_ARG(height >= 0 && width >= 0, "palette_l1: negative image size");
  GSB_CHECK_ARG(palette && loss, "palette_l1: null pointer");
  GSB_CHECK_ARG(((int64_t)height * width == 0) || (layer && target), "palette_l1: null input");
  return launch_palette_l1(K, height, width, layer, palette, target, image, loss, dlayer, dpalette,
                           ST(stream));
}

GSB_API int gsb_palette_l1_ssim(int K, int height, int width, const float* layer,
                                const float* palette, const float* target, float lambda_ssim,
                                float lambda_pos, float data_range, float* image, float* loss,
                                float* dlayer, float* dpalette, void* stream) {
  GSB_CHECK_ARG(K >= 1 && K <= GSB_MAX_CHANNELS, "palette_l1_ssim: channels must be in [1, %d]",
                GSB_MAX_CHANNELS);
  GSB_CHECK_ARG(palette || K == 3, "palette_l1_ssim: without a palette the image has 3 channels");
  GSB_CHECK_ARG(palette || !dpalette, "palette_l1_ssim: dpalette needs a palette");
  GSB_CHECK_ARG(height >= 0 && width >= 0, "palette_l1_ssim: negative image size");
  GSB_CHECK_ARG(loss, "palette_l1_ssim: null loss");
  GSB_CHECK_ARG(((int64_t)height * width == 0) || (layer && target),
                "palette_l1_ssim: null input");
  GSB_CHECK_ARG(std::isfinite(lambda_ssim) && std::isfinite(lambda_pos) &&
                    std::isfinite(data_range) && data_range > 0.f,
                "palette_l1_ssim: lambdas must be finite and data_range positive");
  return launch_palette_l1_ssim(K, height, width, layer, palette, target, lambda_ssim, lambda_pos,
                                data_range, image, loss, dlayer, dpalette, ST(stream));
}

GSB_API int gsb_palette_geo_loss(int chroma_count, int height, int width, const float* layer,
                                 const float* target, const float* chroma, int clamp, int kind,
                                 float lambda_pos, float* target_weights, float* loss,
                                 float* dlayer, float* dchroma, void* stream) {
  GSB_CHECK_ARG(chroma_count >= 2 && chroma_count <= GSB_MAX_CHANNELS - 2,
                "palette_geo_loss: chromatic palette size must be in [2, %d]",
                GSB_MAX_CHANNELS - 2);
  GSB_CHECK_ARG(height >= 0 && width >= 0, "palette_geo_loss: negative image size");
  GSB_CHECK_ARG(kind == GSB_LOSS_MSE || kind == GSB_LOSS_L1, "palette_geo_loss: bad loss kind");
  GSB_CHECK_ARG(chroma && loss, "palette_geo_loss: null pointer");
  GSB_CHECK_ARG(((int64_t)height * width == 0) || (layer && target),
                "palette_geo_loss: null input");
  return launch_palette_geo_loss(chroma_count, height, width, layer, target, chroma, clamp != 0,
                                 kind, lambda_pos, target_weights, loss, dlayer, dchroma,
                                 ST(stream));
}

// ------------------------------------------------------------- fused path
static int check_params(const char* op, int64_t n, const gsb_palette_params* p) {
  GSB_CHECK_ARG(p, "%s: null palette parameters", op);
  GSB_CHECK_ARG(p->mode == GSB_WEIGHTS_FULL || p->mode == GSB_WEIGHTS_LOWRANK, "%s: bad mode %d",
                op, p->mode);
  GSB_CHECK_ARG(valid_dtype(p->dtype), "%s: bad dtype %d", op, p->dtype);
  GSB_CHECK_ARG(p->K >= 1 && p->K <= GSB_MAX_CHANNELS, "%s: K must be in [1, %d]", op,
                GSB_MAX_CHANNELS);
  GSB_CHECK_ARG(n == 0 || p->w0, "%s: null weight parameters", op);
  if (p->mode == GSB_WEIGHTS_LOWRANK) {
    GSB_CHECK_ARG(p->P > 0 && p->Q > 0 && p->rank > 0 && (p->P * p->Q) % p->K == 0,
                  "%s: bad low-rank shape P=%d Q=%d rank=%d K=%d", op, p->P, p->Q, p->rank, p->K);
    GSB_CHECK_ARG(n == 0 || (p->A && p->B), "%s: null low-rank factors", op);
  }
  return GSB_OK;
}

static CamArgs cam_args(const gsb_camera* c) {
  CamArgs a;
  a.R = c->Rcw;
  a.t = c->tcw;
  a.c = c->twc;
  a.fx = c->fx;
  a.fy = c->fy;
  a.cx = c->cx;
  a.cy = c->cy;
  // tan of the half field of view, formed in FP32 as gsplatcu/gausplat.cu:357-358
  a.tanx = c->width / (2 * c->fx);
  a.tany = c->height / (2 * c->fy);
  return a;
}

GSB_API int gsb_render_preprocess(int64_t n, const gsb_camera* cam, const float* pws,
                                  const float* rots, const float* scales, const float* alphas,
                                  const gsb_palette_params* params, void* state,
                                  float* depths_out, void* stream) {
  GSB_CHECK_ARG(cam && cam->Rcw && cam->tcw && cam->twc, "render_preprocess: null camera");
  int rc = check_image("render_preprocess", n, cam->height, cam->width, params ? params->K : 1);
  if (rc) return rc;
  if ((rc = check_params("render_preprocess", n, params))) return rc;
  GSB_CHECK_ARG(state && ((uintptr_t)state & 255) == 0,
                "render_preprocess: state must be 256-byte aligned");
  GSB_CHECK_ARG(n == 0 || (pws && rots && scales && alphas), "render_preprocess: null input");
  const SplatState s =
      carve_state(state, n, params->palette ? 3 : params->K, cam->height, cam->width);
  FusedArgs f{};
  f.n = n;
  f.gx = (uint32_t)div_up(cam->width, kTile);
  f.gy = (uint32_t)div_up(cam->height, kTile);
  f.cam = cam_args(cam);
  f.pws = pws;
  f.rots = rots;
  f.scales = scales;
  f.alphas = alphas;
  f.w0 = params->w0;
  f.wa = params->A;
  f.wb = params->B;
  f.st = s;
  f.depths_out = depths_out;
  f.palette = params->palette;
  rc = launch_render(params->mode, params->dtype, params->K, params->P, params->Q, params->rank, f,
                     false, ST(stream));
  if (rc) return rc;
  return launch_count_scan(n, s, ST(stream), true);
}

GSB_API size_t gsb_render_backward_bytes(int64_t n, int K) {
  if (n < 0 || K < 1 || K > GSB_MAX_CHANNELS) return 0;
  return (size_t)n * (K + 5) * sizeof(float) + 256;
}

static int render_backward(int64_t n, const gsb_camera* cam, const float* pws, const float* rots,
                           const float* scales, const float* alphas,
                           const gsb_palette_params* params, const void* state,
                           const int32_t* ranges, const int32_t* gsid, const int32_t* contrib,
                           const float* final_tau, const float* dloss_dout,
                           const float* dloss_dtau, void* scratch, float* dpws, float* drots,
                           float* dscales, float* dalphas, float* dw0, float* dA, float* dB,
                           bool acc, void* stream) {
  GSB_CHECK_ARG(cam && cam->Rcw && cam->tcw && cam->twc, "render_backward: null camera");
  int rc = check_image("render_backward", n, cam->height, cam->width, params ? params->K : 1);
  if (rc) return rc;
  if ((rc = check_params("render_backward", n, params))) return rc;
  GSB_CHECK_ARG(state && ranges && contrib && final_tau && dloss_dout,
                "render_backward: null pointer");
  GSB_CHECK_ARG(n == 0 || (scratch && dw0 && pws && rots && scales && alphas),
                "render_backward: null input/output");
  GSB_CHECK_ARG(params->mode == GSB_WEIGHTS_FULL || n == 0 || (dA && dB),
                "render_backward: null low-rank gradient outputs");
  const bool geom = dpws || drots || dscales || dalphas;
  GSB_CHECK_ARG(!geom || (dpws && drots && dscales && dalphas),
                "render_backward: pass all of dpws, drots, dscales, dalphas or none");
  GSB_CHECK_ARG(!params->palette, "render_backward: the palette-colour render has no adjoint here");
  const int K = params->K;
  const SplatState s = carve_state((void*)state, n, K, cam->height, cam->width);
  float* g_feat = (float*)scratch;
  float* g_u = g_feat + (size_t)n * K;
  float* g_conic = g_u + (size_t)n * 2;
  // (accumulating: dalphas keeps the previous views' sum; the adjoint adds to it)
  if (n > 0 && (rc = launch_zero2(scratch, n * (geom ? K + 5 : K),
                                  geom && !acc ? dalphas : nullptr, geom && !acc ? n : 0,
                                  ST(stream))))
    return rc;
  rc = launch_draw_backward(n, cam->height, cam->width, K, ranges, gsid, s, contrib, final_tau,
                            dloss_dout, geom ? dloss_dtau : nullptr, g_feat,
                            geom ? dalphas : nullptr, geom ? g_u : nullptr,
                            geom ? g_conic : nullptr, ST(stream));
  if (rc) return rc;
  FusedArgs f{};
  f.n = n;
  f.cam = cam_args(cam);
  f.pws = pws;
  f.rots = rots;
  f.scales = scales;
  f.alphas = alphas;
  f.w0 = params->w0;
  f.wa = params->A;
  f.wb = params->B;
  f.g_feat = g_feat;
  f.g_u = geom ? g_u : nullptr;
  f.g_conic = geom ? g_conic : nullptr;
  f.d_pws = dpws;
  f.d_rots = drots;
  f.d_scales = dscales;
  f.d_w0 = dw0;
  f.d_wa = dA;
  f.d_wb = dB;
  f.accumulate = acc;
  return launch_render(params->mode, params->dtype, K, params->P, params->Q, params->rank, f, true,
                       ST(stream));
}

GSB_API size_t gsb_draw_batch_bytes(int max_jobs) { return draw_queue_bytes(max_jobs); }

GSB_API int gsb_draw_batch_pack(const gsb_draw_job* jobs, int njobs, void* host_table,
                                size_t table_bytes) {
  GSB_CHECK_ARG(njobs >= 0 && (njobs == 0 || jobs) && host_table, "draw_batch_pack: null pointer");
  for (int i = 0; i < njobs; ++i) {
    const gsb_draw_job& j = jobs[i];
    int rc = check_image("draw_batch_pack", j.n, j.height, j.width, j.channels);
    if (rc) return rc;
    GSB_CHECK_ARG(j.channels == jobs[0].channels, "draw_batch_pack: job %d has %d channels, job 0 %d",
                  i, j.channels, jobs[0].channels);
    GSB_CHECK_ARG(j.state && ((uintptr_t)j.state & 255) == 0 && j.ranges && j.out && j.contrib &&
                      j.final_tau,
                  "draw_batch_pack: job %d: null or misaligned pointer", i);
  }
  const int rc = draw_queue_pack(jobs, njobs, host_table, table_bytes);
  if (rc) set_error("draw_batch_pack: %d jobs need %zu table bytes, %zu given", njobs,
                    draw_queue_bytes(njobs), table_bytes);
  return rc;
}

GSB_API int gsb_draw_batch(const void* dev_table, int channels, void* stream) {
  GSB_CHECK_ARG(dev_table && ((uintptr_t)dev_table & 15) == 0,
                "draw_batch: table must be a 16-byte aligned device buffer");
  GSB_CHECK_ARG(channels >= 1 && channels <= GSB_MAX_CHANNELS, "draw_batch: bad channel count");
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return check_launch("draw_batch (device query)", 0);
  return launch_draw_queue(channels, dev_table, 4 * sms, ST(stream));
}

GSB_API int gsb_palette_weights_backward(int64_t n, const gsb_camera* cam, const float* pws,
                                         const gsb_palette_params* params,
                                         const float* dloss_dweights, float* dw0, float* dA,
                                         float* dB, void* stream) {
  GSB_CHECK_ARG(cam && cam->twc, "palette_weights_backward: null camera");
  GSB_CHECK_ARG(n >= 0, "palette_weights_backward: n < 0");
  int rc = check_params("palette_weights_backward", n, params);
  if (rc) return rc;
  GSB_CHECK_ARG(!params->palette, "palette_weights_backward: palette-colour parameters have no adjoint here");
  GSB_CHECK_ARG(n == 0 || (pws && dloss_dweights && dw0), "palette_weights_backward: null pointer");
  GSB_CHECK_ARG(params->mode == GSB_WEIGHTS_FULL || n == 0 || (dA && dB),
                "palette_weights_backward: null low-rank gradient outputs");
  if (n == 0) return GSB_OK;
  FusedArgs f{};
  f.n = n;
  f.cam = cam_args(cam);
  f.pws = pws;
  f.w0 = params->w0;
  f.wa = params->A;
  f.wb = params->B;
  f.g_feat = dloss_dweights;  // g_u null: the weights-only chain
  f.d_w0 = dw0;
  f.d_wa = dA;
  f.d_wb = dB;
  return launch_render(params->mode, params->dtype, params->K, params->P, params->Q, params->rank,
                       f, true, ST(stream));
}

GSB_API int gsb_render_backward(int64_t n, const gsb_camera* cam, const float* pws,
                                const float* rots, const float* scales, const float* alphas,
                                const gsb_palette_params* params, const void* state,
                                const int32_t* ranges, const int32_t* gsid,
                                const int32_t* contrib, const float* final_tau,
                                const float* dloss_dout, const float* dloss_dtau, void* scratch,
                                float* dpws, float* drots, float* dscales, float* dalphas,
                                float* dw0, float* dA, float* dB, void* stream) {
  return render_backward(n, cam, pws, rots, scales, alphas, params, state, ranges, gsid, contrib,
                         final_tau, dloss_dout, dloss_dtau, scratch, dpws, drots, dscales, dalphas,
                         dw0, dA, dB, false, stream);
}

GSB_API int gsb_render_backward_accumulate(
    int64_t n, const gsb_camera* cam, const float* pws, const float* rots, const float* scales,
    const float* alphas, const gsb_palette_params* params, const void* state,
    const int32_t* ranges, const int32_t* gsid, const int32_t* contrib, const float* final_tau,
    const float* dloss_dout, const float* dloss_dtau, void* scratch, float* dpws, float* drots,
    float* dscales, float* dalphas, float* dw0, float* dA, float* dB, void* stream) {
  return render_backward(n, cam, pws, rots, scales, alphas, params, state, ranges, gsid, contrib,
                         final_tau, dloss_dout, dloss_dtau, scratch, dpws, drots, dscales, dalphas,
                         dw0, dA, dB, true, stream);
}
