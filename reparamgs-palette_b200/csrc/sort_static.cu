// gsb_splat_sort_static: the tile sort of gsb_splat_sort with its temporary
// storage in this library's own device memory instead of a caller-supplied
// workspace.
//
// Some callers cannot allocate device memory at the point where they render:
// a host whose device memory is owned by another runtime's pool (and must
// not be fragmented or grown behind that pool's back), a plug-in that is
// handed its input and output buffers and nothing else, or a process that
// fixes its device footprint at start-up.  For them the sort keeps its
// keys, values and digit histograms in one file-scope device array of
// kStaticSortBytes bytes.  Every GPU that loads this library reserves that
// array when the library's device code is loaded and keeps it until the
// process exits, whether or not this entry point is ever called.
//
// The array is shared by every call on a device and keeps whatever the last
// call left in it.  Nothing in it has to start at zero: each call writes
// every byte it later reads (emission writes the keys and values, the
// upsweep every histogram entry, the scan every digit total).  Two calls
// that overlap on the GPU -- on different streams, or from different host
// threads without ordering -- use the same bytes and race; order them on one
// stream or with events.
#include <cuda.h>  // CUcontext / CUresult types only: the two driver calls below are
                   // resolved at run time through the runtime's entry-point query
#include <mutex>

#include "gsb_common.cuh"
#include "gsb_internal.h"

namespace gsb {

// 32 MiB: about 2.0M patches with 32-bit keys, 1.3M with 64-bit keys.
constexpr size_t kStaticSortBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_sort_scratch[kStaticSortBytes];

// Host code may not take the address of g_sort_scratch (that would be a
// host-side stand-in, not device memory); the device address comes from
// cudaGetSymbolAddress, with the device current.  It is looked up once per
// device and CUDA context: the cache is keyed by the context's process-unique
// id (cuCtxGetId), so after a device reset or a re-created primary context
// the next call looks the address up again instead of reusing a stale one.
constexpr int kMaxStaticDevices = 64;
struct ScratchEntry {
  unsigned long long ctx_id;
  void* addr;
};
static ScratchEntry g_scratch[kMaxStaticDevices];
static std::mutex g_scratch_mutex;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

}  // namespace gsb

namespace gsb {

// Process-unique id of the calling thread's current context (0 if unknown).
// Callers hold their own lock; the one-time resolution of the two driver
// entry points is guarded here.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  static std::mutex resolve_mutex;
  std::lock_guard<std::mutex> guard(resolve_mutex);
  if (!resolved) {
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q1) !=
            cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess)
      get_current = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q2) !=
            cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess)
      get_id = nullptr;
    (void)cudaGetLastError();
    resolved = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx ||
      get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

static int static_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("splat_sort_static (device)", 0);
  if (dev < 0 || dev >= kMaxStaticDevices) {
    set_error("splat_sort_static: device %d beyond the %d supported", dev, kMaxStaticDevices);
    return GSB_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  // (no context current yet: id 0, the address is looked up, which makes the
  // device's primary context current for the launch)
  const unsigned long long ctx = current_context_id();
  ScratchEntry& e = g_scratch[dev];
  if (!e.addr || ctx == 0 || e.ctx_id != ctx) {
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (err != cudaSuccess || !p) {
      (void)cudaGetLastError();
      set_error("splat_sort_static: cudaGetSymbolAddress failed on device %d: %s", dev,
                cudaGetErrorString(err));
      return GSB_ERR_CUDA;
    }
    e.addr = p;
    e.ctx_id = ctx;
  }
  *out = e.addr;
  return GSB_OK;
}

}  // namespace gsb

using namespace gsb;

extern "C" __attribute__((visibility("default"))) size_t gsb_splat_sort_static_max_bytes(void) {
  return kStaticSortBytes;
}

extern "C" __attribute__((visibility("default"))) int gsb_splat_sort_static(
    int64_t n, int height, int width, const gsb_splat_plan* plan, const void* state,
    int32_t* gsid_out, int32_t* ranges_out, void* stream) {
  GSB_CHECK_ARG(n >= 0 && n < (int64_t)INT32_MAX, "splat_sort_static: Gaussian count %lld out of range",
                (long long)n);
  GSB_CHECK_ARG(height >= 0 && width >= 0, "splat_sort_static: negative image size");
  GSB_CHECK_ARG((int64_t)div_up(width, kTile) < 65536 && (int64_t)div_up(height, kTile) < 65536,
                "splat_sort_static: image too large (%d x %d)", width, height);
  GSB_CHECK_ARG(plan && plan->patches >= 0 && plan->patches < (int64_t)INT32_MAX,
                "splat_sort_static: bad plan");
  GSB_CHECK_ARG(state && ranges_out, "splat_sort_static: null pointer");
  GSB_CHECK_ARG(plan->patches == 0 || gsid_out, "splat_sort_static: null output");
  const SortPlan p = make_sort_plan(n, height, width, plan->patches, plan->max_depth_key);
  if (p.bytes_total > kStaticSortBytes) {
    set_error("splat_sort_static: %lld patches need %zu bytes of sort scratch, above the "
              "built-in %zu bytes; use gsb_splat_sort with a caller workspace",
              (long long)plan->patches, p.bytes_total, kStaticSortBytes);
    return GSB_ERR_CAPACITY;
  }
  void* ws = nullptr;
  const int rc = static_scratch(&ws);
  if (rc) return rc;
  const SplatState s = carve_state((void*)state, n, 1, height, width);
  return launch_sort(p, n, height, width, s, ws, gsid_out, ranges_out, (cudaStream_t)stream);
}
