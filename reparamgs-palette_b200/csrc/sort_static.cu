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
#include <mutex>

#include "gsb_common.cuh"
#include "gsb_internal.h"

namespace gsb {

// 32 MiB: about 2.0M patches with 32-bit keys, 1.3M with 64-bit keys.
constexpr size_t kStaticSortBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_sort_scratch[kStaticSortBytes];

// Host code may not take the address of g_sort_scratch (that would be a
// host-side stand-in, not device memory); the device address comes from
// cudaGetSymbolAddress, once per device, with that device current.
constexpr int kMaxStaticDevices = 64;
static void* g_scratch_addr[kMaxStaticDevices];
static std::mutex g_scratch_mutex;

static int static_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("splat_sort_static (device)", 0);
  if (dev < 0 || dev >= kMaxStaticDevices) {
    set_error("splat_sort_static: device %d beyond the %d supported", dev, kMaxStaticDevices);
    return GSB_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess || !p) {
      (void)cudaGetLastError();
      set_error("splat_sort_static: cudaGetSymbolAddress failed on device %d: %s", dev,
                cudaGetErrorString(e));
      return GSB_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
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
