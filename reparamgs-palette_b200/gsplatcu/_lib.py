"""ctypes binding of libgsplat_b200.so (the C ABI declared in include/gsplat_b200.h).

The library is loaded from this directory.  There is no fallback: if it is
missing or CUDA is unavailable, every operator raises instead of computing
anything another way.
"""
import contextlib
import ctypes as C
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgsplat_b200.so")

GSB_OK = 0
GSB_ERR_INVALID_ARGUMENT = 1
GSB_ERR_CUDA = 2
GSB_ERR_UNSUPPORTED = 3
GSB_ERR_CAPACITY = 4
GSB_ERR_DEVICE_TIMEOUT = 5
STATUS_BULK_TIMEOUT = 1
STATUS_PATCH_OVERFLOW = 2
STATUS_DEPTH_KEY_OVERFLOW = 4
DTYPE_F32 = 0
DTYPE_BF16 = 1
MAX_CHANNELS = 8
WEIGHTS_FULL = 0
LOSS_MSE = 0
LOSS_L1 = 1
WEIGHTS_LOWRANK = 1

_i64, _i32, _u32, _f32, _p, _sz = C.c_int64, C.c_int, C.c_uint32, C.c_float, C.c_void_p, C.c_size_t

# name -> (restype, argtypes)
_SIGS = {
    "gsb_last_error": (C.c_char_p, []),
    "gsb_version": (_i32, []),
    "gsb_launch_count": (C.c_ulonglong, []),
    "gsb_device_status": (_i32, [_p, _i32, _p]),
    "gsb_device_status_fetch": (_i32, [_p, _p]),
    "gsb_debug_expire_bulk_wait": (_i32, [_u32, _p]),
    "gsb_project": (_i32, [_i64, _p, _p, _p, _f32, _f32, _f32, _f32, _p, _p, _p, _p, _p]),
    "gsb_compute_cov3d": (_i32, [_i64, _p, _p, _p, _p, _p, _p, _p]),
    "gsb_compute_cov2d": (_i32, [_i64, _p, _p, _p, _p, _f32, _f32, _f32, _f32, _p, _p, _p, _p]),
    "gsb_inverse_cov2d": (_i32, [_i64, _p, _p, _p, _p, _p, _p]),
    "gsb_sh2weight": (_i32, [_i64, _p, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p]),
    "gsb_sh2weight_fast": (_i32, [_i64, _p, _p, _p, _i32, _i32, _i32, _i32, _i32, _p, _p, _p, _p,
                                  _p, _p]),
    "gsb_sh2weight_fast_backward": (_i32, [_i64, _p, _p, _i32, _p, _p, _i32, _i32, _i32, _i32,
                                           _p, _p, _p]),
    "gsb_sh2color": (_i32, [_i64, _p, _i32, _i32, _p, _p, _p, _p, _p, _p]),
    "gsb_lab2rgb": (_i32, [_i32, _i32, _p, _p, _p]),
    "gsb_splat_state_bytes": (_sz, [_i64, _i32, _i32, _i32]),
    "gsb_splat_pack": (_i32, [_i64, _i32, _i32, _i32, _p, _p, _p, _p, _i32, _p, _p, _p, _p]),
    "gsb_splat_counts": (_i32, [_i64, _i32, _i32, _p, _p, _p]),
    "gsb_splat_sort_bytes": (_sz, [_i64, _i32, _i32, _p]),
    "gsb_splat_sort": (_i32, [_i64, _i32, _i32, _p, _p, _p, _p, _p, _p]),
    "gsb_splat_sort_capacity_bytes": (_sz, [_i64, _i32, _i32, _i64, _u32]),
    "gsb_splat_sort_capacity": (_i32, [_i64, _i32, _i32, _i64, _u32, _p, _p, _p, _p, _p, _p]),
    "gsb_splat_patch_status": (_i32, [_i64, _i32, _i32, _i64, _u32, _p, _p, _p]),
    "gsb_splat_sort_static_max_bytes": (_sz, []),
    "gsb_splat_sort_static": (_i32, [_i64, _i32, _i32, _p, _p, _p, _p, _p]),
    "gsb_splat_draw": (_i32, [_i64, _i32, _i32, _i32, _p, _p, _p, _f32, _p, _p, _p, _p]),
    "gsb_splat_backward": (_i32, [_i64, _i32, _i32, _i32, _p, _p, _p, _p, _i32, _p, _p, _p, _p,
                                  _p, _p, _p, _p, _p, _p, _p, _p]),
    "gsb_palette_l1": (_i32, [_i32, _i32, _i32, _p, _p, _p, _p, _p, _p, _p, _p]),
    "gsb_palette_geo_loss": (_i32, [_i32, _i32, _i32, _p, _p, _p, _i32, _i32, _f32, _p, _p, _p,
                                    _p, _p]),
    "gsb_palette_l1_ssim": (_i32, [_i32, _i32, _i32, _p, _p, _p, _f32, _f32, _f32, _p, _p, _p, _p,
                                   _p]),
    "gsb_splat_backward_packed": (_i32, [_i64, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p, _p, _p,
                                         _p, _p, _p, _p]),
    "gsb_render_preprocess": (_i32, [_i64, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "gsb_render_backward_bytes": (_sz, [_i64, _i32]),
    "gsb_palette_weights_backward": (_i32, [_i64, _p, _p, _p, _p, _p, _p, _p, _p]),
    "gsb_draw_batch_bytes": (_sz, [_i32]),
    "gsb_draw_batch_pack": (_i32, [_p, _i32, _p, _sz]),
    "gsb_draw_batch": (_i32, [_p, _i32, _p]),
    "gsb_render_backward": (_i32, [_i64, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p,
                                   _p, _p, _p, _p, _p, _p, _p, _p]),
    "gsb_render_backward_accumulate": (_i32, [_i64, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p,
                                              _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
}

_lib = None


class SplatPlan(C.Structure):
    """gsb_splat_plan: sizes gsb_splat_counts reads back for the sort step."""
    _fields_ = [("patches", C.c_int64), ("max_depth_key", C.c_uint32),
                ("reserved", C.c_uint32)]


class Camera(C.Structure):
    """gsb_camera: device pointers to Rcw [3,3], tcw [3], twc [3]; intrinsics."""
    _fields_ = [("Rcw", C.c_void_p), ("tcw", C.c_void_p), ("twc", C.c_void_p),
                ("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("width", C.c_int), ("height", C.c_int)]


class PaletteParams(C.Structure):
    """gsb_palette_params: weight mode, storage dtype, shape and device pointers."""
    _fields_ = [("mode", C.c_int), ("dtype", C.c_int), ("K", C.c_int), ("P", C.c_int),
                ("Q", C.c_int), ("rank", C.c_int), ("w0", C.c_void_p), ("A", C.c_void_p),
                ("B", C.c_void_p), ("palette", C.c_void_p)]


class DrawJob(C.Structure):
    """gsb_draw_job: one image of a batched compositing launch."""
    _fields_ = [("state", C.c_void_p), ("n", C.c_int64), ("height", C.c_int),
                ("width", C.c_int), ("channels", C.c_int), ("ranges", C.c_void_p),
                ("gsid", C.c_void_p), ("tau_init", C.c_float), ("out", C.c_void_p),
                ("contrib", C.c_void_p), ("final_tau", C.c_void_p)]


class GsplatError(RuntimeError):
    """A CUDA-side failure reported by libgsplat_b200; ``status`` is the
    library's status code (GSB_ERR_*)."""

    def __init__(self, msg, status=GSB_ERR_CUDA):
        super().__init__(msg)
        self.status = status


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libgsplat_b200.so not found at {LIB_PATH}; build it with "
                "`python reparamgs-palette_b200/build.py` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return sorted(_SIGS)


_FN = {}


def call(op, name, *args):
    """Invoke C entry `name`; raise with the library's message on failure."""
    f = _FN.get(name)
    if f is None:
        f = _FN[name] = getattr(lib(), name)
    rc = f(*args)
    if rc != GSB_OK:
        msg = (lib().gsb_last_error() or b"").decode(errors="replace")
        if rc == GSB_ERR_INVALID_ARGUMENT:
            raise ValueError(f"gsplatcu.{op}: {msg}")
        raise GsplatError(f"gsplatcu.{op}: {msg} (status {rc})", rc)


def ptr(t):
    """Device address of `t` as an int (ctypes passes it as void*), or None."""
    return None if t is None else t.data_ptr()


# torch's raw current-stream query returns the cudaStream_t as an int without
# building a Stream object (a few microseconds per operator call otherwise)
_RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def stream_of(t):
    """The current CUDA stream of `t`'s device, as an int handle."""
    if _RAW_STREAM is not None:
        return _RAW_STREAM(t.device.index)
    return torch.cuda.current_stream(t.device).cuda_stream


_CUR_DEV = getattr(torch._C, "_cuda_getDevice", None) or torch.cuda.current_device


def on_device(dev):
    """``torch.cuda.device(dev)`` when `dev` is not already the current device;
    a no-op context otherwise (the switch costs a few microseconds per call)."""
    return contextlib.nullcontext() if dev.index == _CUR_DEV() else torch.cuda.device(dev)


def mapped_address(host):
    """Device address of a pinned host tensor, or None when the runtime does
    not map it into the device's address space."""
    try:
        from cuda.bindings import runtime as rt
        err, dptr = rt.cudaHostGetDevicePointer(host.data_ptr(), 0)
        if err == rt.cudaError_t.cudaSuccess:
            return int(dptr)
        rt.cudaGetLastError()  # a refused query must not surface at the next launch check
    except Exception:
        pass
    return None


# ------------------------------------------------- bounded device waits
# Kernels that stage through bulk copies wait on them a bounded number of
# times; when a wait runs out the kernel sets a device status bit and returns
# without its results.  After every call that launches such kernels the
# operators enqueue gsb_device_status_fetch into a pinned host word of the
# calling thread; wherever the host waits for the stream anyway (the patch
# count read-back of splat_weight / render_palette, check_device_status) the
# word is read and a set bit raises GsplatError(GSB_ERR_DEVICE_TIMEOUT).
_TIMEOUT_WORDS = {}


def _timeout_word(dev):
    key = (dev.index, threading.get_ident())
    w = _TIMEOUT_WORDS.get(key)
    if w is None:
        host = torch.zeros((1,), dtype=torch.int32, pin_memory=True)
        addr = mapped_address(host)
        dword = None if addr is not None else torch.zeros((1,), dtype=torch.int32, device=dev)
        w = _TIMEOUT_WORDS[key] = (host, addr, dword)
    return w


def fetch_device_status(dev, stream):
    """Enqueue, on `stream` (an int handle or a c_void_p), the copy of the
    device status bits into this thread's host word for `dev`."""
    host, addr, dword = _timeout_word(dev)
    if addr is not None:
        call("device_status_fetch", "gsb_device_status_fetch", addr, stream)
    else:
        call("device_status_fetch", "gsb_device_status_fetch", ptr(dword), stream)
        handle = stream.value if isinstance(stream, C.c_void_p) else stream
        with torch.cuda.stream(torch.cuda.ExternalStream(handle or 0, device=dev)):
            host.copy_(dword, non_blocking=True)


def raise_if_timed_out(dev, op):
    """Call once the stream has passed the fetches of interest: raises
    GsplatError(GSB_ERR_DEVICE_TIMEOUT) if a bounded wait expired (and
    clears the bits, so that later calls start clean)."""
    w = _TIMEOUT_WORDS.get((dev.index, threading.get_ident()))
    if w is None or int(w[0][0]) == 0:
        return
    bits = int(w[0][0])
    # clear the device bits (this synchronises the stream, so fetches enqueued
    # before it -- which may still OR the old bits into the host word -- have
    # run), then the host word
    cleared = C.c_uint32(0)
    with torch.cuda.device(dev):
        call("device_status", "gsb_device_status", C.byref(cleared), 1,
             C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    w[0].zero_()
    if w[2] is not None:
        w[2].zero_()
    raise GsplatError(
        f"gsplatcu.{op}: a bounded device-side wait for a bulk copy ran out (status bits "
        f"{bits:#x}); the results of the calls since the last check are incomplete "
        f"(status {GSB_ERR_DEVICE_TIMEOUT})", GSB_ERR_DEVICE_TIMEOUT)
