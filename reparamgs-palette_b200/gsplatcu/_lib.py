"""ctypes binding of libgsplat_b200.so (the C ABI declared in include/gsplat_b200.h).

The library is loaded from this directory.  There is no fallback: if it is
missing or CUDA is unavailable, every operator raises instead of computing
anything another way.
"""
import ctypes as C
import os

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


class GsplatError(RuntimeError):
    """A CUDA-side failure reported by libgsplat_b200."""


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


def call(op, name, *args):
    """Invoke C entry `name`; raise with the library's message on failure."""
    rc = getattr(lib(), name)(*args)
    if rc != GSB_OK:
        msg = (lib().gsb_last_error() or b"").decode(errors="replace")
        if rc == GSB_ERR_INVALID_ARGUMENT:
            raise ValueError(f"gsplatcu.{op}: {msg}")
        raise GsplatError(f"gsplatcu.{op}: {msg} (status {rc})")


def ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def stream_of(t):
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)
