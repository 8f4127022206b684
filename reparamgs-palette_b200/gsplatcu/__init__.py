"""Drop-in replacement for the reference ``gsplatcu`` extension (ReparamGS-Palette).

``import gsplatcu as gsc`` resolves to this package when
``reparamgs-palette_b200/`` is on ``sys.path``.  It exports the reference's
13 operators with the same names, positional signatures, output lists, output
shapes/dtypes and in-place side effects (gsplatcu/ext.cpp:125-139), backed by
hand-written sm_100a kernels in ``libgsplat_b200.so``.  Differences from the
reference are additions only:

* ``sh2Weight_fast`` / ``sh2Weight_fast_B`` also accept rank-r factors
  ``shs_A [N,P,r]``, ``shs_B [N,r,Q]`` (2-D inputs are the reference's rank 1);
* SH / weight / factor tensors may be bfloat16 (FP32 accumulation);
* ``splat_color_B`` / ``splat_weight_B`` accept an optional
  ``dloss_dfinal_tau`` keyword (the final-transmittance adjoint);
* ``splat_weight_B_full`` returns the opacity / centre / conic adjoint too;
* calc_J=False is accepted by ``sh2Weight_fast`` (the reference writes through
  null pointers there).

Errors raise ValueError (bad arguments) or ``GsplatError``; the reference
printed CUDA errors and continued.  Every operator runs on the current
torch CUDA stream without device synchronisation, except ``splat_weight`` /
``splat_color``, which read the patch count back to size their outputs (as the
reference does).
"""
import collections
import ctypes as C
import threading

import torch

from . import _lib
from ._lib import GsplatError, call, on_device, ptr, stream_of

__all__ = [
    "project", "computeCov3D", "computeCov2D", "inverseCov2D", "sh2Weight", "sh2Weight_fast",
    "sh2Weight_fast_B", "sh2Color", "splat_weight", "splat_weight_B", "splat_color",
    "splat_color_B", "lab2rgb", "splat_weight_B_full", "GsplatError", "check_device_status",
]

TILE = 16
_F32 = torch.float32


# ------------------------------------------------------------------ helpers
def _cuda(op, name, t, dtypes=(_F32,)):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"gsplatcu.{op}: {name} must be a torch.Tensor")
    if not t.is_cuda:
        raise ValueError(f"gsplatcu.{op}: {name} must be a CUDA tensor (no CPU path exists)")
    if t.dtype not in dtypes:
        raise TypeError(f"gsplatcu.{op}: {name} must have dtype in {[str(d) for d in dtypes]}, "
                        f"got {t.dtype}")
    return t.contiguous()


def _inplace(op, name, t, dtype):
    """Tensor the kernel updates in place.  Like the reference, which writes
    through ``t.contiguous().data_ptr()``, a non-contiguous input is updated in
    a private copy (the caller's tensor is left unchanged)."""
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype):
        raise TypeError(f"gsplatcu.{op}: {name} must be a CUDA {dtype} tensor")
    return t.contiguous()


def _sh_dtype(t):
    return _lib.DTYPE_BF16 if t.dtype == torch.bfloat16 else _lib.DTYPE_F32


def _n(t):
    return int(t.shape[0])


def _empty(shape, like, dtype=_F32):
    return torch.empty(shape, dtype=dtype, device=like.device)


def _grid(H, W):
    return (W + TILE - 1) // TILE, (H + TILE - 1) // TILE


# ---------------------------------------------------------------- geometry
def project(pws, Rcw, tcw, focal_x, focal_y, center_x, center_y, calc_J):
    """gsplatcu/gausplat.cu:381-419 -> [us [N,2], pcs [N,3], depths [N], (du_dpcs [N,2,3])]."""
    op = "project"
    pws, Rcw, tcw = (_cuda(op, k, v) for k, v in (("pws", pws), ("Rcw", Rcw), ("tcw", tcw)))
    n = _n(pws)
    us, pcs, depths = _empty((n, 2), pws), _empty((n, 3), pws), _empty((n,), pws)
    du = _empty((n, 2, 3), pws) if calc_J else None
    with on_device(pws.device):
        call(op, "gsb_project", n, ptr(pws), ptr(Rcw), ptr(tcw), float(focal_x), float(focal_y),
             float(center_x), float(center_y), ptr(us), ptr(pcs), ptr(depths), ptr(du),
             stream_of(pws))
    return [us, pcs, depths, du] if calc_J else [us, pcs, depths]


def computeCov3D(rots, scales, depths, calc_J):
    """gsplatcu/gausplat.cu:298-331 -> [cov3ds [N,6], (dcov3d_drots [N,6,4], dcov3d_dscales [N,6,3])]."""
    op = "computeCov3D"
    rots, scales, depths = (_cuda(op, k, v) for k, v in
                            (("rots", rots), ("scales", scales), ("depths", depths)))
    n = _n(rots)
    cov = _empty((n, 6), rots)
    dq = _empty((n, 6, 4), rots) if calc_J else None
    ds = _empty((n, 6, 3), rots) if calc_J else None
    with on_device(rots.device):
        call(op, "gsb_compute_cov3d", n, ptr(rots), ptr(scales), ptr(depths), ptr(cov), ptr(dq),
             ptr(ds), stream_of(rots))
    return [cov, dq, ds] if calc_J else [cov]


def computeCov2D(cov3ds, pcs, Rcw, depths, focal_x, focal_y, width, height, calc_J):
    """gsplatcu/gausplat.cu:333-379 -> [cov2ds [N,3], (dcov2d_dcov3ds [N,3,6], dcov2d_dpcs [N,3,3])]."""
    op = "computeCov2D"
    cov3ds, pcs, Rcw, depths = (_cuda(op, k, v) for k, v in
                                (("cov3ds", cov3ds), ("pcs", pcs), ("Rcw", Rcw), ("depths", depths)))
    n = _n(pcs)
    out = _empty((n, 3), pcs)
    d3 = _empty((n, 3, 6), pcs) if calc_J else None
    dp = _empty((n, 3, 3), pcs) if calc_J else None
    with on_device(pcs.device):
        call(op, "gsb_compute_cov2d", n, ptr(cov3ds), ptr(pcs), ptr(Rcw), ptr(depths),
             float(focal_x), float(focal_y), float(width), float(height), ptr(out), ptr(d3),
             ptr(dp), stream_of(pcs))
    return [out, d3, dp] if calc_J else [out]


def inverseCov2D(cov2ds, depths, calc_J):
    """gsplatcu/gausplat.cu:590-617 -> [cinv2ds [N,3], areas int32 [N,2], (dcinv2d_dcov2ds [N,3,3])].
    Sets depths[i] = -1 in place where 1/det is NaN."""
    op = "inverseCov2D"
    cov2ds = _cuda(op, "cov2ds", cov2ds)
    depths = _inplace(op, "depths", depths, _F32)
    n = _n(cov2ds)
    cinv = _empty((n, 3), cov2ds)
    areas = _empty((n, 2), cov2ds, torch.int32)
    dc = _empty((n, 3, 3), cov2ds) if calc_J else None
    with on_device(cov2ds.device):
        call(op, "gsb_inverse_cov2d", n, ptr(cov2ds), ptr(depths), ptr(cinv), ptr(areas), ptr(dc),
             stream_of(cov2ds))
    return [cinv, areas, dc] if calc_J else [cinv, areas]


# ------------------------------------------------------ spherical harmonics
_SH_DTYPES = (torch.float32, torch.bfloat16)


def sh2Weight(shs, pws, twc, calc_J, num_palette):
    """gsplatcu/gausplat.cu:425-462 -> [weights [N,K], (dweight_dshs [N,1,nb], dweight_dpws [N,K,3])].
    shs [N, nb*K] band-major, nb = shs.shape[1] // K in {1,4,9,16}."""
    op = "sh2Weight"
    shs = _cuda(op, "shs", shs, _SH_DTYPES)
    pws, twc = _cuda(op, "pws", pws), _cuda(op, "twc", twc)
    K = int(num_palette)
    if K < 1 or K > _lib.MAX_CHANNELS:
        raise ValueError(f"gsplatcu.{op}: num_palette must be in [1, {_lib.MAX_CHANNELS}]")
    n = _n(pws)
    nb = int(shs.shape[1]) // K
    w = _empty((n, K), pws)
    dshs = _empty((n, 1, nb), pws) if calc_J else None
    dpws = _empty((n, K, 3), pws) if calc_J else None
    with on_device(pws.device):
        call(op, "gsb_sh2weight", n, ptr(shs), _sh_dtype(shs), nb, K, ptr(pws), ptr(twc), ptr(w),
             ptr(dshs), ptr(dpws), stream_of(pws))
    return [w, dshs, dpws] if calc_J else [w]


def sh2Color(shs, pws, twc, calc_J):
    """gsplatcu/gausplat.cu:551-584 -> [colors [N,3], (dcolor_dshs [N,1,nb], dcolor_dpws [N,3,3])]."""
    op = "sh2Color"
    shs = _cuda(op, "shs", shs, _SH_DTYPES)
    pws, twc = _cuda(op, "pws", pws), _cuda(op, "twc", twc)
    n = _n(pws)
    nb = int(shs.shape[1]) // 3
    col = _empty((n, 3), pws)
    dshs = _empty((n, 1, nb), pws) if calc_J else None
    dpws = _empty((n, 3, 3), pws) if calc_J else None
    with on_device(pws.device):
        call(op, "gsb_sh2color", n, ptr(shs), _sh_dtype(shs), nb, ptr(pws), ptr(twc), ptr(col),
             ptr(dshs), ptr(dpws), stream_of(pws))
    return [col, dshs, dpws] if calc_J else [col]


def _factor_dims(op, A, B, Q):
    if A.dim() == 2 and B.dim() == 2:
        P, rank = int(A.shape[1]), 1
        if int(B.shape[1]) != Q:
            raise ValueError(f"gsplatcu.{op}: shs_B must be [N, Q={Q}], got {tuple(B.shape)}")
    elif A.dim() == 3 and B.dim() == 3:
        P, rank = int(A.shape[1]), int(A.shape[2])
        if int(B.shape[1]) != rank or int(B.shape[2]) != Q:
            raise ValueError(f"gsplatcu.{op}: shs_B must be [N, {rank}, {Q}], got {tuple(B.shape)}")
    else:
        raise ValueError(f"gsplatcu.{op}: factors must be 2-D (rank 1) or 3-D (rank r)")
    return P, rank


def sh2Weight_fast(shs_dc, shs_A, shs_B, pws, twc, calc_J, num_palette, Q):
    """gsplatcu/gausplat.cu:469-509 (rank r) -> [weights [N,K], (dweight_ddc [N,K], Ylm [N,L])]."""
    op = "sh2Weight_fast"
    dc = _cuda(op, "shs_dc", shs_dc, _SH_DTYPES)
    A = _cuda(op, "shs_A", shs_A, _SH_DTYPES)
    B = _cuda(op, "shs_B", shs_B, _SH_DTYPES)
    if not (dc.dtype == A.dtype == B.dtype):
        raise TypeError(f"gsplatcu.{op}: shs_dc, shs_A and shs_B must share a dtype")
    pws, twc = _cuda(op, "pws", pws), _cuda(op, "twc", twc)
    K, Q = int(num_palette), int(Q)
    P, rank = _factor_dims(op, A, B, Q)
    n = _n(pws)
    L = P * Q // K if K > 0 else 0
    w = _empty((n, K), pws)
    ddc = _empty((n, K), pws) if calc_J else None
    ylm = _empty((n, L), pws) if calc_J else None
    with on_device(pws.device):
        st = stream_of(pws)
        call(op, "gsb_sh2weight_fast", n, ptr(dc), ptr(A), ptr(B), _sh_dtype(A), K, P, Q, rank,
             ptr(pws), ptr(twc), ptr(w), ptr(ddc), ptr(ylm), st)
        _lib.fetch_device_status(pws.device, st)
    return [w, ddc, ylm] if calc_J else [w]


def sh2Weight_fast_B(shs_A, shs_B, Ylm_stored, dloss_dw, num_palette, Q):
    """gsplatcu/gausplat.cu:512-541 (rank r) -> [dloss_dA (shape of A), dloss_dB (shape of B)]."""
    op = "sh2Weight_fast_B"
    A = _cuda(op, "shs_A", shs_A, _SH_DTYPES)
    B = _cuda(op, "shs_B", shs_B, _SH_DTYPES)
    ylm, dw = _cuda(op, "Ylm_stored", Ylm_stored), _cuda(op, "dloss_dw", dloss_dw)
    K, Q = int(num_palette), int(Q)
    P, rank = _factor_dims(op, A, B, Q)
    n = _n(A)
    if int(ylm.shape[1]) * K != P * Q:
        raise ValueError(f"gsplatcu.{op}: Ylm has {int(ylm.shape[1])} bands but P*Q/K = {P * Q // K}")
    dA, dB = _empty(tuple(A.shape), A), _empty(tuple(B.shape), A)
    with on_device(A.device):
        st = stream_of(A)
        call(op, "gsb_sh2weight_fast_backward", n, ptr(A), ptr(B), _sh_dtype(A), ptr(ylm), ptr(dw),
             K, P, Q, rank, ptr(dA), ptr(dB), st)
        _lib.fetch_device_status(A.device, st)
    return [dA, dB]


def check_device_status(device=None):
    """Wait for the current stream of `device` and raise
    ``GsplatError`` (``status == GSB_ERR_DEVICE_TIMEOUT``) if a bounded
    device-side wait of an earlier call on this thread ran out.  The forward
    operators check at their own patch-count read-back; call this after a
    backward pass or a batch of calls whose results are used without one."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else \
        torch.device(device)
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    torch.cuda.current_stream(dev).synchronize()
    _lib.raise_if_timed_out(dev, "check_device_status")


# --------------------------------------------------------------- splatting
# Per (Gaussian count, image size): patch capacity (1.25x the largest count
# seen, plus slack) and depth-key bound for the overlapped read-back below.
_CAPACITY = {}
_READBACK = {}


_mapped_address = _lib.mapped_address


def _readback_buffers(dev):
    """(device status words, pinned host words, event, device address of the
    host words or None) of the calling thread on `dev`.  With an address the
    status kernel writes the host words directly (no copy in the stream
    between it and the sort); the host words are read before the thread
    renders again."""
    key = (dev, threading.get_ident())
    b = _READBACK.get(key)
    if b is None:
        host = torch.empty((4,), dtype=torch.int32, pin_memory=True)
        b = (torch.empty((4,), dtype=torch.int32, device=dev), host, torch.cuda.Event(),
             _mapped_address(host))
        _READBACK[key] = b
    return b


def _sort_and_draw(op, n, H, W, C_, state, ranges, out, contrib, final_tau, tau_init, dev, st):
    """Tile sort and compositing of a packed `state`; returns the tile lists
    (gsid, exactly the patch count long).  The reference reads the patch
    count back before it sorts (gsplatcu/gausplat.cu:199-201), and so does
    the first render of each size here.  Later renders of that size enqueue
    the sort -- sized by the stored capacity -- and the compositing at once,
    and read the count back while they run; if the count or a depth key
    exceeded the capacity, those kernels left every range empty and the tile
    lists are sorted and composited again exactly (results identical)."""
    L = _lib.lib()
    key = (n, H, W)
    if key in _CAPACITY:
        cap, dkey = _CAPACITY[key]
        status, host, counted, mapped = _readback_buffers(dev)
        if mapped is not None:
            call(op, "gsb_splat_patch_status", n, H, W, cap, dkey, ptr(state), C.c_void_p(mapped),
                 st)
        else:
            call(op, "gsb_splat_patch_status", n, H, W, cap, dkey, ptr(state), ptr(status), st)
            host.copy_(status, non_blocking=True)
        counted.record(torch.cuda.current_stream(dev))
        ws = torch.empty(max(1, int(L.gsb_splat_sort_capacity_bytes(n, H, W, cap, dkey))),
                         dtype=torch.uint8, device=dev)
        full = torch.empty((max(1, cap),), dtype=torch.int32, device=dev)
        call(op, "gsb_splat_sort_capacity", n, H, W, cap, dkey, ptr(state), ptr(ws), ptr(full),
             ptr(ranges), None, st)  # (status read above)
        call(op, "gsb_splat_draw", n, H, W, C_, ptr(ranges), ptr(full), ptr(state),
             float(tau_init), ptr(out), ptr(contrib), ptr(final_tau), st)
        counted.synchronize()
        _lib.raise_if_timed_out(dev, op)
        if int(host[0]) == 0:
            return full[:int(host[1]) | (int(host[2]) << 32)]
    plan = _lib.SplatPlan()
    call(op, "gsb_splat_counts", n, H, W, ptr(state), C.byref(plan), st)
    _lib.raise_if_timed_out(dev, op)
    M = int(plan.patches)
    ws = torch.empty(max(1, int(L.gsb_splat_sort_bytes(n, H, W, C.byref(plan)))),
                     dtype=torch.uint8, device=dev)
    gsid = torch.empty((M,), dtype=torch.int32, device=dev)
    call(op, "gsb_splat_sort", n, H, W, C.byref(plan), ptr(state), ptr(ws), ptr(gsid), ptr(ranges),
         st)
    call(op, "gsb_splat_draw", n, H, W, C_, ptr(ranges), ptr(gsid), ptr(state), float(tau_init),
         ptr(out), ptr(contrib), ptr(final_tau), st)
    _CAPACITY[key] = (int(M * 1.25) + 4096, (1 << int(plan.max_depth_key).bit_length()) - 1)
    return gsid


def _splat_forward(op, H, W, C_, us, cinv2ds, alphas, depths, feats, areas, tau_init):
    us, cinv = _cuda(op, "us", us), _cuda(op, "cinv2ds", cinv2ds)
    alphas = _cuda(op, "alphas", alphas)
    feats = _cuda(op, "weights" if C_ != 3 or op == "splat_weight" else "colors", feats, _SH_DTYPES)
    depths = _inplace(op, "depths", depths, _F32)
    areas = _inplace(op, "areas", areas, torch.int32)
    H, W, n = int(H), int(W), _n(us)
    gx, gy = _grid(H, W)
    dev = us.device
    L = _lib.lib()
    with on_device(dev):
        st = stream_of(us)
        state = torch.empty(int(L.gsb_splat_state_bytes(n, C_, H, W)), dtype=torch.uint8,
                            device=dev)
        call(op, "gsb_splat_pack", n, H, W, C_, ptr(us), ptr(cinv), ptr(alphas), ptr(feats),
             _sh_dtype(feats), ptr(depths), ptr(areas), ptr(state), st)
        # outputs that do not depend on the patch count are allocated while the
        # device is still packing
        ranges = torch.empty((gx * gy, 2), dtype=torch.int32, device=dev)
        out = torch.empty((C_, H, W), dtype=_F32, device=dev)
        contrib = torch.empty((H, W), dtype=torch.int32, device=dev)
        final_tau = torch.empty((H, W), dtype=_F32, device=dev)
        gsid = _sort_and_draw(op, n, H, W, C_, state, ranges, out, contrib, final_tau, tau_init,
                              dev, st)
    _keep_packed(gsid, H, W, C_, state, us, cinv, alphas, feats)
    return [out, contrib, final_tau, ranges, gsid]


# The compositing records of the last two forward renders, keyed by their
# tile-list tensor.  The reference's backward is handed the forward's inputs and
# lists again and packs the records a second time; here the backward reuses the
# forward's records when every input is the same tensor, unmodified since (torch
# version counter).  An entry holds references to its tensors, so their memory
# cannot be recycled under the same address while it lives; the backward drops
# the entry it uses, and ``release_packed()`` drops all of them.
_PACKED = collections.OrderedDict()
_PACKED_MAX = 2
_PACKED_LOCK = threading.Lock()


def _signature(ts):
    return tuple((t.data_ptr(), t._version, tuple(t.shape), t.dtype) for t in ts)


def _keep_packed(gsid, H, W, C_, state, *inputs):
    key = (gsid.data_ptr(), gsid.numel(), H, W, C_)
    ts = (gsid,) + inputs
    with _PACKED_LOCK:
        _PACKED[key] = (state, ts, _signature(ts))
        _PACKED.move_to_end(key)
        while len(_PACKED) > _PACKED_MAX:
            _PACKED.popitem(last=False)


def _take_packed(gsid, H, W, C_, *inputs):
    with _PACKED_LOCK:
        e = _PACKED.pop((gsid.data_ptr(), gsid.numel(), H, W, C_), None)
    return e[0] if e is not None and e[2] == _signature((gsid,) + inputs) else None


def release_packed():
    """Drop the forward records kept for the next backward (frees their HBM)."""
    with _PACKED_LOCK:
        _PACKED.clear()


def splat_weight(height, width, num_palette, us, cinv2ds, alphas, depths, weights, areas):
    """gsplatcu/gausplat.cu:161-249 -> [layer [K,H,W], contrib int32 [H,W], final_tau [H,W],
    patch_range_per_tile int32 [T,2], gsid_per_patch int32 [M]].  Updates depths/areas in place
    for Gaussians whose tile rectangle is empty; final_tau of empty tiles is 0."""
    K = int(num_palette)
    if K < 1 or K > _lib.MAX_CHANNELS:
        raise ValueError(f"gsplatcu.splat_weight: num_palette must be in [1, {_lib.MAX_CHANNELS}]")
    return _splat_forward("splat_weight", height, width, K, us, cinv2ds, alphas, depths, weights,
                          areas, 0.0)


def splat_color(height, width, us, cinv2ds, alphas, depths, colors, areas):
    """gsplatcu/gausplat.cu:25-109 -> [image [3,H,W], contrib, final_tau, ranges, gsid];
    final_tau of empty tiles is 1."""
    return _splat_forward("splat_color", height, width, 3, us, cinv2ds, alphas, depths, colors,
                          areas, 1.0)


def _splat_backward(op, H, W, C_, us, cinv2ds, alphas, feats, contrib, final_tau, ranges, gsid,
                    dloss, dloss_dtau, geom):
    us, cinv = _cuda(op, "us", us), _cuda(op, "cinv2ds", cinv2ds)
    alphas = _cuda(op, "alphas", alphas)
    feats = _cuda(op, "features", feats, _SH_DTYPES)
    contrib = _cuda(op, "contrib", contrib, (torch.int32,))
    final_tau = _cuda(op, "final_tau", final_tau)
    ranges = _cuda(op, "patch_range_per_tile", ranges, (torch.int32,))
    gsid = _cuda(op, "gsid_per_patch", gsid, (torch.int32,))
    dloss = _cuda(op, "dloss", dloss)
    dtau = None if dloss_dtau is None else _cuda(op, "dloss_dfinal_tau", dloss_dtau)
    H, W, n = int(H), int(W), _n(us)
    dev = us.device
    dfeat = torch.zeros((n, 1, C_), dtype=_F32, device=dev)
    dalpha = torch.zeros((n, 1, 1), dtype=_F32, device=dev) if geom else None
    du = torch.zeros((n, 1, 2), dtype=_F32, device=dev) if geom else None
    dq = torch.zeros((n, 1, 3), dtype=_F32, device=dev) if geom else None
    with on_device(dev):
        packed = _take_packed(gsid, H, W, C_, us, cinv, alphas, feats)
        if packed is not None:  # the forward's records, inputs unchanged since
            call(op, "gsb_splat_backward_packed", n, H, W, C_, ptr(ranges), ptr(gsid),
                 ptr(contrib), ptr(final_tau), ptr(dloss), ptr(dtau), ptr(packed), ptr(dfeat),
                 ptr(dalpha), ptr(du), ptr(dq), stream_of(us))
            return dfeat, dalpha, du, dq
        state = torch.empty(int(_lib.lib().gsb_splat_state_bytes(n, C_, H, W)),
                            dtype=torch.uint8, device=dev)
        call(op, "gsb_splat_backward", n, H, W, C_, ptr(us), ptr(cinv), ptr(alphas), ptr(feats),
             _sh_dtype(feats), ptr(ranges), ptr(gsid), ptr(contrib), ptr(final_tau), ptr(dloss),
             ptr(dtau), ptr(state), ptr(dfeat), ptr(dalpha), ptr(du), ptr(dq), stream_of(us))
    return dfeat, dalpha, du, dq


def splat_weight_B(height, width, num_palette, us, cinv2ds, alphas, depths, weights, contrib,
                   final_tau, patch_range_per_tile, gsid_per_patch, dloss_dgammas):
    """gsplatcu/gausplat.cu:252-292 -> [dloss_dweights [N,1,K]]."""
    dfeat, _, _, _ = _splat_backward("splat_weight_B", height, width, int(num_palette), us,
                                     cinv2ds, alphas, weights, contrib, final_tau,
                                     patch_range_per_tile, gsid_per_patch, dloss_dgammas, None,
                                     geom=False)
    return [dfeat]


def splat_weight_B_full(height, width, num_palette, us, cinv2ds, alphas, depths, weights, contrib,
                        final_tau, patch_range_per_tile, gsid_per_patch, dloss_dgammas,
                        dloss_dfinal_tau=None):
    """Full adjoint of splat_weight -> [dloss_dweights [N,1,K], dloss_dus [N,1,2],
    dloss_dcinv2ds [N,1,3], dloss_dalphas [N,1,1]] (no counterpart in the reference, which
    back-propagates only into the weights)."""
    dfeat, da, du, dq = _splat_backward("splat_weight_B_full", height, width, int(num_palette), us,
                                        cinv2ds, alphas, weights, contrib, final_tau,
                                        patch_range_per_tile, gsid_per_patch, dloss_dgammas,
                                        dloss_dfinal_tau, geom=True)
    return [dfeat, du, dq, da]


def splat_color_B(height, width, us, cinv2ds, alphas, depths, colors, contrib, final_tau,
                  patch_range_per_tile, gsid_per_patch, dloss_dgammas, dloss_dfinal_tau=None):
    """gsplatcu/gausplat.cu:111-155 -> [dloss_dus [N,1,2], dloss_dcinv2ds [N,1,3],
    dloss_dalphas [N,1,1], dloss_dcolors [N,1,3]]."""
    dfeat, da, du, dq = _splat_backward("splat_color_B", height, width, 3, us, cinv2ds, alphas,
                                        colors, contrib, final_tau, patch_range_per_tile,
                                        gsid_per_patch, dloss_dgammas, dloss_dfinal_tau, geom=True)
    return [du, dq, da, dfeat]


# The stage-1 extension of the same project (vanilla_3dgs/gsplatcu/ext.cpp:71-77)
# names its colour splat `splat` / `splatB`; the backward also takes the
# gradient of the final transmittance (vanilla_3dgs/gsplatcu/gausplat.cu:114-160),
# which is how its training drives transparent regions empty
# (vanilla_3dgs/gsplat/gsmodel.py:27-75).
def splat(height, width, us, cinv2ds, alphas, depths, colors, areas):
    """vanilla_3dgs/gsplatcu/gausplat.cu:24-112 -> [image [3,H,W], contrib, final_tau, ranges,
    gsid] (final_tau of empty tiles is 1), as splat_color."""
    return splat_color(height, width, us, cinv2ds, alphas, depths, colors, areas)


def splatB(height, width, us, cinv2ds, alphas, depths, colors, contrib, final_tau,
           patch_range_per_tile, gsid_per_patch, dloss_dgammas, dloss_dfinal_taus):
    """vanilla_3dgs/gsplatcu/gausplat.cu:114-160 -> [dloss_dus [N,1,2], dloss_dcinv2ds [N,1,3],
    dloss_dalphas [N,1,1], dloss_dcolors [N,1,3]], including the final-transmittance term."""
    return splat_color_B(height, width, us, cinv2ds, alphas, depths, colors, contrib, final_tau,
                         patch_range_per_tile, gsid_per_patch, dloss_dgammas, dloss_dfinal_taus)


def lab2rgb(lab_image):
    """gsplatcu/gausplat.cu:623-641: [3,H,W] CIE Lab (L in [0,1]) -> sRGB [3,H,W]."""
    op = "lab2rgb"
    lab = _cuda(op, "lab_image", lab_image)
    H, W = int(lab.shape[1]), int(lab.shape[2])
    rgb = torch.empty((3, H, W), dtype=_F32, device=lab.device)
    with on_device(lab.device):
        call(op, "gsb_lab2rgb", H, W, ptr(lab), ptr(rgb), stream_of(lab))
    return rgb
