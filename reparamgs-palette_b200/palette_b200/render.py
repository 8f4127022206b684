"""Fused palette-weight rendering with the full adjoint.

``render_palette(pws, rots, scales, alphas, cam, shs=... | dc=..., A=..., B=...)``
renders one view and returns ``(layer [K,H,W], final_tau [H,W], depths [N])``.
The forward runs the per-Gaussian work of project / computeCov3D /
computeCov2D / sh2Weight(_fast) / inverseCov2D in one kernel and then the same
binning and compositing as ``gsplatcu.splat_weight``; it computes what the
reference operator sequence computes (gsplat/gsmodel.py:107-118, 155-170),
with ``depths`` the reference's depths after its in-place updates
(``depths > 0.2`` is the visibility mask ``WeightGSFunctionTest`` returns).

Unlike the reference's backward, which only differentiates the weights, the
backward here returns gradients for every input that requires one: means,
rotations, scales, opacities and the weight parameters (full ``shs [N,16K]``
or low-rank ``dc [N,K], A [N,P,r], B [N,r,Q]``), including the
final-transmittance term when ``final_tau`` feeds the loss.  When no geometry
input requires a gradient only the weight gradients are computed.  Weight
parameters may be bfloat16 (FP32 arithmetic; gradients are returned in the
parameter's dtype).

``render_palette_views(pws, rots, scales, alphas, cams, ...)`` renders a batch
of views of one scene (a training step's batch) and returns per-view lists;
its backward sums the views' gradients in FP32 inside the kernels (the first
view overwrites the FP32 gradient buffers, the others add to them) and casts
once, so BF16 parameters are not accumulated in BF16.
"""
import ctypes as C
import weakref

import torch

from gsplatcu import _lib, _sort_and_draw

_F32 = torch.float32


def _f32c(t):
    return t if t.dtype == _F32 and t.is_contiguous() else t.to(_F32).contiguous()


# gsb_camera structs of recently used camera objects, rebuilt when any of the
# camera's fields or tensors (identity or in-place version) changes.  An entry
# holds its tensors, so their identities cannot be reused while it lives.
_CAMS = weakref.WeakKeyDictionary()


def _cam_signature(cam):
    return (id(cam.Rcw), cam.Rcw._version, id(cam.tcw), cam.tcw._version, id(cam.twc),
            cam.twc._version, float(cam.fx), float(cam.fy), float(cam.cx), float(cam.cy),
            int(cam.width), int(cam.height))


def camera_struct(cam):
    """(gsb_camera, tensors to keep alive) for a camera-like object."""
    try:
        hit = _CAMS.get(cam)
    except TypeError:  # not weak-referenceable: no caching
        hit = None
    if hit is not None and hit[0] == _cam_signature(cam):
        return hit[1], hit[2]
    Rcw, tcw, twc = _f32c(cam.Rcw), _f32c(cam.tcw), _f32c(cam.twc)
    c = _lib.Camera(Rcw.data_ptr(), tcw.data_ptr(), twc.data_ptr(), float(cam.fx), float(cam.fy),
                    float(cam.cx), float(cam.cy), int(cam.width), int(cam.height))
    try:  # the entry keeps the camera's own tensors, so their ids stay theirs
        _CAMS[cam] = (_cam_signature(cam), c, (Rcw, tcw, twc, cam.Rcw, cam.tcw, cam.twc))
    except TypeError:
        pass
    return c, (Rcw, tcw, twc)


_PARAMS = {}
_STATE_BYTES = {}


def _params(mode, K, P, Q, rank, w0, A, B):
    """gsb_palette_params of the weight parameters (pointers and shapes only,
    so a struct built for the same tensors' storage can be reused)."""
    key = (mode, w0.dtype, K, P, Q, rank, w0.data_ptr(),
           A.data_ptr() if A is not None else 0, B.data_ptr() if B is not None else 0)
    p = _PARAMS.get(key)
    if p is None:
        if len(_PARAMS) > 64:
            _PARAMS.clear()
        p = _PARAMS[key] = _lib.PaletteParams(
            mode, _lib.DTYPE_BF16 if w0.dtype == torch.bfloat16 else _lib.DTYPE_F32, K, P, Q,
            rank, key[6], A.data_ptr() if A is not None else None,
            B.data_ptr() if B is not None else None)
    return p


def _state_bytes(n, K, H, W):
    key = (n, K, H, W)
    b = _STATE_BYTES.get(key)
    if b is None:
        if len(_STATE_BYTES) > 256:
            _STATE_BYTES.clear()
        b = _STATE_BYTES[key] = int(_lib.lib().gsb_splat_state_bytes(n, K, H, W))
    return b


def _check(name, t, dtypes=(_F32,)):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype in dtypes):
        raise TypeError(f"render_palette: {name} must be a CUDA tensor of dtype {dtypes}")
    return t.contiguous()


def _render_one(pws, rots, scales, alphas, w0, A, B, cam, mode, K, P, Q, rank):
    """One view: fused preprocess, tile sort and compositing.  Returns
    (layer, final_tau, depths, state, ranges, gsid, contrib)."""
    dev = pws.device
    n = int(pws.shape[0])
    H, W = int(cam.height), int(cam.width)
    L = _lib.lib()
    camst, keep = camera_struct(cam)
    params = _params(mode, K, P, Q, rank, w0, A, B)
    with _lib.on_device(dev):
        st = _lib.stream_of(pws)
        state = torch.empty(_state_bytes(n, K, H, W), dtype=torch.uint8, device=dev)
        depths = torch.empty((n,), dtype=_F32, device=dev)
        _lib.call("render_palette", "gsb_render_preprocess", n, C.byref(camst), _lib.ptr(pws),
                  _lib.ptr(rots), _lib.ptr(scales), _lib.ptr(alphas), C.byref(params),
                  _lib.ptr(state), _lib.ptr(depths), st)
        _lib.fetch_device_status(dev, st)  # checked at the patch-count read-back below
        gx, gy = (W + 15) // 16, (H + 15) // 16
        ranges = torch.empty((gx * gy, 2), dtype=torch.int32, device=dev)
        layer = torch.empty((K, H, W), dtype=_F32, device=dev)
        contrib = torch.empty((H, W), dtype=torch.int32, device=dev)
        final_tau = torch.empty((H, W), dtype=_F32, device=dev)
        gsid = _sort_and_draw("render_palette", n, H, W, K, state, ranges, layer, contrib,
                              final_tau, 0.0, dev, st)
    return layer, final_tau, depths, state, ranges, gsid, contrib


class _RenderPalette(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pws, rots, scales, alphas, w0, A, B, cam, mode, K, P, Q, rank):
        layer, final_tau, depths, state, ranges, gsid, contrib = _render_one(
            pws, rots, scales, alphas, w0, A, B, cam, mode, K, P, Q, rank)
        ctx.meta = (cam, mode, K, P, Q, rank)
        ctx.save_for_backward(pws, rots, scales, alphas, w0, A, B, state, ranges, gsid, contrib,
                              final_tau)
        ctx.mark_non_differentiable(depths)
        return layer, final_tau, depths

    @staticmethod
    def backward(ctx, dlayer, dtau, _ddepths):
        cam, mode, K, P, Q, rank = ctx.meta
        (pws, rots, scales, alphas, w0, A, B, state, ranges, gsid, contrib,
         final_tau) = ctx.saved_tensors
        dev = pws.device
        n = int(pws.shape[0])
        camst, _keep = camera_struct(cam)
        params = _params(mode, K, P, Q, rank, w0, A, B)
        L = _lib.lib()
        if dlayer is None:
            dlayer = torch.zeros((K,) + tuple(final_tau.shape), dtype=_F32, device=dev)
        dlayer = dlayer.contiguous()
        dtau = dtau.contiguous() if dtau is not None else None
        # geometry gradients only when a geometry input needs one (the
        # reference's own backward differentiates the weights alone)
        geom = any(ctx.needs_input_grad[:4])
        e = (lambda *shape: torch.empty(shape, dtype=_F32, device=dev)) if geom else \
            (lambda *shape: None)
        with _lib.on_device(dev):
            scratch = torch.empty(int(L.gsb_render_backward_bytes(n, K)), dtype=torch.uint8,
                                  device=dev)
            dpws, drots, dscales, dalphas = e(n, 3), e(n, 4), e(n, 3), e(n)
            dw0 = torch.empty(tuple(w0.shape), dtype=_F32, device=dev)
            dA = torch.empty(tuple(A.shape), dtype=_F32, device=dev) if A is not None else None
            dB = torch.empty(tuple(B.shape), dtype=_F32, device=dev) if B is not None else None
            _lib.call("render_palette.backward", "gsb_render_backward", n, C.byref(camst),
                      _lib.ptr(pws), _lib.ptr(rots), _lib.ptr(scales), _lib.ptr(alphas),
                      C.byref(params), _lib.ptr(state), _lib.ptr(ranges), _lib.ptr(gsid),
                      _lib.ptr(contrib), _lib.ptr(final_tau), _lib.ptr(dlayer), _lib.ptr(dtau),
                      _lib.ptr(scratch), _lib.ptr(dpws), _lib.ptr(drots), _lib.ptr(dscales),
                      _lib.ptr(dalphas), _lib.ptr(dw0), _lib.ptr(dA), _lib.ptr(dB),
                      _lib.stream_of(pws))
            _lib.fetch_device_status(dev, _lib.stream_of(pws))
        if dalphas is not None:
            dalphas = dalphas.reshape(alphas.shape)
        cast = lambda g, like: None if g is None else g.to(like.dtype)
        return (dpws, drots, dscales, dalphas, cast(dw0, w0), cast(dA, A), cast(dB, B),
                None, None, None, None, None, None)


def _weight_args(shs, dc, A, B, K):
    """(w0, A, B, mode, K, P, Q, rank) of the palette weight parameters."""
    wt = (torch.float32, torch.bfloat16)
    if shs is not None:
        shs = _check("shs", shs, wt)
        K = int(K) if K is not None else int(shs.shape[1]) // 16
        if int(shs.shape[1]) != 16 * K:
            raise ValueError("render_palette: shs must be [N, 16*K] (SH order 3)")
        return shs, None, None, _lib.WEIGHTS_FULL, K, 0, 0, 0
    if dc is None or A is None or B is None:
        raise ValueError("render_palette: pass shs, or dc, A and B")
    dc, A, B = _check("dc", dc, wt), _check("A", A, wt), _check("B", B, wt)
    if not (dc.dtype == A.dtype == B.dtype):
        raise TypeError("render_palette: dc, A and B must share a dtype")
    K = int(dc.shape[1])
    if A.dim() == 2:
        P, rank, Q = int(A.shape[1]), 1, int(B.shape[1])
    else:
        P, rank, Q = int(A.shape[1]), int(A.shape[2]), int(B.shape[2])
    return dc, A, B, _lib.WEIGHTS_LOWRANK, K, P, Q, rank


def render_palette(pws, rots, scales, alphas, cam, shs=None, dc=None, A=None, B=None, K=None):
    """Render palette weights for one camera.  Pass ``shs [N,16K]`` (full SH
    order 3) or the low-rank ``dc [N,K], A [N,P,r] (or [N,P]), B [N,r,Q] (or
    [N,Q])``.  Returns ``(layer [K,H,W], final_tau [H,W], depths [N])``."""
    pws, rots, scales = _check("pws", pws), _check("rots", rots), _check("scales", scales)
    alphas = _check("alphas", alphas)
    w0, A, B, mode, K, P, Q, rank = _weight_args(shs, dc, A, B, K)
    if not (torch.is_grad_enabled() and any(
            t is not None and t.requires_grad for t in (pws, rots, scales, alphas, w0, A, B))):
        # nothing to differentiate: render without the autograd node
        return _render_one(pws, rots, scales, alphas, w0, A, B, cam, mode, K, P, Q, rank)[:3]
    return _RenderPalette.apply(pws, rots, scales, alphas, w0, A, B, cam, mode, K, P, Q, rank)


class _RenderPaletteViews(torch.autograd.Function):
    """Several views of one scene.  Forward: one render per camera, as
    _RenderPalette.  Backward: the views' adjoints summed into one FP32 buffer
    per parameter (the first view overwrites it, the others add to it:
    gsb_render_backward_accumulate), cast to the parameters' dtype once."""

    @staticmethod
    def forward(ctx, pws, rots, scales, alphas, w0, A, B, cams, mode, K, P, Q, rank):
        V = len(cams)
        layers, taus, depths, flat = [], [], [], [pws, rots, scales, alphas, w0, A, B]
        for cam in cams:
            layer, ft, d, state, ranges, gsid, contrib = _render_one(
                pws, rots, scales, alphas, w0, A, B, cam, mode, K, P, Q, rank)
            layers.append(layer)
            taus.append(ft)
            depths.append(d)
            flat.extend((state, ranges, gsid, contrib, ft))
        ctx.meta = (cams, mode, K, P, Q, rank, V)
        ctx.save_for_backward(*flat)
        ctx.mark_non_differentiable(*depths)
        return tuple(layers) + tuple(taus) + tuple(depths)

    @staticmethod
    def backward(ctx, *grads):
        cams, mode, K, P, Q, rank, V = ctx.meta
        t = ctx.saved_tensors
        pws, rots, scales, alphas, w0, A, B = t[:7]
        views = [t[7 + 5 * v: 12 + 5 * v] for v in range(V)]
        dev = pws.device
        n = int(pws.shape[0])
        geom = any(ctx.needs_input_grad[:4])
        e = (lambda *shape: torch.empty(shape, dtype=_F32, device=dev)) if geom else \
            (lambda *shape: None)
        L = _lib.lib()
        params = _params(mode, K, P, Q, rank, w0, A, B)
        with _lib.on_device(dev):
            st = _lib.stream_of(pws)
            scratch = torch.empty(int(L.gsb_render_backward_bytes(n, K)), dtype=torch.uint8,
                                  device=dev)
            dpws, drots, dscales, dalphas = e(n, 3), e(n, 4), e(n, 3), e(n)
            dw0 = torch.empty(tuple(w0.shape), dtype=_F32, device=dev)
            dA = torch.empty(tuple(A.shape), dtype=_F32, device=dev) if A is not None else None
            dB = torch.empty(tuple(B.shape), dtype=_F32, device=dev) if B is not None else None
            for v, (state, ranges, gsid, contrib, final_tau) in enumerate(views):
                dlayer, dtau = grads[v], grads[V + v]
                if dlayer is None:
                    dlayer = torch.zeros((K,) + tuple(final_tau.shape), dtype=_F32, device=dev)
                dlayer = dlayer.contiguous()
                dtau = dtau.contiguous() if dtau is not None else None
                camst, _keep = camera_struct(cams[v])
                _lib.call("render_palette_views.backward",
                          "gsb_render_backward" if v == 0 else "gsb_render_backward_accumulate",
                          n, C.byref(camst), _lib.ptr(pws), _lib.ptr(rots), _lib.ptr(scales),
                          _lib.ptr(alphas), C.byref(params), _lib.ptr(state), _lib.ptr(ranges),
                          _lib.ptr(gsid), _lib.ptr(contrib), _lib.ptr(final_tau),
                          _lib.ptr(dlayer), _lib.ptr(dtau), _lib.ptr(scratch), _lib.ptr(dpws),
                          _lib.ptr(drots), _lib.ptr(dscales), _lib.ptr(dalphas), _lib.ptr(dw0),
                          _lib.ptr(dA), _lib.ptr(dB), st)
            _lib.fetch_device_status(dev, st)
        if dalphas is not None:
            dalphas = dalphas.reshape(alphas.shape)
        cast = lambda g, like: None if g is None else g.to(like.dtype)
        return (dpws, drots, dscales, dalphas, cast(dw0, w0), cast(dA, A), cast(dB, B),
                None, None, None, None, None, None)


def render_palette_views(pws, rots, scales, alphas, cams, shs=None, dc=None, A=None, B=None,
                         K=None):
    """Render palette weights for several cameras of one scene (a training
    step's batch of views).  Parameters as ``render_palette``.  Returns lists
    ``(layers [K,H,W] per view, final_taus [H,W] per view, depths [N] per
    view)``.  The backward sums the views' gradients in FP32 before casting
    them to the parameters' dtype (BF16 factors are not summed in BF16)."""
    pws, rots, scales = _check("pws", pws), _check("rots", rots), _check("scales", scales)
    alphas = _check("alphas", alphas)
    cams = list(cams)
    if not cams:
        raise ValueError("render_palette_views: no cameras")
    w0, A, B, mode, K, P, Q, rank = _weight_args(shs, dc, A, B, K)
    out = _RenderPaletteViews.apply(pws, rots, scales, alphas, w0, A, B, cams, mode, K, P, Q, rank)
    V = len(cams)
    return list(out[:V]), list(out[V:2 * V]), list(out[2 * V:])
