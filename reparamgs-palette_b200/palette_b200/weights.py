"""Palette-weight splatting through the drop-in ``gsplatcu`` operators, with a
fused weight-parameter adjoint.

``splat_palette_weights(pws, alphas, scales, rots, cam, shs=... | dc=, A=, B=)``
returns ``(layer [K,H,W], visible [N])`` -- the rendered palette-weight layers
and the ``depths > 0.2`` mask -- and is differentiable in the weight
parameters (geometry is frozen, as in ReparamGS-Palette's finetune stage,
gsplat/gsmodel.py:104-200).  It computes what the reference's own autograd
functions compute, organised differently:

* forward: the operator chain project -> computeCov3D -> computeCov2D ->
  sh2Weight / sh2Weight_fast -> inverseCov2D -> splat_weight, with the weight
  operator called *without* its Jacobian outputs (no per-Gaussian SH basis or
  dweight_ddc tensors are written or kept);
* backward: ``splat_weight_B`` for dL/dweights, then one kernel
  (``gsb_palette_weights_backward``) that recomputes the view direction and SH
  basis per Gaussian and writes dL/dshs [N,16K] -- or dL/ddc, dL/dA, dL/dB for
  rank-r factors -- directly, where the reference runs a batched outer product
  in torch (full weights) or an elementwise product plus sh2Weight_fast_B
  (low rank).

Weight parameters may be FP32 or BF16 (FP32 arithmetic; gradients come back
in the parameter's dtype).  Low-rank factors are ``A [N,P]``/``B [N,Q]``
(rank 1, the reference's layout) or ``A [N,P,r]``/``B [N,r,Q]``.  Supported
shapes are those of the fused kernels (full SH with K in 3..8; low-rank
(K,P,Q,r) in (5,5,15,1..4), (3,3,15,1), (4,4,15,1), (6,6,15,1), (6,6,15,3));
for other shapes use the operators directly.
"""
import ctypes as C

import torch

import gsplatcu as gsc
from gsplatcu import _lib

from .render import _params, _weight_args, camera_struct

_F32 = torch.float32


class _OperatorSplat(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pws, alphas, scales, rots, w0, A, B, cam, mode, K, P, Q, rank):
        us, pcs, depths = gsc.project(pws, cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
        cov3, = gsc.computeCov3D(rots, scales, depths, False)
        cov2, = gsc.computeCov2D(cov3, pcs, cam.Rcw, depths, cam.fx, cam.fy, cam.width,
                                 cam.height, False)
        if mode == _lib.WEIGHTS_FULL:
            w, = gsc.sh2Weight(w0, pws, cam.twc, False, K)
        else:
            w, = gsc.sh2Weight_fast(w0, A, B, pws, cam.twc, False, K, Q)
        cinv, areas = gsc.inverseCov2D(cov2, depths, False)
        layer, contrib, ft, ranges, gsid = gsc.splat_weight(cam.height, cam.width, K, us, cinv,
                                                            alphas, depths, w, areas)
        ctx.meta = (cam, mode, K, P, Q, rank)
        ctx.save_for_backward(pws, alphas, w0, A, B, us, cinv, depths, w, contrib, ft, ranges, gsid)
        visible = depths > 0.2
        ctx.mark_non_differentiable(visible)
        return layer, visible

    @staticmethod
    def backward(ctx, dlayer, _dvisible):
        cam, mode, K, P, Q, rank = ctx.meta
        pws, alphas, w0, A, B, us, cinv, depths, w, contrib, ft, ranges, gsid = ctx.saved_tensors
        dev = pws.device
        n = int(pws.shape[0])
        dW, = gsc.splat_weight_B(cam.height, cam.width, K, us, cinv, alphas, depths, w, contrib,
                                 ft, ranges, gsid, dlayer.contiguous())
        camst, _keep = camera_struct(cam)
        params = _params(mode, K, P, Q, rank, w0, A, B)
        dw0 = torch.empty(tuple(w0.shape), dtype=_F32, device=dev)
        dA = torch.empty(tuple(A.shape), dtype=_F32, device=dev) if A is not None else None
        dB = torch.empty(tuple(B.shape), dtype=_F32, device=dev) if B is not None else None
        with _lib.on_device(dev):
            st = _lib.stream_of(pws)
            _lib.call("splat_palette_weights.backward", "gsb_palette_weights_backward", n,
                      C.byref(camst), _lib.ptr(pws), C.byref(params), _lib.ptr(dW),
                      _lib.ptr(dw0), _lib.ptr(dA), _lib.ptr(dB), st)
            _lib.fetch_device_status(dev, st)
        cast = lambda g, like: None if g is None else g.to(like.dtype)
        return (None, None, None, None, cast(dw0, w0), cast(dA, A), cast(dB, B),
                None, None, None, None, None, None)


def splat_palette_weights(pws, alphas, scales, rots, cam, shs=None, dc=None, A=None, B=None,
                          K=None):
    """Render palette-weight layers through the gsplatcu operators.  Pass
    ``shs [N,16K]`` (full SH order 3, band-major) or ``dc [N,K], A, B``
    (low rank).  Returns ``(layer [K,H,W], visible [N] bool)``; gradients
    flow to the weight parameters only."""
    for name, t in (("pws", pws), ("alphas", alphas), ("scales", scales), ("rots", rots)):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == _F32):
            raise TypeError(f"splat_palette_weights: {name} must be a CUDA float32 tensor")
    w0, A, B, mode, K, P, Q, rank = _weight_args(shs, dc, A, B, K)
    return _OperatorSplat.apply(pws.contiguous(), alphas.contiguous(), scales.contiguous(),
                                rots.contiguous(), w0, A, B, cam, mode, K, P, Q, rank)
