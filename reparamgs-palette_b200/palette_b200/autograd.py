"""Autograd functions over the drop-in ``gsplatcu`` operators.

``WeightGSFunctionTest`` and ``WeightGSFunctionFast`` have the signatures and
gradient semantics of the reference's own functions (gsplat/gsmodel.py:104-200):
the forward runs project -> computeCov3D -> computeCov2D -> sh2Weight(_fast)
-> inverseCov2D -> splat_weight and returns ``(layer_W [K,H,W], depths > 0.2)``;
the backward returns gradients for the colour parameters only (``shs``, or
``shs_dc / shs_A / shs_B``), geometry being frozen.  ``WeightGSFunctionFast``
also accepts rank-r factors ``shs_A [N,P,r]``, ``shs_B [N,r,Q]``.

The reference's own gsmodel.py runs unchanged on ``gsplatcu`` too; these
copies let callers use the B200 operators without importing it.
"""
import torch

import gsplatcu as gsc

SH_C0 = 0.28209479177387814


class WeightGSFunctionTest(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pws, shs, alphas, scales, rots, cam, num_palette):
        us, pcs, depths = gsc.project(pws, cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
        cov3ds, = gsc.computeCov3D(rots, scales, depths, False)
        cov2ds, = gsc.computeCov2D(cov3ds, pcs, cam.Rcw, depths, cam.fx, cam.fy, cam.width,
                                   cam.height, False)
        weights, dweight_dshs, _ = gsc.sh2Weight(shs, pws, cam.twc, True, num_palette)
        cinv2ds, areas = gsc.inverseCov2D(cov2ds, depths, False)
        layer, contrib, final_tau, ranges, gsid = gsc.splat_weight(
            cam.height, cam.width, num_palette, us, cinv2ds, alphas, depths, weights, areas)
        ctx.cam, ctx.num_palette, ctx.shs_dtype = cam, num_palette, shs.dtype
        ctx.save_for_backward(us, cinv2ds, alphas, depths, weights, contrib, final_tau, ranges,
                              gsid, dweight_dshs)
        return layer, depths > 0.2

    @staticmethod
    def backward(ctx, dloss_dlayer, _):
        cam, K = ctx.cam, ctx.num_palette
        (us, cinv2ds, alphas, depths, weights, contrib, final_tau, ranges, gsid,
         dweight_dshs) = ctx.saved_tensors
        dW, = gsc.splat_weight_B(cam.height, cam.width, K, us, cinv2ds, alphas, depths, weights,
                                 contrib, final_tau, ranges, gsid, dloss_dlayer.contiguous())
        dshs = (dW.permute(0, 2, 1) @ dweight_dshs).permute(0, 2, 1)  # [N, nb, K] outer product
        n, nb, k = dshs.shape
        return (None, dshs.reshape(n, nb * k).to(ctx.shs_dtype), None, None, None, None, None)


class WeightGSFunctionFast(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pws, shs_dc, shs_A, shs_B, alphas, scales, rots, cam, num_palette, Q):
        us, pcs, depths = gsc.project(pws, cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
        cov3ds, = gsc.computeCov3D(rots, scales, depths, False)
        cov2ds, = gsc.computeCov2D(cov3ds, pcs, cam.Rcw, depths, cam.fx, cam.fy, cam.width,
                                   cam.height, False)
        weights, dweight_ddc, ylm = gsc.sh2Weight_fast(shs_dc, shs_A, shs_B, pws, cam.twc, True,
                                                       num_palette, Q)
        cinv2ds, areas = gsc.inverseCov2D(cov2ds, depths, False)
        layer, contrib, final_tau, ranges, gsid = gsc.splat_weight(
            cam.height, cam.width, num_palette, us, cinv2ds, alphas, depths, weights, areas)
        ctx.cam, ctx.num_palette, ctx.Q, ctx.dtype = cam, num_palette, Q, shs_dc.dtype
        ctx.save_for_backward(us, cinv2ds, alphas, depths, weights, contrib, final_tau, ranges,
                              gsid, dweight_ddc, ylm, shs_A, shs_B)
        return layer, depths > 0.2

    @staticmethod
    def backward(ctx, dloss_dlayer, _):
        cam, K, Q = ctx.cam, ctx.num_palette, ctx.Q
        (us, cinv2ds, alphas, depths, weights, contrib, final_tau, ranges, gsid, dweight_ddc, ylm,
         shs_A, shs_B) = ctx.saved_tensors
        dW, = gsc.splat_weight_B(cam.height, cam.width, K, us, cinv2ds, alphas, depths, weights,
                                 contrib, final_tau, ranges, gsid, dloss_dlayer.contiguous())
        dw = dW.squeeze(1)
        ddc = dw * dweight_ddc
        dA, dB = gsc.sh2Weight_fast_B(shs_A, shs_B, ylm, dw, K, Q)
        d = ctx.dtype
        return (None, ddc.to(d), dA.to(d), dB.to(d), None, None, None, None, None, None)
