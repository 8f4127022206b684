"""Fused loss-side operators.

``palette_geo_loss(layer, chroma, target, clamp, lambda_pos, kind)`` is the
finetune step's loss on the rendered palette weights (finetune.py:356-389):
the barycentric target of the colour image in the palette {black, white,
chroma} (gsplat/gsmodel.py:219-285), optionally clamped to non-negative and
renormalised, then MSE (or L1) against the weights plus ``lambda_pos *
mean(relu(-layer))``.  One kernel computes the loss and both gradients
(the target depends on the learnt palette).

``palette_l1_loss(layer, palette, target)`` composites the palette colour
image ``image[c] = sum_k palette[k][c] * layer[k]`` and returns
``mean(|image - target|)``; its forward pass also produces the adjoint w.r.t.
``layer`` and ``palette`` in the same sweep over the image (one kernel), so
the backward is a scale by the incoming gradient.  It replaces the torch
``einsum`` + L1 sequence a finetune step would otherwise run (whose backward
is a large-K split GEMM).

``palette_l1_ssim_loss(layer, palette, target, lambda_ssim, lambda_pos)`` is
the differentiation workload's loss: gau_loss (vanilla_3dgs/gsplat/
pytorch_ssim.py:64-67, ``(1 - lambda) L1 + lambda (1 - SSIM)`` with the 11x11
sigma-1.5 window) on the palette colour image, plus ``lambda_pos *
mean(relu(-layer))``; ``gau_loss(image, gt_image, loss_lambda)`` is the same
kernel on a colour image.  One launch computes the loss and its gradient.
"""
import torch

from gsplatcu import _lib


class PaletteL1Loss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, layer, palette, target):
        if not (layer.is_cuda and layer.dtype == torch.float32):
            raise TypeError("palette_l1_loss: layer must be a CUDA float32 tensor [K,H,W]")
        layer = layer.contiguous()
        palette = palette.detach().to(torch.float32).contiguous()
        target = target.contiguous()
        K, H, W = (int(x) for x in layer.shape)
        if tuple(palette.shape) != (K, 3) or tuple(target.shape) != (3, H, W):
            raise ValueError("palette_l1_loss: palette must be [K,3] and target [3,H,W]")
        loss = torch.empty((), dtype=torch.float32, device=layer.device)
        dlayer = torch.empty_like(layer)
        dpal = torch.empty((K, 3), dtype=torch.float32, device=layer.device)
        with _lib.on_device(layer.device):
            _lib.call("palette_l1_loss", "gsb_palette_l1", K, H, W, _lib.ptr(layer),
                      _lib.ptr(palette), _lib.ptr(target), None, _lib.ptr(loss), _lib.ptr(dlayer),
                      _lib.ptr(dpal), _lib.stream_of(layer))
        ctx.save_for_backward(dlayer, dpal)
        return loss

    @staticmethod
    def backward(ctx, g):
        dlayer, dpal = ctx.saved_tensors
        return dlayer * g, dpal * g, None


def palette_l1_loss(layer, palette, target):
    return PaletteL1Loss.apply(layer, palette, target)


def palette_image(layer, palette):
    """image[c] = sum_k palette[k][c] * layer[k] (no gradient)."""
    K, H, W = (int(x) for x in layer.shape)
    layer = layer.contiguous()
    palette = palette.detach().to(torch.float32).contiguous()
    image = torch.empty((3, H, W), dtype=torch.float32, device=layer.device)
    loss = torch.empty((), dtype=torch.float32, device=layer.device)
    zero = torch.zeros((3, H, W), dtype=torch.float32, device=layer.device)
    with _lib.on_device(layer.device):
        _lib.call("palette_image", "gsb_palette_l1", K, H, W, _lib.ptr(layer), _lib.ptr(palette),
                  _lib.ptr(zero), _lib.ptr(image), _lib.ptr(loss), None, None,
                  _lib.stream_of(layer))
    return image


class PaletteGeoLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, layer, chroma, target, clamp, lambda_pos, kind):
        if not (layer.is_cuda and layer.dtype == torch.float32):
            raise TypeError("palette_geo_loss: layer must be a CUDA float32 tensor [K,H,W]")
        layer = layer.contiguous()
        chroma = chroma.detach().to(torch.float32).contiguous()
        target = target.to(torch.float32).contiguous()
        K, H, W = (int(x) for x in layer.shape)
        Kc = int(chroma.shape[0])
        if tuple(chroma.shape) != (Kc, 3) or K != Kc + 2 or tuple(target.shape) != (3, H, W):
            raise ValueError("palette_geo_loss: layer must be [Kc+2,H,W], chroma [Kc,3] and "
                             "target [3,H,W]")
        loss = torch.empty((3,), dtype=torch.float32, device=layer.device)
        dlayer = torch.empty_like(layer)
        dchroma = torch.empty((Kc, 3), dtype=torch.float32, device=layer.device)
        code = {"mse": _lib.LOSS_MSE, "l1": _lib.LOSS_L1}[kind]
        with _lib.on_device(layer.device):
            _lib.call("palette_geo_loss", "gsb_palette_geo_loss", Kc, H, W, _lib.ptr(layer),
                      _lib.ptr(target), _lib.ptr(chroma), int(bool(clamp)), code,
                      float(lambda_pos), None, _lib.ptr(loss), _lib.ptr(dlayer),
                      _lib.ptr(dchroma), _lib.stream_of(layer))
        ctx.save_for_backward(dlayer, dchroma)
        return loss[0]

    @staticmethod
    def backward(ctx, g):
        dlayer, dchroma = ctx.saved_tensors
        return dlayer * g, dchroma * g, None, None, None, None


def palette_geo_loss(layer, chroma, target, clamp=False, lambda_pos=0.5, kind="mse"):
    """Loss of rendered palette weights `layer` [Kc+2,H,W] against the
    barycentric target of `target` [3,H,W] in {black, white, chroma [Kc,3]}."""
    return PaletteGeoLoss.apply(layer, chroma, target, clamp, lambda_pos, kind)


def barycentric_target(target, chroma, clamp=False):
    """The (optionally clamped and renormalised) barycentric weights
    [Kc+2,H,W] of the colour image `target` (no gradient)."""
    chroma = chroma.detach().to(torch.float32).contiguous()
    target = target.to(torch.float32).contiguous()
    Kc = int(chroma.shape[0])
    H, W = int(target.shape[1]), int(target.shape[2])
    out = torch.empty((Kc + 2, H, W), dtype=torch.float32, device=target.device)
    zero = torch.zeros_like(out)
    loss = torch.empty((3,), dtype=torch.float32, device=target.device)
    with _lib.on_device(target.device):
        _lib.call("barycentric_target", "gsb_palette_geo_loss", Kc, H, W, _lib.ptr(zero),
                  _lib.ptr(target), _lib.ptr(chroma), int(bool(clamp)), _lib.LOSS_MSE, 0.0,
                  _lib.ptr(out), _lib.ptr(loss), None, None, _lib.stream_of(target))
    return out


def _l1_ssim(name, K, H, W, layer, palette, target, lambda_ssim, lambda_pos, data_range,
             need_grad):
    dev = layer.device
    loss = torch.empty((4,), dtype=torch.float32, device=dev)
    dlayer = torch.empty_like(layer) if need_grad else None
    dpal = torch.empty((K, 3), dtype=torch.float32, device=dev) if (
        need_grad and palette is not None) else None
    with _lib.on_device(dev):
        _lib.call(name, "gsb_palette_l1_ssim", K, H, W, _lib.ptr(layer),
                  None if palette is None else _lib.ptr(palette), _lib.ptr(target),
                  float(lambda_ssim), float(lambda_pos), float(data_range), None, _lib.ptr(loss),
                  None if dlayer is None else _lib.ptr(dlayer),
                  None if dpal is None else _lib.ptr(dpal), _lib.stream_of(layer))
    return loss, dlayer, dpal


class PaletteL1SsimLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, layer, palette, target, lambda_ssim, lambda_pos, data_range):
        if not (layer.is_cuda and layer.dtype == torch.float32 and layer.dim() == 3):
            raise TypeError("palette_l1_ssim_loss: layer must be a CUDA float32 tensor [K,H,W]")
        layer = layer.contiguous()
        K, H, W = (int(x) for x in layer.shape)
        target = target.to(torch.float32).contiguous()
        if palette is not None:
            palette = palette.detach().to(torch.float32).contiguous()
            if tuple(palette.shape) != (K, 3):
                raise ValueError("palette_l1_ssim_loss: palette must be [K,3]")
        elif K != 3:
            raise ValueError("gau_loss: the image must be [3,H,W]")
        if tuple(target.shape) != (3, H, W):
            raise ValueError("palette_l1_ssim_loss: target must be [3,H,W]")
        need = any(ctx.needs_input_grad[:2])
        loss, dlayer, dpal = _l1_ssim("palette_l1_ssim_loss", K, H, W, layer, palette, target,
                                      lambda_ssim, lambda_pos, data_range, need)
        ctx.save_for_backward(dlayer, dpal)
        return loss  # [total, L1, SSIM, penalty]; only the total is differentiated

    @staticmethod
    def backward(ctx, g):
        dlayer, dpal = ctx.saved_tensors
        g = g[0]
        return (None if dlayer is None else dlayer * g, None if dpal is None else dpal * g,
                None, None, None, None)


def palette_l1_ssim_loss(layer, palette, target, lambda_ssim=0.2, lambda_pos=0.5,
                         data_range=1.0, parts=False):
    """(1 - lambda_ssim) mean|img - target| + lambda_ssim (1 - mean SSIM(img,
    target)) + lambda_pos mean(relu(-layer)), img = sum_k palette[k] layer[k].
    With ``parts`` also returns the tensor [total, L1, SSIM, penalty]."""
    p = PaletteL1SsimLoss.apply(layer, palette, target, float(lambda_ssim), float(lambda_pos),
                                float(data_range))
    return (p[0], p.detach()) if parts else p[0]


def gau_loss(image, gt_image, loss_lambda=0.2):
    """gau_loss of vanilla_3dgs/gsplat/pytorch_ssim.py:64-67 on a colour image
    [3,H,W]: (1 - loss_lambda) L1 + loss_lambda (1 - SSIM), one kernel."""
    return PaletteL1SsimLoss.apply(image, None, gt_image, float(loss_lambda), 0.0, 1.0)[0]
