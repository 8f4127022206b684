"""Fused loss-side operators.

``palette_l1_loss(layer, palette, target)`` composites the palette colour
image ``image[c] = sum_k palette[k][c] * layer[k]`` and returns
``mean(|image - target|)``; its forward pass also produces the adjoint w.r.t.
``layer`` and ``palette`` in the same sweep over the image (one kernel), so
the backward is a scale by the incoming gradient.  It replaces the torch
``einsum`` + L1 sequence a finetune step would otherwise run (whose backward
is a large-K split GEMM).
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
        with torch.cuda.device(layer.device):
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
    with torch.cuda.device(layer.device):
        _lib.call("palette_image", "gsb_palette_l1", K, H, W, _lib.ptr(layer), _lib.ptr(palette),
                  _lib.ptr(zero), _lib.ptr(image), _lib.ptr(loss), None, None,
                  _lib.stream_of(layer))
    return image
