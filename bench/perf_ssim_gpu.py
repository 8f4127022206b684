#!/usr/bin/env python
"""Timing of the fused L1 + SSIM loss (palette_b200.loss.palette_l1_ssim_loss)
against the same loss written with torch operators the way the reference
computes it (vanilla_3dgs/gsplat/pytorch_ssim.py:26-67: five grouped
conv2d calls with the 11x11 window, then autograd for the gradient), plus the
palette composite and the negative-weight penalty of the finetune loss.  Both
run on this GPU on the same inputs (K = 5 layer stack at the given size);
times are CUDA-event medians of forward + backward.  Not collected by pytest.

    python bench/perf_ssim_gpu.py [--width 1920] [--height 1080] [--reps 50]
"""
import argparse
import json
import math
import os
import statistics
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, os.path.join(ROOT, "reparamgs-palette_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import torch  # noqa: E402
import torch.nn.functional as F  # noqa: E402


def torch_window(device):
    g = torch.tensor([math.exp(-(x - 5) ** 2 / (2 * 1.5 ** 2)) for x in range(11)],
                     dtype=torch.float32)
    g = g / g.sum()
    w = g.unsqueeze(1).mm(g.unsqueeze(1).t()).float()
    return w.expand(3, 1, 11, 11).contiguous().to(device)


def torch_loss(layer, pal, tgt, win):
    img = torch.einsum("kc,khw->chw", pal, layer)
    mu1 = F.conv2d(img, win, padding=5, groups=3)
    mu2 = F.conv2d(tgt, win, padding=5, groups=3)
    s1 = F.conv2d(img * img, win, padding=5, groups=3) - mu1 * mu1
    s2 = F.conv2d(tgt * tgt, win, padding=5, groups=3) - mu2 * mu2
    s12 = F.conv2d(img * tgt, win, padding=5, groups=3) - mu1 * mu2
    C1, C2 = 0.01 ** 2, 0.03 ** 2
    ssim = (((2 * mu1 * mu2 + C1) * (2 * s12 + C2)) /
            ((mu1 * mu1 + mu2 * mu2 + C1) * (s1 + s2 + C2))).mean()
    return 0.8 * (img - tgt).abs().mean() + 0.2 * (1 - ssim) + 0.5 * F.relu(-layer).mean()


def median_ms(fn, reps):
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        e.synchronize()
        ts.append(s.elapsed_time(e))
    return statistics.median(ts)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--reps", type=int, default=50)
    ap.add_argument("--only-fused", action="store_true", help="skip the torch-operator form")
    a = ap.parse_args()
    from palette_b200.loss import palette_l1_ssim_loss
    dev = torch.device("cuda")
    g = torch.Generator("cuda").manual_seed(0)
    K, H, W = 5, a.height, a.width
    layer = (torch.rand((K, H, W), device=dev, generator=g) * 0.6 - 0.1).requires_grad_()
    pal = torch.rand((K, 3), device=dev, generator=g).requires_grad_()
    tgt = torch.rand((3, H, W), device=dev, generator=g)

    def fused():
        layer.grad = pal.grad = None
        palette_l1_ssim_loss(layer, pal, tgt, 0.2, 0.5).backward()
    out = dict(width=W, height=H, K=K, fused_ms=round(median_ms(fused, a.reps), 4))
    if not a.only_fused:
        win = torch_window(dev)

        def ops():
            layer.grad = pal.grad = None
            torch_loss(layer, pal, tgt, win).backward()
        out["torch_ops_ms"] = round(median_ms(ops, a.reps), 4)
        out["speedup"] = round(out["torch_ops_ms"] / out["fused_ms"], 2)
        # the two agree
        fused()
        g1, p1 = layer.grad.clone(), pal.grad.clone()
        ops()
        out["dlayer_rel_diff"] = float((g1 - layer.grad).norm() / layer.grad.norm())
        out["dpalette_rel_diff"] = float((p1 - pal.grad).norm() / pal.grad.norm())
    print(json.dumps(out))


if __name__ == "__main__":
    main()
