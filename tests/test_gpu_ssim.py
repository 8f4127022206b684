"""GPU tests of the fused L1 + SSIM loss kernel (gsb_palette_l1_ssim) against
the FP64 oracle (oracle.palette_l1_ssim_loss / l1_ssim_loss), and of its plain
gau_loss form against the golden vectors of the reference's own gau_loss
(vanilla_3dgs/gsplat/pytorch_ssim.py:64-67, tests/golden/ssim_gau_loss.npz).

Tolerances: the kernel computes in FP32 and sums the per-pixel terms with
atomics, so the loss parts are compared to 2e-6 absolute (means of values in
[0, 1]) and the gradients to 1e-4 of their largest magnitude, elementwise."""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from palette_b200.loss import gau_loss, palette_l1_ssim_loss
from helpers import np_of, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ssim_gau_loss.npz")
LOSS_TOL = 2e-6
GRAD_TOL = 1e-4


def _inputs(K, H, W, seed):
    rng = np.random.default_rng(seed)
    layer = rng.normal(0.2, 0.3, (K, H, W)).astype(np.float32)
    pal = rng.random((K, 3)).astype(np.float32)
    tgt = rng.random((3, H, W)).astype(np.float32)
    return layer, pal, tgt


def _close(a, b, what):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    err = np.abs(a - b).max() / scale
    assert err < GRAD_TOL, f"{what}: max error {err:.3g} of the largest magnitude"


@pytest.mark.parametrize("K,H,W", [(5, 64, 64), (5, 37, 23), (5, 7, 5), (3, 1, 1), (8, 33, 65),
                                   (5, 135, 240), (1, 40, 96)])
def test_palette_l1_ssim_matches_oracle(cuda_ok, K, H, W):
    layer, pal, tgt = _inputs(K, H, W, seed=K * 1000 + H + W)
    ref = orc.palette_l1_ssim_loss(layer, pal, tgt, 0.2, 0.5)
    L = torch.from_numpy(layer).cuda().requires_grad_()
    P = torch.from_numpy(pal).cuda().requires_grad_()
    T = torch.from_numpy(tgt).cuda()
    loss, parts = palette_l1_ssim_loss(L, P, T, 0.2, 0.5, parts=True)
    loss.backward()
    parts = np_of(parts)
    assert abs(float(loss) - ref["loss"]) < LOSS_TOL
    assert abs(parts[1] - ref["l1"]) < LOSS_TOL
    assert abs(parts[2] - ref["ssim"]) < LOSS_TOL
    assert abs(parts[3] - ref["penalty"]) < LOSS_TOL
    _close(np_of(L.grad), ref["dlayer"], "dlayer")
    _close(np_of(P.grad), ref["dpalette"], "dpalette")


def test_gau_loss_matches_reference_golden(cuda_ok):
    z = np.load(GOLDEN)
    keys = sorted({k.rsplit("_", 1)[0] for k in z.files if k.endswith("_x")})
    for key in keys:
        x = torch.from_numpy(z[key + "_x"].astype(np.float32)).cuda().requires_grad_()
        y = torch.from_numpy(z[key + "_y"].astype(np.float32)).cuda()
        loss = gau_loss(x, y)
        loss.backward()
        assert abs(float(loss) - float(z[key + "_f64_loss"])) < LOSS_TOL, key
        _close(np_of(x.grad), z[key + "_f64_dx"], key)


def test_upstream_gradient_scales_and_large_image_properties(cuda_ok):
    """At 1080p (beyond the oracle's comfortable size): an image against
    itself has SSIM 1, L1 0 and a vanishing gradient; doubling the upstream
    gradient doubles the parameter gradients; the penalty is 0 for
    non-negative weights."""
    K, H, W = 5, 1080, 1920
    g = torch.Generator("cuda").manual_seed(3)
    img = torch.rand((3, H, W), device="cuda", generator=g)
    x = img.clone().requires_grad_()
    loss = gau_loss(x, img)
    assert abs(float(loss)) < 1e-6
    loss.backward()
    assert float(x.grad.abs().max()) < 1e-9
    layer = torch.rand((K, H, W), device="cuda", generator=g)
    pal = torch.rand((K, 3), device="cuda", generator=g)
    # a real target: the gradient is linear in the upstream gradient
    tgt = torch.rand((3, H, W), device="cuda", generator=g)
    L1_ = layer.clone().requires_grad_()
    P1 = pal.clone().requires_grad_()
    loss, parts = palette_l1_ssim_loss(L1_, P1, tgt, parts=True)
    assert float(parts[3]) == 0.0
    loss.backward()
    L2_ = layer.clone().requires_grad_()
    P2 = pal.clone().requires_grad_()
    (2.0 * palette_l1_ssim_loss(L2_, P2, tgt)).backward()
    assert rel_err(L2_.grad, np_of(2.0 * L1_.grad).astype(np.float64)) < 1e-6
    assert rel_err(P2.grad, np_of(2.0 * P1.grad).astype(np.float64)) < 1e-5


def test_empty_image_and_bad_arguments(cuda_ok):
    L = torch.zeros((5, 0, 16), device="cuda", requires_grad=True)
    P = torch.rand((5, 3), device="cuda")
    T = torch.zeros((3, 0, 16), device="cuda")
    loss = palette_l1_ssim_loss(L, P, T)
    assert float(loss) == 0.0
    with pytest.raises(ValueError):
        palette_l1_ssim_loss(torch.zeros((5, 4, 4), device="cuda"), torch.rand((4, 3), device="cuda"),
                             torch.zeros((3, 4, 4), device="cuda"))
    with pytest.raises(ValueError):
        gau_loss(torch.zeros((5, 4, 4), device="cuda"), torch.zeros((5, 4, 4), device="cuda"))
