"""GPU tests of the autograd layer: splat_palette_weights (the operator forward
with the fused weight-parameter adjoint; the gradients of the reference's
WeightGSFunctionTest / WeightGSFunctionFast, gsplat/gsmodel.py:104-200) and the
fused palette L1 loss, against torch / the CPU oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from palette_b200.weights import splat_palette_weights
from palette_b200.loss import palette_image, palette_l1_loss
from palette_b200.scene import look_at, synthetic_scene, to_torch
from helpers import np_of, rel_err

pytestmark = pytest.mark.gpu


def test_palette_l1_matches_torch(cuda_ok):
    g = torch.Generator("cuda").manual_seed(0)
    K, H, W = 5, 67, 129
    layer = torch.rand((K, H, W), device="cuda", generator=g).requires_grad_()
    pal = torch.rand((K, 3), device="cuda", generator=g).requires_grad_()
    tgt = torch.rand((3, H, W), device="cuda", generator=g)
    loss = palette_l1_loss(layer, pal, tgt)
    loss.backward()
    l2 = layer.detach().clone().requires_grad_()
    p2 = pal.detach().clone().requires_grad_()
    ref = (torch.einsum("kc,khw->chw", p2, l2) - tgt).abs().mean()
    ref.backward()
    assert abs(float(loss) - float(ref)) < 1e-6 * max(1.0, abs(float(ref)))
    assert rel_err(layer.grad, l2.grad) < 1e-6
    assert rel_err(pal.grad, p2.grad) < 1e-5
    img = palette_image(layer.detach(), pal.detach())
    assert rel_err(img, torch.einsum("kc,khw->chw", pal.detach(), layer.detach())) < 1e-6


def _oracle_grads(st, sc, cam, w, layer_grad):
    """dL/dweights of the reference backward through the oracle."""
    from gsplatcu import project, computeCov3D, computeCov2D, inverseCov2D, splat_weight
    H, W = cam.height, cam.width
    us, pcs, d = project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
    c3, = computeCov3D(st["rots"], st["scales"], d, False)
    c2, = computeCov2D(c3, pcs, cam.Rcw, d, cam.fx, cam.fy, W, H, False)
    cinv, areas = inverseCov2D(c2, d, False)
    layer, contrib, ft, ranges, gsid = splat_weight(H, W, 5, us, cinv, st["alphas"], d, w, areas)
    r = orc.draw_backward(H, W, 5, np_of(ranges), np_of(gsid), np_of(us), np_of(cinv),
                          np_of(st["alphas"]), np_of(w), np_of(ft), np_of(contrib), np_of(layer_grad))
    return r["dfeat"]


@pytest.mark.parametrize("rank", [1, 3])
def test_splat_palette_weights_lowrank_gradients(cuda_ok, rank):
    sc = synthetic_scene(6000, seed=60 + rank, mode="lowrank", rank=rank)
    st = to_torch(sc)
    cam = look_at((0.5, -7.5, 1.0), width=96, height=80)
    A, B = st["A"], st["B"]
    if rank == 1:
        A, B = A[:, :, 0].contiguous(), B[:, 0, :].contiguous()
    dc, A, B = st["dc"].requires_grad_(), A.requires_grad_(), B.requires_grad_()
    layer, mask = splat_palette_weights(st["pws"], st["alphas"], st["scales"], st["rots"], cam,
                                        dc=dc, A=A, B=B)
    G = torch.randn_like(layer)
    (layer * G).sum().backward()
    import gsplatcu as gsc
    w, ddc, ylm = gsc.sh2Weight_fast(dc.detach(), A.detach(), B.detach(), st["pws"], cam.twc, True, 5, 15)
    dw = _oracle_grads(st, sc, cam, w, G)
    twc = orc.camera_arrays(cam, np.float32)[2]
    o_dA, o_dB = orc.sh2weight_fast_b(np_of(A), np_of(B), np_of(ylm), dw, 5, 15)
    assert rel_err(dc.grad, dw * np.float32(0.28209479177387814)) < 1e-4
    assert rel_err(A.grad, o_dA) < 1e-4 and rel_err(B.grad, o_dB) < 1e-4
    assert mask.dtype == torch.bool and mask.shape == (6000,)


def test_splat_palette_weights_full_sh_gradients(cuda_ok):
    sc = synthetic_scene(6000, seed=70)
    st = to_torch(sc)
    cam = look_at((0.5, -7.5, 1.0), width=96, height=80)
    shs = st["shs"].requires_grad_()
    layer, mask = splat_palette_weights(st["pws"], st["alphas"], st["scales"], st["rots"], cam,
                                        shs=shs)
    G = torch.randn_like(layer)
    (layer * G).sum().backward()
    import gsplatcu as gsc
    w, dshs, _ = gsc.sh2Weight(shs.detach(), st["pws"], cam.twc, True, 5)
    dw = _oracle_grads(st, sc, cam, w, G)
    expect = (dw[:, None, :] * np_of(dshs)[:, 0, :, None]).reshape(6000, -1)  # [N,16,K] outer
    assert rel_err(shs.grad, expect) < 1e-4


@pytest.mark.parametrize("clamp,kind", [(False, "mse"), (True, "mse"), (True, "l1")])
def test_palette_geo_loss_matches_oracle(cuda_ok, clamp, kind):
    """The finetune loss kernel (barycentric target + MSE/L1 + negative-weight
    penalty) against the FP64 oracle: loss, target weights, and both
    gradients (weights; chromatic palette through the target)."""
    from oracle import oracle as orc
    from palette_b200.loss import barycentric_target, palette_geo_loss
    g = torch.Generator().manual_seed(11)
    H, W = 96, 128
    chroma = torch.tensor([[0.85, 0.2, 0.15], [0.2, 0.75, 0.3], [0.25, 0.2, 0.85]]) + \
        0.03 * torch.randn((3, 3), generator=g)
    target = torch.rand((3, H, W), generator=g) * 0.9 + 0.05
    layer = torch.randn((5, H, W), generator=g) * 0.3 + 0.2
    ref = orc.palette_geo_loss(layer.double().numpy(), target.double().numpy(),
                               chroma.double().numpy(), clamp=clamp, kind=kind)
    L = layer.cuda().requires_grad_(True)
    P = chroma.cuda().requires_grad_(True)
    loss = palette_geo_loss(L, P, target.cuda(), clamp=clamp, lambda_pos=0.5, kind=kind)
    loss.backward()
    assert abs(float(loss) - ref["loss"]) < 1e-5 * max(1.0, abs(ref["loss"]))
    wb = barycentric_target(target.cuda(), chroma.cuda(), clamp=clamp)
    same = np.abs(np_of(wb) - ref["target_weights"]).max(axis=0) < 1e-4
    assert same.mean() > 0.999  # pixels on a tetrahedron boundary may pick the other one
    assert rel_err(L.grad, ref["dlayer"]) < 1e-4
    assert rel_err(P.grad, ref["dchroma"]) < 1e-3


@pytest.mark.parametrize("clamp,kind", [(True, "l1"), (False, "mse")])
def test_palette_geo_loss_tied_tetrahedra(cuda_ok, clamp, kind):
    """With two chroma colours the two tetrahedra (black, white, c0, c1) and
    (black, white, c1, c0) are the same solid, so every pixel's errors tie and
    the kernel takes its general (non-one-hot) path everywhere; achromatic and
    white pixels are mixed in.  The target is the same whatever the softmax
    weights, so loss, target weights and dL/dlayer match the FP64 oracle.
    (dL/dpalette is not compared: on exact ties the softmax term divides
    FP32 rounding differences by the 1e-9 temperature.)"""
    from oracle import oracle as orc
    from palette_b200.loss import barycentric_target, palette_geo_loss
    g = torch.Generator().manual_seed(4)
    H, W = 64, 96
    chroma = torch.rand((2, 3), generator=g) * 0.8 + 0.1
    target = torch.rand((3, H, W), generator=g)
    grey = torch.rand((H, W), generator=g) < 0.3
    target[:, grey] = target[0, grey]
    target[:, :3, :] = 1.0
    layer = torch.randn((4, H, W), generator=g) * 0.3 + 0.2
    ref = orc.palette_geo_loss(layer.double().numpy(), target.double().numpy(),
                               chroma.double().numpy(), clamp=clamp, kind=kind)
    L = layer.cuda().requires_grad_(True)
    P = chroma.cuda().requires_grad_(True)
    loss = palette_geo_loss(L, P, target.cuda(), clamp=clamp, lambda_pos=0.5, kind=kind)
    loss.backward()
    assert abs(float(loss) - ref["loss"]) < 1e-5 * max(1.0, abs(ref["loss"]))
    wb = barycentric_target(target.cuda(), chroma.cuda(), clamp=clamp)
    assert np.abs(np_of(wb) - ref["target_weights"]).max() < 1e-4
    assert rel_err(L.grad, ref["dlayer"]) < 1e-4
    assert bool(torch.isfinite(P.grad).all())
