"""The drop-in claim, tested with the reference's own caller.

The reference's ``gsplat/gsmodel.py`` (with the ``gsplat/utils.py`` it
imports), staged unchanged into ``oracle/_ref/gsplat`` by
``oracle/build_ref.py``, is executed twice: once with ``import gsplatcu``
resolving to this build's drop-in module and once to the reference's own
extension built from its sources (``oracle/_ref/gsplatcu_ref.so``).  Its
autograd functions ``WeightGSFunctionTest`` (gsmodel.py:104-143) and
``WeightGSFunctionFast`` (gsmodel.py:151-200), ``FinetuneModel``
(gsmodel.py:292-329) with the parameters ``get_finetune_params`` creates
(gsmodel.py:379-485), and the palette-edit render ``bake_palette_edit`` +
``render_vanilla`` (gsmodel.py:488-509, 13-26) then run on identical inputs.

Tolerances: visibility masks equal; rendered layers and images within 1e-5
abs (FP32 storage, the north-star image bound); every gradient within 1e-4
relative (norm-wise per tensor)."""
import numpy as np
import pytest
import torch

import gsplatcu
from oracle.build_ref import load_ref, reference_caller
from palette_b200.scene import look_at, synthetic_scene
from helpers import max_abs, rel_err

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
GRAD_TOL = 1e-4


@pytest.fixture(scope="module")
def callers(cuda_ok):
    ref = load_ref()
    if ref is None:
        pytest.skip("reference build oracle/_ref/gsplatcu_ref.so is missing")
    mine = reference_caller(gsplatcu, "b200")
    theirs = reference_caller(ref, "ref")
    if mine is None or theirs is None:
        pytest.skip("reference caller oracle/_ref/gsplat is not staged")
    assert mine.gsc is gsplatcu and theirs.gsc is ref
    return mine, theirs


def _scene(n, seed, mode):
    sc = synthetic_scene(n, seed=seed, mode=mode, rank=1)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    out = dict(pws=t(sc["pws"]), rots=t(sc["rots"]), scales=t(sc["scales"]),
               alphas=t(sc["alphas"]), palette=t(sc["palette"]))
    if mode == "full":
        out["shs"] = t(sc["shs"])
    else:
        out.update(dc=t(sc["dc"]), A=t(sc["A"][:, :, 0]), B=t(sc["B"][:, 0, :]))
    return out


def _leaf(x):
    return x.detach().clone().requires_grad_()


CASES = [(20000, 256, 256, 11), (200000, 1920, 1080, 12)]


@pytest.mark.parametrize("n,W,H,seed", CASES)
def test_weight_function_test_full_sh(callers, n, W, H, seed):
    s = _scene(n, seed, "full")
    cam = look_at((0.5, -8.0, 1.0), width=W, height=H)
    dl = torch.randn((5, H, W), device="cuda", generator=torch.Generator("cuda").manual_seed(seed))
    res = []
    for gm in callers:
        shs = _leaf(s["shs"])
        layer, mask = gm.WeightGSFunctionTest.apply(s["pws"], shs, s["alphas"], s["scales"],
                                                    s["rots"], cam, 5)
        layer.backward(dl)
        res.append((layer.detach(), mask, shs.grad))
    (la, ma, ga), (lb, mb, gb) = res
    assert torch.equal(ma, mb)
    assert max_abs(la, lb) < IMG_TOL
    assert rel_err(ga, gb) < GRAD_TOL


@pytest.mark.parametrize("n,W,H,seed", CASES)
def test_weight_function_fast_rank1(callers, n, W, H, seed):
    s = _scene(n, seed, "lowrank")
    cam = look_at((-1.0, -7.5, 0.5), width=W, height=H)
    dl = torch.randn((5, H, W), device="cuda", generator=torch.Generator("cuda").manual_seed(seed))
    res = []
    for gm in callers:
        dc, A, B = _leaf(s["dc"]), _leaf(s["A"]), _leaf(s["B"])
        layer, mask = gm.WeightGSFunctionFast.apply(s["pws"], dc, A, B, s["alphas"], s["scales"],
                                                    s["rots"], cam, 5, 15)
        layer.backward(dl)
        res.append((layer.detach(), mask, dc.grad, A.grad, B.grad))
    a, b = res
    assert torch.equal(a[1], b[1])
    assert max_abs(a[0], b[0]) < IMG_TOL
    for ga, gb in zip(a[2:], b[2:]):
        assert rel_err(ga, gb) < GRAD_TOL


@pytest.mark.parametrize("mode", ["full", "lowrank"])
def test_own_autograd_matches_reference_caller(callers, mode):
    """palette_b200.weights.splat_palette_weights (operator forward, fused
    weight-parameter adjoint) against the reference's own autograd function
    on the reference build: same layers, same mask, same gradients."""
    from palette_b200.weights import splat_palette_weights
    n, W, H = 200000, 1920, 1080
    s = _scene(n, 41, mode)
    cam = look_at((1.5, -7.0, 2.0), width=W, height=H)
    dl = torch.randn((5, H, W), device="cuda", generator=torch.Generator("cuda").manual_seed(4))
    theirs = callers[1]
    if mode == "full":
        shs_a, shs_b = _leaf(s["shs"]), _leaf(s["shs"])
        la, ma = splat_palette_weights(s["pws"], s["alphas"], s["scales"], s["rots"], cam, shs=shs_a)
        lb, mb = theirs.WeightGSFunctionTest.apply(s["pws"], shs_b, s["alphas"], s["scales"],
                                                   s["rots"], cam, 5)
        pairs = [(shs_a, shs_b)]
    else:
        a = [_leaf(s[k]) for k in ("dc", "A", "B")]
        b = [_leaf(s[k]) for k in ("dc", "A", "B")]
        la, ma = splat_palette_weights(s["pws"], s["alphas"], s["scales"], s["rots"], cam,
                                       dc=a[0], A=a[1], B=a[2])
        lb, mb = theirs.WeightGSFunctionFast.apply(s["pws"], b[0], b[1], b[2], s["alphas"],
                                                   s["scales"], s["rots"], cam, 5, 15)
        pairs = list(zip(a, b))
    la.backward(dl)
    lb.backward(dl)
    assert torch.equal(ma, mb)
    assert max_abs(la, lb) < IMG_TOL
    for x, y in pairs:
        assert rel_err(x.grad, y.grad) < GRAD_TOL


def _finetune_params(gm, s, low_rank):
    """The reference's own parameter set-up (get_finetune_params), then the
    synthetic scene's weights written into its leaf tensors, so that renders
    are not the near-zero images of its 1e-3 initialisation."""
    n = int(s["pws"].shape[0])
    gs = dict(pw=s["pws"].cpu().numpy(), rot=s["rots"].cpu().numpy(),
              scale=s["scales"].cpu().numpy(), alpha=s["alphas"].cpu().numpy(),
              sh=np.zeros((n, 48), np.float32))
    torch.manual_seed(0)
    frozen, params, _ = gm.get_finetune_params(gs, num_palette=3, low_rank=low_rank,
                                               reshape_Q=15 if low_rank else None,
                                               init_palette_rgb=s["palette"][2:].cpu().numpy())
    with torch.no_grad():
        if low_rank:
            params["low_shs_w"].copy_(s["dc"])
            params["high_shs_A"].copy_(s["A"])
            params["high_shs_B"].copy_(s["B"])
        else:
            params["low_shs_w"].copy_(s["shs"][:, :5])
            params["high_shs_w"].copy_(s["shs"][:, 5:])
    return frozen, params


@pytest.mark.parametrize("low_rank", [False, True])
def test_finetune_model_forward_backward(callers, low_rank):
    n, W, H = 100000, 1280, 720
    s = _scene(n, 21, "lowrank" if low_rank else "full")
    cam = look_at((2.0, -7.0, 1.5), width=W, height=H)
    target = torch.rand((3, H, W), device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    res = []
    for gm in callers:
        frozen, params = _finetune_params(gm, s, low_rank)
        model = gm.FinetuneModel(sh_order=3, num_palette=3, use_fast=True)
        W_tilde, palette_rgb = model(frozen["pws"], params, frozen["alphas"], frozen["scales"],
                                     frozen["rots"], cam)
        P_full = torch.cat([params["black"], params["white"], palette_rgb], 0)
        img = torch.einsum("khw,kc->chw", W_tilde, P_full)
        loss = (img - target).abs().mean() + 0.5 * torch.relu(-W_tilde).mean()
        loss.backward()
        names = ["low_shs_w", "hue_base", "gap_raw", "sat_raw", "lit_raw"] + \
            (["high_shs_A", "high_shs_B"] if low_rank else ["high_shs_w"])
        res.append((W_tilde.detach(), model.mask, float(loss), {k: params[k].grad for k in names}))
    a, b = res
    assert torch.equal(a[1], b[1])
    assert max_abs(a[0], b[0]) < IMG_TOL
    assert abs(a[2] - b[2]) <= 1e-6 * max(1.0, abs(b[2]))
    for k in a[3]:
        assert rel_err(a[3][k], b[3][k]) < GRAD_TOL, k


def test_palette_edit_bake_and_render(callers):
    n, W, H = 200000, 1920, 1080
    s = _scene(n, 31, "full")
    cam = look_at((0.0, -6.5, 2.0), width=W, height=H)
    edit = torch.clamp(s["palette"][2:] + 0.15 * torch.randn(
        (3, 3), device="cuda", generator=torch.Generator("cuda").manual_seed(5)), 0.0, 1.0)
    imgs = []
    for gm in callers:
        frozen, params = _finetune_params(gm, s, False)
        shs = gm.bake_palette_edit(params, frozen, edit)
        imgs.append(gm.render_vanilla(frozen["pws"], shs, frozen["alphas"], frozen["scales"],
                                      frozen["rots"], cam))
    assert max_abs(imgs[0], imgs[1]) < IMG_TOL
