"""CPU checks of the oracle's palette-weight loss (oracle.palette_geo_loss):
the barycentric target reconstructs the pixel colour, and the analytic
gradients w.r.t. the rendered weights and the chromatic palette match central
finite differences in FP64 (clamped and unclamped; MSE and L1)."""
import numpy as np
import pytest

from oracle import oracle as orc


def _case(H=6, W=7, seed=0):
    rng = np.random.default_rng(seed)
    chroma = np.array([[0.9, 0.2, 0.15], [0.15, 0.8, 0.25], [0.2, 0.25, 0.9]]) + \
        rng.normal(0, 0.03, (3, 3))
    target = rng.uniform(0.05, 0.95, (3, H, W))
    layer = rng.normal(0.2, 0.3, (5, H, W))
    return layer, target, chroma


def test_unclamped_target_reconstructs_colour():
    layer, target, chroma = _case()
    r = orc.palette_geo_loss(layer, target, chroma, clamp=False)
    Wb = r["target_weights"].reshape(5, -1)
    pal = np.concatenate([np.zeros((1, 3)), np.ones((1, 3)), chroma])
    recon = pal.T @ Wb  # sum_k W_k P_k
    assert np.allclose(recon, target.reshape(3, -1), atol=1e-9)
    assert np.allclose(Wb.sum(0), 1.0, atol=1e-9)


@pytest.mark.parametrize("clamp,kind", [(True, "mse"), (False, "mse"), (True, "l1")])
def test_gradients_match_finite_differences(clamp, kind):
    layer, target, chroma = _case(seed=3)
    r = orc.palette_geo_loss(layer, target, chroma, clamp=clamp, kind=kind)
    f = lambda L, P: orc.palette_geo_loss(L, target, P, clamp=clamp, kind=kind)["loss"]
    eps = 1e-6
    for idx in [(0, 0, 0), (2, 3, 4), (4, 5, 6), (1, 2, 2)]:
        Lp, Lm = layer.copy(), layer.copy()
        Lp[idx] += eps
        Lm[idx] -= eps
        fd = (f(Lp, chroma) - f(Lm, chroma)) / (2 * eps)
        assert abs(fd - r["dlayer"][idx]) < 1e-7, (idx, fd, r["dlayer"][idx])
    for a in range(3):
        for c in range(3):
            Pp, Pm = chroma.copy(), chroma.copy()
            Pp[a, c] += eps
            Pm[a, c] -= eps
            fd = (f(layer, Pp) - f(layer, Pm)) / (2 * eps)
            assert abs(fd - r["dchroma"][a, c]) < 1e-6 * max(1.0, abs(fd)), (a, c, fd,
                                                                            r["dchroma"][a, c])
