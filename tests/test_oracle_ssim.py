"""The L1 + SSIM loss oracle (oracle.l1_ssim_loss, palette_l1_ssim_loss)
pinned to golden vectors made by the reference's own gau_loss
(vanilla_3dgs/gsplat/pytorch_ssim.py:26-67, tests/golden/make_ssim_golden.py),
and its palette form checked by central differences.  CPU only."""
import os

import numpy as np
import pytest

from oracle import oracle as orc

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ssim_gau_loss.npz")


def _cases():
    z = np.load(GOLDEN)
    return z, sorted({k.rsplit("_", 1)[0] for k in z.files if k.endswith("_x")})


def test_oracle_matches_reference_gau_loss_fp64():
    z, keys = _cases()
    assert len(keys) == 4
    for key in keys:
        r = orc.l1_ssim_loss(z[key + "_x"], z[key + "_y"], lambda_ssim=0.2)
        assert abs(r["loss"] - float(z[key + "_f64_loss"])) < 1e-12, key
        np.testing.assert_allclose(r["dimage"], z[key + "_f64_dx"], rtol=0, atol=1e-15)


def test_oracle_matches_reference_gau_loss_fp32_within_rounding():
    z, keys = _cases()
    for key in keys:
        r = orc.l1_ssim_loss(z[key + "_x"].astype(np.float32), z[key + "_y"].astype(np.float32))
        assert abs(r["loss"] - float(z[key + "_f32_loss"])) < 2e-6, key
        g = z[key + "_f32_dx"]
        assert np.abs(r["dimage"] - g).max() < 1e-4 * np.abs(g).max() + 1e-9, key


def test_palette_form_central_differences():
    rng = np.random.default_rng(7)
    K, H, W = 5, 13, 17
    layer = rng.normal(0.2, 0.3, (K, H, W))
    pal = rng.random((K, 3))
    tgt = rng.random((3, H, W))
    r = orc.palette_l1_ssim_loss(layer, pal, tgt, 0.2, 0.5)
    f = lambda L, P: orc.palette_l1_ssim_loss(L, P, tgt, 0.2, 0.5)["loss"]
    h = 1e-7
    for idx in [(0, 3, 4), (2, 0, 0), (4, 12, 16), (1, 6, 9)]:
        if abs(layer[idx]) < 1e-3:
            continue
        e = np.zeros_like(layer)
        e[idx] = h
        fd = (f(layer + e, pal) - f(layer - e, pal)) / (2 * h)
        assert abs(fd - r["dlayer"][idx]) < 1e-6 * max(1.0, abs(fd)) + 1e-9, idx
    for idx in [(0, 0), (2, 1), (4, 2)]:
        e = np.zeros_like(pal)
        e[idx] = h
        fd = (f(layer, pal + e) - f(layer, pal - e)) / (2 * h)
        assert abs(fd - r["dpalette"][idx]) < 1e-6 * max(1.0, abs(fd)) + 1e-9, idx
