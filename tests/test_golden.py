"""Pin the CPU oracle to golden vectors produced by the reference extension
itself (tests/golden/make_golden.py, run on a B200 against the reference
build).  CPU only.  Geometry (centres, camera-space points, 3D and 2D
covariances, conics, extents, depth updates): bit-exact, the oracle's FP32
instantiation follows the reference build's operation order including its
fused multiply-adds; tile lists, ranges, contributor indices and in-place
updates: bit-exact; images within 1e-5; Jacobians and SH values (the
reference evaluates SH with FP64 constants): FP32 tolerances."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as orc

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


class _Cam:
    def __init__(self, z):
        self.Rcw, self.tcw = z["Rcw"], z["tcw"]
        self.fx, self.fy, self.cx, self.cy, w, h = [float(v) for v in z["cam"]]
        self.width, self.height = int(w), int(h)


def _bits(a, b, live=None):
    """Bitwise equality of FP32 arrays (on the rows in `live`)."""
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    if live is not None:
        a, b = a[live], b[live]
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), \
        float(np.mean(a.view(np.uint32) == b.view(np.uint32)))


def _close(a, b, rtol, atol, frac=1.0):
    ok = np.isclose(a, b, rtol=rtol, atol=atol)
    assert ok.mean() >= frac, (float(ok.mean()), float(np.max(np.abs(a - b))))


def test_golden_fixtures_present():
    names = {os.path.basename(p) for p in GOLDEN}
    assert "full_k5_n1000_64x64.npz" in names, "golden vectors missing"
    assert "lowrank_r1_n1000.npz" in names and "example_color.npz" in names


def _check_geometry(z):
    cam = _Cam(z)
    Rcw, tcw = z["Rcw"].astype(np.float32), z["tcw"].astype(np.float32)
    us, pcs, d, du = orc.project(z["pws"], Rcw, tcw, cam.fx, cam.fy, cam.cx, cam.cy, True)
    live = z["depths_proj"] >= 0.2
    _bits(us, z["us"], live)
    _bits(pcs, z["pcs"], live)
    _bits(d, z["depths_proj"])
    assert _rel(du, z["du_dpcs"]) < 1e-6
    c3, dr, ds = orc.cov3d(z["rots"], z["scales"], z["depths_proj"], True)
    _bits(c3, z["cov3ds"], live)
    # Jacobians: norm-wise (entries with cancellation round differently with FMA)
    assert _rel(dr, z["dcov3d_drots"]) < 1e-5
    assert _rel(ds, z["dcov3d_dscales"]) < 1e-5
    c2, d3, dp = orc.cov2d(z["cov3ds"], z["pcs"], Rcw, z["depths_proj"], cam.fx, cam.fy, cam.width,
                           cam.height, True)
    _bits(c2, z["cov2ds"], live)
    assert _rel(d3, z["dcov2d_dcov3ds"]) < 1e-5
    assert _rel(dp, z["dcov2d_dpcs"]) < 1e-4
    d2 = z["depths_proj"].copy()
    ci, ar, dci = orc.inverse_cov2d(z["cov2ds"], d2, True)
    assert np.array_equal(d2, z["depths_pre"])
    _bits(ci, z["cinv2ds"], live)
    assert np.array_equal(ar[live], z["areas_pre"][live])
    assert _rel(dci, z["dcinv2d_dcov2ds"]) < 1e-5
    return cam


def _check_splat(z, K, feats, out_key, dkey, tau_init):
    cam = _cam_hw(z)
    H, W = cam
    d, a = z["depths_pre"].copy(), z["areas_pre"].copy()
    b = orc.bin_gaussians(z["us"], a, d, H, W)
    assert np.array_equal(b["gsid"], z["gsid"]), "tile lists differ from the reference"
    assert np.array_equal(b["ranges"], z["ranges"]), "tile ranges differ from the reference"
    assert np.array_equal(d, z["depths_post"]) and np.array_equal(a, z["areas_post"])
    out, contrib, ft = orc.draw(H, W, K, z["ranges"], z["gsid"], z["us"], z["cinv2ds"], z["alphas"],
                                feats, tau_init)
    assert np.array_equal(contrib, z["contrib"])
    assert np.max(np.abs(out - z[out_key])) < 1e-5
    assert np.max(np.abs(ft - z["final_tau"])) < 1e-5
    return out, contrib, ft


def _cam_hw(z):
    c = z["cam"]
    return int(c[5]), int(c[4])


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("path", [p for p in GOLDEN if "full_k5" in p])
def test_oracle_matches_reference_full_weights(path):
    z = dict(np.load(path))
    _check_geometry(z)
    twc = z["twc"].astype(np.float32)
    w, dws, dwp = orc.sh2feat(z["shs"], z["pws"], twc, 5, True, ref_quirk=True)
    _close(w, z["weights"], 1e-5, 2e-7)
    _close(dws, z["dweight_dshs"], 1e-5, 2e-7)
    assert _rel(dwp, z["dweight_dpws"]) < 1e-5
    H, W = _cam_hw(z)
    _, contrib, ft = _check_splat(z, 5, z["weights"], "layer", "weights", 0.0)
    g = orc.draw_backward(H, W, 5, z["ranges"], z["gsid"], z["us"], z["cinv2ds"], z["alphas"],
                          z["weights"], z["final_tau"], z["contrib"], z["dloss_dlayer"])
    assert _rel(g["dfeat"], z["dweights"][:, 0]) < 1e-4


@pytest.mark.parametrize("path", [p for p in GOLDEN if "lowrank" in p])
def test_oracle_matches_reference_lowrank(path):
    z = dict(np.load(path))
    twc = z["twc"].astype(np.float32)
    w, ddc, ylm = orc.sh2weight_fast(z["dc"], z["A"], z["B"], z["pws"], twc, 5, 15, True)
    _close(w, z["weights"], 1e-5, 1e-7)
    _close(ylm, z["ylm"], 1e-5, 1e-7)
    assert np.allclose(ddc, z["dweight_ddc"])
    dA, dB = orc.sh2weight_fast_b(z["A"], z["B"], z["ylm"], z["dloss_dw"], 5, 15)
    assert _rel(dA, z["dA"]) < 1e-5 and _rel(dB, z["dB"]) < 1e-5


@pytest.mark.parametrize("path", [p for p in GOLDEN if "color" in p])
def test_oracle_matches_reference_color(path):
    z = dict(np.load(path))
    _check_geometry(z)
    twc = z["twc"].astype(np.float32)
    col, dcs, dcp = orc.sh2feat(z["shs"], z["pws"], twc, 3, True, ref_quirk=True)
    _close(col, z["colors"], 1e-5, 2e-7)
    assert _rel(dcp, z["dcolor_dpws"]) < 1e-5
    H, W = _cam_hw(z)
    _check_splat(z, 3, z["colors"], "image", "colors", 1.0)
    g = orc.draw_backward(H, W, 3, z["ranges"], z["gsid"], z["us"], z["cinv2ds"], z["alphas"],
                          z["colors"], z["final_tau"], z["contrib"], z["dloss_dimage"])
    assert _rel(g["dfeat"], z["dcolors"][:, 0]) < 1e-4
    assert _rel(g["dalpha"], z["dalphas"].reshape(-1)) < 1e-4
    assert _rel(g["du"], z["dus"][:, 0]) < 1e-4
    assert _rel(g["dconic"], z["dcinv2ds"][:, 0]) < 1e-4
