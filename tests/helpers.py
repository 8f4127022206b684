"""Shared test helpers: scenes, the reference operator sequence, comparisons."""
import numpy as np
import torch

from palette_b200.scene import Camera, look_at, synthetic_scene, to_torch

# The reference's only fixture: 4 hand-placed Gaussians (gsplat/gau_io.py:180-204)
# -- centre, quaternion (w,x,y,z), scale, opacity, SH DC colour.
EXAMPLE_GS = np.array([
    [0., 0., 0., 1., 0., 0., 0., 0.05, 0.05, 0.05, 1., 1.772484, -1.772484, 1.772484],
    [1., 0., 0., 1., 0., 0., 0., 0.2, 0.05, 0.05, 1., 1.772484, -1.772484, -1.772484],
    [0., 1., 0., 1., 0., 0., 0., 0.05, 0.2, 0.05, 1., -1.772484, 1.772484, -1.772484],
    [0., 0., 1., 1., 0., 0., 0., 0.05, 0.05, 0.2, 1., -1.772484, -1.772484, 1.772484],
], dtype=np.float32)


def example_scene():
    g = EXAMPLE_GS
    return dict(pws=g[:, 0:3].copy(), rots=g[:, 3:7].copy(), scales=g[:, 7:10].copy(),
                alphas=g[:, 10:11].copy(), colors_dc=g[:, 11:14].copy())


def np_of(t):
    """numpy copy of a tensor: floating types as float32 (numpy has no BF16),
    integer types unchanged (a float32 copy would round them above 2^24)."""
    if not isinstance(t, torch.Tensor):
        return np.asarray(t)
    t = t.detach()
    return (t.float() if t.is_floating_point() else t).cpu().numpy()


def forward_ops(gsc, sc, cam, mode="full"):
    """The WeightGSFunctionTest / WeightGSFunctionFast forward sequence
    (gsplat/gsmodel.py:107-118, 155-170) through operator module `gsc`."""
    K = sc["K"]
    us, pcs, depths = gsc.project(sc["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
    cov3ds, = gsc.computeCov3D(sc["rots"], sc["scales"], depths, False)
    cov2ds, = gsc.computeCov2D(cov3ds, pcs, cam.Rcw, depths, cam.fx, cam.fy, cam.width,
                               cam.height, False)
    out = dict(us=us, pcs=pcs, cov3ds=cov3ds, cov2ds=cov2ds)
    if mode == "full":
        w, dwdshs, _ = gsc.sh2Weight(sc["shs"], sc["pws"], cam.twc, True, K)
        out.update(weights=w, dweight_dshs=dwdshs)
    else:
        w, ddc, ylm = gsc.sh2Weight_fast(sc["dc"], sc["A"], sc["B"], sc["pws"], cam.twc, True, K,
                                         sc["Q"])
        out.update(weights=w, dweight_ddc=ddc, ylm=ylm)
    cinv, areas = gsc.inverseCov2D(cov2ds, depths, False)
    layer, contrib, ft, ranges, gsid = gsc.splat_weight(cam.height, cam.width, K, out["us"], cinv,
                                                       sc["alphas"], depths, out["weights"], areas)
    out.update(cinv=cinv, areas=areas, depths=depths, layer=layer, contrib=contrib,
               final_tau=ft, ranges=ranges, gsid=gsid)
    return out


def max_abs(a, b):
    a, b = np_of(a).astype(np.float64), np_of(b).astype(np.float64)
    return float(np.max(np.abs(a - b))) if a.size else 0.0


def rel_err(a, b):
    a, b = np_of(a).astype(np.float64).ravel(), np_of(b).astype(np.float64).ravel()
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a))
