"""Generate golden vectors by running the REFERENCE gsplatcu extension on a GPU.

The reference ships no tests or golden data, so its outputs on small seeded
inputs are captured here (once, on a B200, from the build that
oracle/build_ref.py makes under oracle/_ref) and committed as
tests/golden/*.npz.  tests/test_golden.py then pins the CPU oracle to them
without a GPU.  Cases follow the reference's own call sequences
(gsplat/gsmodel.py:13-26, 107-143, 155-200): every geometry op with and
without Jacobians, sh2Weight / sh2Weight_fast(_B) / sh2Color, splat_weight(_B)
and splat_color(_B), plus the 4-Gaussian fixture of gsplat/gau_io.py:180-204.

    python tests/golden/make_golden.py --out <directory for the .npz files>
"""
import argparse
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "reparamgs-palette_b200"), os.path.join(ROOT, "tests")]

from oracle.build_ref import load_ref  # noqa: E402
from palette_b200.scene import look_at, synthetic_scene, to_torch  # noqa: E402
from helpers import example_scene  # noqa: E402


def npy(t):
    return t.detach().cpu().numpy()


def cam_fields(cam):
    return dict(Rcw=npy(cam.Rcw), tcw=npy(cam.tcw), twc=npy(cam.twc),
                cam=np.array([cam.fx, cam.fy, cam.cx, cam.cy, cam.width, cam.height], np.float64))


def geometry(ref, st, cam, out):
    us, pcs, d, du = ref.project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, True)
    out.update(us=npy(us), pcs=npy(pcs), depths_proj=npy(d), du_dpcs=npy(du))
    c3, dr, ds = ref.computeCov3D(st["rots"], st["scales"], d, True)
    out.update(cov3ds=npy(c3), dcov3d_drots=npy(dr), dcov3d_dscales=npy(ds))
    c2, d3, dp = ref.computeCov2D(c3, pcs, cam.Rcw, d, cam.fx, cam.fy, cam.width, cam.height, True)
    out.update(cov2ds=npy(c2), dcov2d_dcov3ds=npy(d3), dcov2d_dpcs=npy(dp))
    cinv, areas, dci = ref.inverseCov2D(c2, d, True)
    out.update(cinv2ds=npy(cinv), areas_pre=npy(areas), depths_pre=npy(d), dcinv2d_dcov2ds=npy(dci))
    return us, cinv, d, areas


def case_full(ref, n, W, H, seed):
    sc = synthetic_scene(n, seed=seed)
    st = to_torch(sc)
    cam = look_at((1.0, -8.0, 0.5), width=W, height=H)
    out = dict(pws=sc["pws"], rots=sc["rots"], scales=sc["scales"], alphas=sc["alphas"],
               shs=sc["shs"], **cam_fields(cam))
    us, cinv, d, areas = geometry(ref, st, cam, out)
    w, dws, dwp = ref.sh2Weight(st["shs"], st["pws"], cam.twc, True, 5)
    out.update(weights=npy(w), dweight_dshs=npy(dws), dweight_dpws=npy(dwp))
    layer, contrib, ft, ranges, gsid = ref.splat_weight(H, W, 5, us, cinv, st["alphas"], d, w, areas)
    out.update(layer=npy(layer), contrib=npy(contrib), final_tau=npy(ft), ranges=npy(ranges),
               gsid=npy(gsid), depths_post=npy(d), areas_post=npy(areas))
    g = torch.randn((5, H, W), device="cuda", generator=torch.Generator("cuda").manual_seed(seed))
    dW, = ref.splat_weight_B(H, W, 5, us, cinv, st["alphas"], d, w, contrib, ft, ranges, gsid, g)
    out.update(dloss_dlayer=npy(g), dweights=npy(dW))
    return out


def case_lowrank(ref, n, seed):
    sc = synthetic_scene(n, seed=seed, mode="lowrank", rank=1)
    st = to_torch(sc)
    A, B = st["A"][:, :, 0].contiguous(), st["B"][:, 0, :].contiguous()
    cam = look_at((0.5, -7.0, 1.0), width=64, height=64)
    w, ddc, ylm = ref.sh2Weight_fast(st["dc"], A, B, st["pws"], cam.twc, True, 5, 15)
    dw = torch.randn((n, 5), device="cuda", generator=torch.Generator("cuda").manual_seed(seed))
    dA, dB = ref.sh2Weight_fast_B(A, B, ylm, dw, 5, 15)
    return dict(pws=sc["pws"], dc=sc["dc"], A=npy(A), B=npy(B), weights=npy(w), dweight_ddc=npy(ddc),
                ylm=npy(ylm), dloss_dw=npy(dw), dA=npy(dA), dB=npy(dB), **cam_fields(cam))


def case_color(ref, pws, rots, scales, alphas, shs, W, H, eye, target, seed):
    st = dict(pws=torch.from_numpy(pws).cuda(), rots=torch.from_numpy(rots).cuda(),
              scales=torch.from_numpy(scales).cuda(), alphas=torch.from_numpy(alphas).cuda())
    cam = look_at(eye, target=target, width=W, height=H)
    out = dict(pws=pws, rots=rots, scales=scales, alphas=alphas, shs=shs, **cam_fields(cam))
    us, cinv, d, areas = geometry(ref, st, cam, out)
    col, dcs, dcp = ref.sh2Color(torch.from_numpy(shs).cuda(), st["pws"], cam.twc, True)
    out.update(colors=npy(col), dcolor_dshs=npy(dcs), dcolor_dpws=npy(dcp))
    img, contrib, ft, ranges, gsid = ref.splat_color(H, W, us, cinv, st["alphas"], d, col, areas)
    out.update(image=npy(img), contrib=npy(contrib), final_tau=npy(ft), ranges=npy(ranges),
               gsid=npy(gsid), depths_post=npy(d), areas_post=npy(areas))
    g = torch.randn((3, H, W), device="cuda", generator=torch.Generator("cuda").manual_seed(seed))
    dus, dq, da, dc = ref.splat_color_B(H, W, us, cinv, st["alphas"], d, col, contrib, ft, ranges,
                                        gsid, g)
    out.update(dloss_dimage=npy(g), dus=npy(dus), dcinv2ds=npy(dq), dalphas=npy(da), dcolors=npy(dc))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the .npz files are written to")
    a = ap.parse_args()
    ref = load_ref()
    if ref is None:
        sys.exit("reference build missing: run oracle/build_ref.py first")
    os.makedirs(a.out, exist_ok=True)
    torch.manual_seed(0)
    cases = {}
    cases["full_k5_n1000_64x64"] = case_full(ref, 1000, 64, 64, seed=100)
    cases["full_k5_n600_80x48"] = case_full(ref, 600, 80, 48, seed=103)
    cases["lowrank_r1_n1000"] = case_lowrank(ref, 1000, seed=101)
    ex = example_scene()
    shs_dc = ex["colors_dc"].copy()  # one SH band: shs [N, 3]
    cases["example_color"] = case_color(ref, ex["pws"], ex["rots"], ex["scales"], ex["alphas"], shs_dc,
                                        64, 48, (4.0, 4.0, 3.0), (0.3, 0.3, 0.3), seed=104)
    sc = synthetic_scene(800, seed=102)
    cases["color_sh16_n800_80x48"] = case_color(ref, sc["pws"], sc["rots"], sc["scales"], sc["alphas"],
                                                sc["shs"][:, :48].copy(), 80, 48, (0.0, -8.0, 0.0),
                                                (0.0, 0.0, 0.0), seed=105)
    for name, d in cases.items():
        path = os.path.join(a.out, name + ".npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in d.items()})
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
