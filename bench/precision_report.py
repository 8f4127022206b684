#!/usr/bin/env python
"""Precision of the B200 path against the FP64 oracle: FP32 and BF16 storage.

Scene: 3M Gaussians drawn as the benchmark scenes, full palette weights
[N,16,5] at SH order 3.  For each of `--poses` seeded poses on a sphere of
radius 8 and each resolution, the fused forward (palette_b200.render) runs
with the weights stored in FP32 and in BF16 (all arithmetic FP32); the CPU
oracle renders the same view in FP64 from the FP32 parameters (the BF16 error
therefore includes the storage rounding).  The FP64 composite covers every
`--tile-stride`-th tile (tiles are independent given the tile lists), and the
errors are taken over those tiles: max / mean abs error of the K-channel
weight image and of the palette colour image, and PSNR (peak 1).  Gradients:
for the first `--grad-poses` poses, every parameter group's relative error
||g - g64|| / ||g64|| of the full adjoint against the oracle's FP64 chain
rule, with dL/dlayer random on the sampled tiles and zero elsewhere -- and
split in two: pixels where the FP32 render and the FP64 oracle take a
different discrete decision (a Gaussian skipped at alpha' < 0.002 in one and
blended in the other, or the T < 1e-4 stop at a different Gaussian: the
contributor index differs, or the final transmittance differs by more than
1e-4 relative, far above FP32 rounding) are found, dL/dlayer is zeroed on
them, and the relative error recomputed: that is the arithmetic part, the
rest is the decision (threshold-flip) part.

With ``--serving`` it instead measures the two storage forms of the serving
benchmark as served: one scene with full SH weights in FP32 and one with
rank-3 low-rank factors in BF16 (``--serve-gaussians`` each, the serving
benchmark's generators), palette-edit requests at 1920x1080 (cameras on a
sphere of radius 6..10, palettes perturbed as in the serving stream) rendered
through ``PaletteServer`` -- per-slot preparation graphs and the persistent
batched compositing kernel -- and each image compared with the FP64 oracle's
palette colour image of the same request, rendered from the FP32 parameters
(so the BF16 error includes the storage rounding), over every
``--tile-stride``-th tile: PSNR (peak 1) and max / mean abs error per form.

Not collected by pytest (it is a report, minutes of CPU time): run it on a
GPU box and keep the printed JSON.

    python bench/precision_report.py [--gaussians 3000000] [--poses 32] [--tile-stride 8]
    python bench/precision_report.py --serving [--serve-gaussians 250000] [--serve-requests 8]
"""
import argparse
import json
import math
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, os.path.join(ROOT, "reparamgs-palette_b200"), HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402
import torch  # noqa: E402


def sampled_lists(orc, pre32, H, W, stride):
    b = orc.bin_gaussians(pre32["us"], pre32["areas"].copy(), pre32["depths"].copy(), H, W)
    ranges = b["ranges"].copy()
    keep = np.zeros(len(ranges), bool)
    keep[::stride] = True
    ranges[~keep] = 0
    gx = (W + 15) // 16
    mask = np.zeros((H, W), bool)
    for t in np.flatnonzero(keep):
        ty, tx = divmod(int(t), gx)
        mask[ty * 16:(ty + 1) * 16, tx * 16:(tx + 1) * 16] = True
    return (ranges, b["gsid"]), mask


def stats(a, b, mask):
    d = np.abs((a - b)[..., mask])
    mse = float(np.mean(d * d))
    return dict(max_abs=float(d.max()), mean_abs=float(d.mean()),
                p9999_abs=float(np.quantile(d, 0.9999)), frac_over_1e5=float(np.mean(d > 1e-5)),
                psnr=float("inf") if mse == 0 else 10 * math.log10(1.0 / mse))


def serving_precision(a):
    """PSNR vs FP64 of the serving path's two storage forms (see module doc)."""
    from oracle import oracle as orc
    from palette_b200.scene import look_at, sphere_poses, synthetic_scene, to_torch
    from palette_b200.serve import PaletteServer, Request, Scene
    orc.set_threads(os.cpu_count() or 1)
    W, H, K, Q = 1920, 1080, 5, 15
    n = a.serve_gaussians
    forms = {}
    sc = synthetic_scene(n, seed=100, mode="full")
    st = to_torch(sc, "cuda", torch.float32)
    forms["fp32_full"] = (sc, Scene("fp32_full", st["pws"], st["rots"], st["scales"], st["alphas"],
                                    shs=st["shs"]))
    sc = synthetic_scene(n, seed=200, mode="lowrank", rank=3)
    st = to_torch(sc, "cuda", torch.bfloat16)
    forms["bf16_lowrank"] = (sc, Scene("bf16_lowrank", st["pws"], st["rots"], st["scales"],
                                       st["alphas"], dc=st["dc"], A=st["A"], B=st["B"]))
    c0 = look_at((0, -8, 0), width=W, height=H, device="cpu")
    res = [(W, H, c0.fx, c0.fy, c0.cx, c0.cy)]
    probes = [(c.Rcw.numpy(), c.tcw.numpy()) for c in
              (look_at(e, device="cpu") for e in sphere_poses(8, 6.0, seed=3))]
    srv = PaletteServer(hbm_budget=8 << 30, slots=4, keep_images=True)
    for _, scene in forms.values():
        if not srv.admit_scene(scene, res, probes):
            raise RuntimeError(f"scene {scene.id} not admitted")
    rng = np.random.default_rng(11)
    eyes = sphere_poses(a.serve_requests, (6.0, 10.0), seed=12)
    report = dict(gaussians_per_scene=n, resolution=f"{W}x{H}", requests_per_form=a.serve_requests,
                  tile_stride=a.tile_stride, host_threads=orc.get_threads(), forms={})
    t0 = time.time()
    for form, (sc, scene) in forms.items():
        reqs, cams = [], []
        for i in range(a.serve_requests):
            cam = look_at(eyes[i], width=W, height=H, device="cpu")
            pal = np.array(sc["palette"], np.float32)
            pal[2:] = np.clip(pal[2:] + rng.normal(0, 0.15, pal[2:].shape), 0, 1)
            reqs.append(Request(scene.id, cam.Rcw.numpy(), cam.tcw.numpy(), cam.fx, cam.fy,
                                cam.cx, cam.cy, W, H, pal))
            cams.append(cam)
        srv.run_closed_loop(reqs)  # the batched persistent path
        rows = []
        for req, cam in zip(reqs, cams):
            twc = req.twc.numpy().astype(np.float64)
            pre32 = orc.preprocess(sc["pws"], sc["rots"], sc["scales"], cam, np.float32)
            lists, mask = sampled_lists(orc, pre32, H, W, a.tile_stride)
            f64 = {k: np.asarray(sc[k], np.float64) for k in ("pws", "rots", "scales", "alphas")}
            if "shs" in sc:
                w64, = orc.sh2feat(np.asarray(sc["shs"], np.float64), f64["pws"], twc, K, False,
                                   np.float64, ref_quirk=False)
            else:
                w64, = orc.sh2weight_fast(np.asarray(sc["dc"], np.float64),
                                          np.asarray(sc["A"], np.float64),
                                          np.asarray(sc["B"], np.float64), f64["pws"], twc, K, Q,
                                          False, np.float64)
            o = orc.render_weights(f64["pws"], f64["rots"], f64["scales"], f64["alphas"], w64, cam,
                                   np.float64, lists=lists)
            img64 = np.einsum("kc,khw->chw", req.palette.numpy().astype(np.float64), o["layer"])
            img = req.image.double().cpu().numpy().reshape(3, H, W)
            rows.append(stats(img, img64, mask))
        report["forms"][form] = dict(
            psnr_min=min(r["psnr"] for r in rows), psnr_mean=float(np.mean([r["psnr"] for r in rows])),
            max_abs=max(r["max_abs"] for r in rows),
            mean_abs=float(np.mean([r["mean_abs"] for r in rows])),
            frac_over_1e5=float(np.mean([r["frac_over_1e5"] for r in rows])))
    report["wall_s"] = round(time.time() - t0, 1)
    print(json.dumps(report, indent=1))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gaussians", type=int, default=3_000_000)
    ap.add_argument("--poses", type=int, default=32)
    ap.add_argument("--grad-poses", type=int, default=2)
    ap.add_argument("--tile-stride", type=int, default=8)
    ap.add_argument("--resolutions", default="3840x2160,1920x1080")
    ap.add_argument("--serving", action="store_true")
    ap.add_argument("--serve-gaussians", type=int, default=250_000)
    ap.add_argument("--serve-requests", type=int, default=8)
    a = ap.parse_args()
    if a.serving:
        return serving_precision(a)
    from oracle import oracle as orc
    from palette_b200.render import render_palette
    from palette_b200.scene import look_at, sphere_poses, synthetic_scene, to_torch
    orc.set_threads(os.cpu_count() or 1)
    sc = synthetic_scene(a.gaussians, seed=2, mode="full")
    K = 5
    st32 = to_torch(sc, "cuda", torch.float32)
    st16 = to_torch(sc, "cuda", torch.bfloat16)
    pal = sc["palette"].astype(np.float64)
    f64 = {k: sc[k].astype(np.float64) for k in ("pws", "rots", "scales", "alphas", "shs")}
    res = [tuple(int(v) for v in r.split("x")) for r in a.resolutions.split(",")]
    report = dict(gaussians=a.gaussians, poses=a.poses, tile_stride=a.tile_stride,
                  host_threads=orc.get_threads(), resolutions={}, gradients=[])
    t0 = time.time()
    for W, H in res:
        rows = {"fp32": [], "bf16": []}
        for pi, eye in enumerate(sphere_poses(a.poses, 8.0, seed=2)):
            cam = look_at(eye, width=W, height=H, device="cuda")
            twc = cam.twc.detach().double().cpu().numpy()
            pre32 = orc.preprocess(sc["pws"], sc["rots"], sc["scales"], cam, np.float32)
            lists, mask = sampled_lists(orc, pre32, H, W, a.tile_stride)
            w64, = orc.sh2feat(f64["shs"], f64["pws"], twc, K, False, np.float64, ref_quirk=False)
            o = orc.render_weights(f64["pws"], f64["rots"], f64["scales"], f64["alphas"], w64, cam,
                                   np.float64, lists=lists)
            img64 = np.einsum("kc,khw->chw", pal, o["layer"])
            for name, st in (("fp32", st32), ("bf16", st16)):
                with torch.no_grad():
                    layer, _, _ = render_palette(st["pws"], st["rots"], st["scales"], st["alphas"],
                                                 cam, shs=st["shs"])
                L = layer.double().cpu().numpy()
                img = np.einsum("kc,khw->chw", pal, L)
                rows[name].append(dict(layer=stats(L, o["layer"], mask), image=stats(img, img64, mask)))
            if pi < a.grad_poses and (W, H) == res[-1]:
                rng = np.random.default_rng(pi)
                dout = rng.standard_normal((K, H, W)) * mask
                g64 = orc.render_weights_backward(f64["pws"], f64["rots"], f64["scales"],
                                                  f64["alphas"], cam, twc, K, shs=f64["shs"],
                                                  lists=lists, dout=dout)
                pairs = dict(pws="dpws", rots="drots", scales="dscales", alphas="dalphas",
                             shs="dshs")
                # pixels whose discrete decisions differ between the FP32 render
                # and the FP64 oracle
                from palette_b200.render import _render_one, _weight_args
                w0, A_, B_, md, K_, P_, Q_, rk = _weight_args(st32["shs"], None, None, None, K)
                with torch.no_grad():
                    _l, ft32, _d, _s, _r, _g, c32 = _render_one(
                        st32["pws"], st32["rots"], st32["scales"], st32["alphas"], w0, A_, B_,
                        cam, md, K_, P_, Q_, rk)
                c32, ft32 = c32.cpu().numpy(), ft32.double().cpu().numpy()
                flip = (c32 != o["contrib"]) | (np.abs(ft32 - o["final_tau"]) >
                                                1e-4 * np.maximum(np.abs(o["final_tau"]), 1e-6))
                flip &= mask
                dout_ar = dout * ~flip
                g64_ar = orc.render_weights_backward(f64["pws"], f64["rots"], f64["scales"],
                                                     f64["alphas"], cam, twc, K, shs=f64["shs"],
                                                     lists=lists, dout=dout_ar)
                for name, st in (("fp32", st32), ("bf16", st16)):
                    rel, rel_ar = {}, {}
                    for d_out, ref, out in ((dout, g64, rel), (dout_ar, g64_ar, rel_ar)):
                        leaves = {k: st[k].detach().clone().requires_grad_(True) for k in pairs}
                        layer, _, _ = render_palette(leaves["pws"], leaves["rots"], leaves["scales"],
                                                     leaves["alphas"], cam, shs=leaves["shs"])
                        layer.backward(torch.from_numpy(d_out.astype(np.float32)).cuda())
                        for k, gk in pairs.items():
                            g = leaves[k].grad.double().cpu().numpy().reshape(len(ref[gk]), -1)
                            r = ref[gk].reshape(len(g), -1)
                            out[k] = float(np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-300))
                    report["gradients"].append(dict(
                        storage=name, width=W, height=H, pose=pi, rel_err=rel,
                        rel_err_arithmetic=rel_ar, flipped_pixels=int(flip.sum()),
                        sampled_pixels=int(mask.sum())))
        summ = {}
        for name, rs in rows.items():
            summ[name] = {
                part: dict(max_abs=max(r[part]["max_abs"] for r in rs),
                           mean_abs=float(np.mean([r[part]["mean_abs"] for r in rs])),
                           p9999_abs=max(r[part]["p9999_abs"] for r in rs),
                           frac_over_1e5=float(np.mean([r[part]["frac_over_1e5"] for r in rs])),
                           psnr_min=min(r[part]["psnr"] for r in rs),
                           psnr_mean=float(np.mean([r[part]["psnr"] for r in rs])))
                for part in ("layer", "image")}
        report["resolutions"][f"{W}x{H}"] = summ
    report["wall_s"] = round(time.time() - t0, 1)
    print(json.dumps(report, indent=1))


if __name__ == "__main__":
    main()
