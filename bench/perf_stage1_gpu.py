#!/usr/bin/env python
"""Speed of the stage-1 colour path (vanilla_3dgs/gsplatcu: project,
computeCov3D, computeCov2D, sh2Color, inverseCov2D, splat, and splatB with
the final-transmittance gradient) through the stage-1 reference extension
(oracle/_ref/vanilla, compiled from its sources by oracle/build_ref.py) and
through this build's gsplatcu, on identical synthetic inputs.  Device time per
iteration by CUDA events (median of `--reps` after warm-up, then the median
over `--rounds` rounds in which the two alternate, after 2 s of GPU load).
`splatB` returns d/d (u, conic, opacity, colour); the backward includes the
colour path's d/d final T input.  Not collected by pytest: run it on a GPU
box and keep the printed JSON.

    python bench/perf_stage1_gpu.py [--gaussians 1000000] [--width 1920] [--height 1080]
"""
import argparse
import json
import os
import statistics
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, os.path.join(ROOT, "reparamgs-palette_b200"), HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

import torch  # noqa: E402

from perf_reference_gpu import burn, timed  # noqa: E402


def forward(g, st, cam):
    """The stage-1 forward sequence through operator module g."""
    us, pcs, depths = g.project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
    cov3ds, = g.computeCov3D(st["rots"], st["scales"], depths, False)
    cov2ds, = g.computeCov2D(cov3ds, pcs, cam.Rcw, depths, cam.fx, cam.fy, cam.width, cam.height,
                             False)
    col, = g.sh2Color(st["shs48"], st["pws"], cam.twc, False)
    cinv, areas = g.inverseCov2D(cov2ds, depths, False)
    img, contrib, ft, ranges, gsid = g.splat(cam.height, cam.width, us, cinv, st["alphas"], depths,
                                             col, areas)
    return (us, cinv, depths, col, contrib, ft, ranges, gsid), img


def backward(g, st, cam, saved, dimg, dtau):
    us, cinv, depths, col, contrib, ft, ranges, gsid = saved
    return g.splatB(cam.height, cam.width, us, cinv, st["alphas"], depths, col, contrib, ft,
                    ranges, gsid, dimg, dtau)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gaussians", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--rounds", type=int, default=3)
    a = ap.parse_args()
    import gsplatcu as gsc
    from oracle.build_ref import load_vanilla_ref
    from palette_b200.scene import look_at, synthetic_scene, to_torch
    van = load_vanilla_ref()
    if van is None:
        raise SystemExit("stage-1 reference build oracle/_ref/vanilla is missing "
                         "(python oracle/build_ref.py)")
    sc = synthetic_scene(a.gaussians, seed=1, mode="full")
    st = to_torch(sc, "cuda")
    st["shs48"] = st["shs"][:, :48].contiguous()  # SH order 3, 3 colour channels
    cam = look_at((0.0, -8.0, 0.0), width=a.width, height=a.height, device="cuda")
    gen = torch.Generator("cuda").manual_seed(1)
    dimg = torch.randn((3, a.height, a.width), device="cuda", generator=gen)
    dtau = torch.randn((a.height, a.width), device="cuda", generator=gen)
    res = {}
    burn()
    for _ in range(a.rounds):
        for name, g in (("reference", van), ("b200", gsc)):
            saved, _ = forward(g, st, cam)
            res.setdefault(name + "_forward", []).append(timed(lambda: forward(g, st, cam), a.reps))
            res.setdefault(name + "_splatB", []).append(
                timed(lambda: backward(g, st, cam, saved, dimg, dtau), a.reps))

            def fb():
                s, _ = forward(g, st, cam)
                backward(g, st, cam, s, dimg, dtau)
            res.setdefault(name + "_fwd_bwd", []).append(timed(fb, a.reps))
            del saved
    out = {k: round(statistics.median(v), 4) for k, v in res.items()}
    for k in ("forward", "splatB", "fwd_bwd"):
        out["speedup_" + k] = round(out["reference_" + k] / out["b200_" + k], 3)
    out.update(gaussians=a.gaussians, width=a.width, height=a.height, unit="ms per iteration",
               gpu=torch.cuda.get_device_name(0),
               patches=int(forward(gsc, st, cam)[0][7].numel()))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
