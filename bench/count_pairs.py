#!/usr/bin/env python
"""Work counts of the compositing kernels on the bench scene, by the CPU
oracle (whose FP32 preprocess, tile lists and compositing decisions equal the
GPU's bit for bit): patches M, nominal Gaussian-pixel evaluations (M x 256),
blended (pixel, Gaussian) pairs of the forward -- the pairs the adjoint walks
back over -- and pixels.  The ncu summaries divide the kernels' executed
instructions by these counts.

    python bench/count_pairs.py [--gaussians 1000000] [--width 1920] [--height 1080] [--rank 3]
"""
import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, os.path.join(ROOT, "reparamgs-palette_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gaussians", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--rank", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args()
    from oracle import oracle as orc
    from palette_b200.scene import look_at, synthetic_scene
    orc.set_threads(os.cpu_count() or 1)
    sc = synthetic_scene(a.gaussians, seed=a.seed, mode="lowrank", rank=a.rank)
    cam = look_at((0.0, -8.0, 0.0), width=a.width, height=a.height, device="cpu")
    H, W, K = a.height, a.width, 5
    pre = orc.preprocess(sc["pws"], sc["rots"], sc["scales"], cam, np.float32)
    w, = orc.sh2weight_fast(sc["dc"], sc["A"], sc["B"], sc["pws"], pre["twc"], K, 15, False)
    b = orc.bin_gaussians(pre["us"], pre["areas"], pre["depths"], H, W)
    out, contrib, ft, blends = orc.draw_count(H, W, K, b["ranges"], b["gsid"], pre["us"],
                                              pre["cinv"], sc["alphas"], w, 0.0)
    M = int(len(b["gsid"]))
    print(json.dumps(dict(workload=f"{a.gaussians} Gaussians, {W}x{H}, rank {a.rank}",
                          patches=M, nominal_evaluations=M * 256,
                          blended_pairs=int(blends.sum()), pixels=H * W,
                          mean_blends_per_pixel=float(blends.mean()),
                          mean_contrib_index=float(contrib.mean())), indent=1))


if __name__ == "__main__":
    main()
