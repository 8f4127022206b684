#!/usr/bin/env python
"""Per-operator timing of the drop-in `gsplatcu` module on one view: every
operator the reference caller's forward and backward use
(gsplat/gsmodel.py:104-200), in the order it calls them. Each time is the
median CUDA-event time of one call, after warm-up; it includes the call's host
work and its output allocations. Also reported for each operator:
- the bytes of its input and output tensors;
- those bytes divided by the time, in GB/s.

The byte count is an upper bound on the operator's compulsory traffic, since an
operator may read only part of an input. `splat_weight` and `splat_weight_B`
are compositing operators; their bytes say little about their time.

Not collected by pytest. Its command line is also the recipe for the ncu
capture of the per-Gaussian kernels (`k_sh2feat` and the like).

    python bench/perf_ops_gpu.py [--gaussians 1000000] [--width 1920] [--height 1080]
                                 [--dtype f32|bf16] [--reps 50]
"""
import argparse
import json
import os
import statistics
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, os.path.join(ROOT, "reparamgs-palette_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import torch  # noqa: E402


def median_ms(fn, reps, warm=5, prep=None):
    for _ in range(warm):
        if prep:
            prep()
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        if prep:
            prep()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        e.synchronize()
        ts.append(s.elapsed_time(e))
    return statistics.median(ts)


def nbytes(ts):
    return sum(int(t.numel()) * t.element_size() for t in ts
               if isinstance(t, torch.Tensor))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gaussians", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--dtype", default="f32", choices=["f32", "bf16"])
    ap.add_argument("--reps", type=int, default=50)
    a = ap.parse_args()
    if not torch.cuda.is_available():
        raise SystemExit("perf_ops_gpu.py: CUDA is required")
    import gsplatcu as gsc
    from palette_b200.scene import look_at, synthetic_scene, to_torch
    dt = torch.bfloat16 if a.dtype == "bf16" else torch.float32
    K, Q, H, W = 5, 15, a.height, a.width
    full = to_torch(synthetic_scene(a.gaussians, seed=1, mode="full"), "cuda", dt)
    low = to_torch(synthetic_scene(a.gaussians, seed=1, mode="lowrank", rank=3), "cuda", dt)
    cam = look_at((0.0, -8.0, 0.0), width=W, height=H, device="cuda")
    pws, rots, scales = full["pws"], full["rots"], full["scales"]
    alphas = full["alphas"]
    rows = []

    def op(name, fn, ins, prep=None):
        if prep:
            prep()
        outs = fn()
        ms = median_ms(fn, a.reps, prep=prep)
        b = nbytes(ins) + nbytes(outs)
        rows.append(dict(op=name, ms=round(ms, 4), bytes=b,
                         gb_per_s=round(b / (ms * 1e-3) / 1e9, 1)))
        return outs

    with torch.no_grad():
        us, pcs, depths = op("project", lambda: gsc.project(
            pws, cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False), [pws])
        cov3ds, = op("computeCov3D", lambda: gsc.computeCov3D(rots, scales, depths, False),
                     [rots, scales, depths])
        cov2ds, = op("computeCov2D", lambda: gsc.computeCov2D(
            cov3ds, pcs, cam.Rcw, depths, cam.fx, cam.fy, W, H, False), [cov3ds, pcs, depths])
        op("sh2Weight", lambda: gsc.sh2Weight(full["shs"], pws, cam.twc, False, K),
           [full["shs"], pws])
        weights, _, _ = op("sh2Weight (Jacobians)",
                           lambda: gsc.sh2Weight(full["shs"], pws, cam.twc, True, K),
                           [full["shs"], pws])
        op("sh2Weight_fast (Jacobians)", lambda: gsc.sh2Weight_fast(
            low["dc"], low["A"], low["B"], pws, cam.twc, True, K, Q),
           [low["dc"], low["A"], low["B"], pws])
        cinv2ds, areas = op("inverseCov2D", lambda: gsc.inverseCov2D(cov2ds, depths, False),
                            [cov2ds, depths])
        layer, contrib, final_tau, ranges, gsid = op("splat_weight", lambda: gsc.splat_weight(
            H, W, K, us, cinv2ds, alphas, depths, weights, areas),
            [us, cinv2ds, alphas, depths, weights, areas])
        g = torch.rand_like(layer)
        fw = {}

        def forward():  # untimed: the backward reuses the records of the forward before it
            fw["o"] = gsc.splat_weight(H, W, K, us, cinv2ds, alphas, depths, weights, areas)

        def backward():
            _, c, t, r, s = fw["o"]
            return gsc.splat_weight_B(H, W, K, us, cinv2ds, alphas, depths, weights, c, t, r, s,
                                      g)
        op("splat_weight_B", backward,
           [us, cinv2ds, alphas, weights, contrib, final_tau, ranges, gsid, g], prep=forward)
    print(json.dumps(dict(gaussians=a.gaussians, width=W, height=H, dtype=a.dtype,
                          patches=int(gsid.numel()), ops=rows)))


if __name__ == "__main__":
    main()
