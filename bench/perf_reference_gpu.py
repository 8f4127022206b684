#!/usr/bin/env python
"""Speed of this build against the reference extension on the same GPU.

Runs the reference's own autograd sequences -- WeightGSFunctionTest (full SH
weights, gsplat/gsmodel.py:104-139) and WeightGSFunctionFast (low-rank, rank 1
as the reference supports, gsplat/gsmodel.py:151-200) -- once through the
reference build (oracle/_ref, compiled from its sources by oracle/build_ref.py)
and once through this build's gsplatcu, on identical synthetic inputs, plus
this build's fused path (palette_b200.render.render_palette, weights-only
backward) on the same scene.  Device time per iteration by CUDA events
(median of 10 repeats after warm-up, then the median over 3 rounds in which
the implementations alternate, after 2 s of GPU load to settle the clocks).
Forward calls are also timed back to back (``*_forward_pipelined``: 10 calls
between one pair of events), where a call's host work overlaps the device
work of the calls before it.  Not collected by pytest: run it
on a GPU box and keep the printed JSON.

    python bench/perf_reference_gpu.py [--gaussians 1000000] [--width 1920] [--height 1080]
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


def forward(g, st, cam, mode, K=5):
    """The WeightGSFunction forward sequence through operator module g."""
    us, pcs, depths = g.project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
    cov3ds, = g.computeCov3D(st["rots"], st["scales"], depths, False)
    cov2ds, = g.computeCov2D(cov3ds, pcs, cam.Rcw, depths, cam.fx, cam.fy, cam.width, cam.height,
                             False)
    if mode == "full":
        w, dwd, _ = g.sh2Weight(st["shs"], st["pws"], cam.twc, True, K)
        extra = (dwd,)
    else:
        w, ddc, ylm = g.sh2Weight_fast(st["dc"], st["A"], st["B"], st["pws"], cam.twc, True, K, 15)
        extra = (ddc, ylm)
    cinv, areas = g.inverseCov2D(cov2ds, depths, False)
    layer, contrib, ft, ranges, gsid = g.splat_weight(cam.height, cam.width, K, us, cinv,
                                                      st["alphas"], depths, w, areas)
    return (us, cinv, depths, w, contrib, ft, ranges, gsid) + extra, layer


def backward(g, st, cam, mode, saved, dlayer, K=5):
    us, cinv, depths, w, contrib, ft, ranges, gsid = saved[:8]
    dW, = g.splat_weight_B(cam.height, cam.width, K, us, cinv, st["alphas"], depths, w, contrib,
                           ft, ranges, gsid, dlayer)
    if mode == "full":
        dwd = saved[8]
        return (dW.permute(0, 2, 1) @ dwd).permute(0, 2, 1)
    ddc, ylm = saved[8], saved[9]
    dw = dW.squeeze(1)
    return dw * ddc, g.sh2Weight_fast_B(st["A"], st["B"], ylm, dw, K, 15)


def timed(fn, reps=10, warm=3):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        ts.append(s.elapsed_time(e))
    return statistics.median(ts)


def timed_pipelined(fn, reps=10, warm=3):
    """Time per call of `reps` calls issued back to back between one pair of
    events: the host work of a call overlaps the device work of the calls
    before it (a throughput, where timed() measures the latency of one call)."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def burn(seconds=2.0):
    """Keep the GPU busy so that its clocks have ramped up before timing."""
    a = torch.randn((4096, 4096), device="cuda")
    t = torch.cuda.Event(enable_timing=True)
    s = torch.cuda.Event(enable_timing=True)
    s.record()
    while True:
        for _ in range(20):
            a = a @ a
            a = a / a.norm()
        t.record()
        torch.cuda.synchronize()
        if s.elapsed_time(t) > seconds * 1000:
            return


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gaussians", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--rounds", type=int, default=3,
                    help="alternating rounds; each figure is the median over rounds")
    a = ap.parse_args()
    import gsplatcu as ours
    from oracle.build_ref import load_ref
    from palette_b200.render import render_palette
    from palette_b200.scene import look_at, synthetic_scene, to_torch
    ref = load_ref()
    if ref is None:
        raise SystemExit("reference build oracle/_ref/gsplatcu_ref.so is missing")
    cam = look_at((0.0, -8.0, 0.0), width=a.width, height=a.height, device="cuda")
    out = dict(gaussians=a.gaussians, width=a.width, height=a.height, unit="ms per iteration",
               gpu=torch.cuda.get_device_name(0), cases={})
    for mode in ("full", "lowrank"):
        sc = synthetic_scene(a.gaussians, seed=1, mode=mode, rank=1)
        st = to_torch(sc, "cuda")
        if mode == "lowrank":  # the reference's rank-1 shapes
            st["A"], st["B"] = st["A"][:, :, 0].contiguous(), st["B"][:, 0, :].contiguous()
        dlayer = torch.rand((5, a.height, a.width), device="cuda")
        wn = dict(shs=st["shs"]) if mode == "full" else dict(dc=st["dc"], A=st["A"], B=st["B"])
        leaves = {k: v.detach().clone().requires_grad_(True) for k, v in wn.items()}

        def fused(bwd):
            layer, _, _ = render_palette(st["pws"], st["rots"], st["scales"], st["alphas"], cam,
                                         **leaves)
            if bwd:
                layer.backward(dlayer)

        burn()
        rounds = []
        for _ in range(a.rounds):  # alternate the implementations within each round
            row = {}
            for name, g in (("reference", ref), ("b200_ops", ours)):
                row[name + "_forward"] = timed(lambda: forward(g, st, cam, mode), a.reps)
                row[name + "_forward_pipelined"] = timed_pipelined(
                    lambda: forward(g, st, cam, mode), a.reps)

                def fb():
                    saved, _ = forward(g, st, cam, mode)
                    backward(g, st, cam, mode, saved, dlayer)
                row[name + "_fwd_bwd"] = timed(fb, a.reps)
            with torch.no_grad():
                row["b200_fused_forward"] = timed(lambda: fused(False), a.reps)
                row["b200_fused_forward_pipelined"] = timed_pipelined(lambda: fused(False), a.reps)
            row["b200_fused_fwd_bwd"] = timed(lambda: fused(True), a.reps)
            rounds.append(row)
        row = {k: statistics.median(r[k] for r in rounds) for k in rounds[0]}
        row["reference_forward_range"] = [min(r["reference_forward"] for r in rounds),
                                          max(r["reference_forward"] for r in rounds)]
        for k in ("forward", "forward_pipelined", "fwd_bwd"):
            row[f"speedup_ops_{k}"] = row[f"reference_{k}"] / row[f"b200_ops_{k}"]
            row[f"speedup_fused_{k}"] = row[f"reference_{k}"] / row[f"b200_fused_{k}"]
        out["cases"][mode + ("" if mode == "full" else "_rank1")] = {
            k: (round(v, 4) if not isinstance(v, list) else [round(x, 4) for x in v])
            for k, v in row.items()}
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
