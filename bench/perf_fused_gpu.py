#!/usr/bin/env python
"""Timing of the fused render path (palette_b200.render.render_palette) for
one weight form: full SH order 3 (``--mode full``) or rank-r low-rank factors
(``--mode lowrank --rank r``), FP32 or BF16 storage, on the benchmark
generator's scene.  Prints CUDA-event medians of the forward and of forward +
weights-only backward (dL/dlayer random), and the fused preprocess kernel
alone through the C ABI.  Not collected by pytest; also the command the
preprocess kernels' ncu summaries are captured from.

    python bench/perf_fused_gpu.py [--mode full|lowrank] [--rank 3] [--dtype f32|bf16]
                                   [--gaussians 1000000] [--width 1920] [--height 1080]
"""
import argparse
import ctypes as C
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


def median_ms(fn, reps, warm=3):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        e.synchronize()
        ts.append(s.elapsed_time(e))
    return statistics.median(ts)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", default="full", choices=["full", "lowrank"])
    ap.add_argument("--rank", type=int, default=3)
    ap.add_argument("--dtype", default="f32", choices=["f32", "bf16"])
    ap.add_argument("--gaussians", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args()
    from gsplatcu import _lib
    from palette_b200.render import camera_struct, render_palette
    from palette_b200.scene import look_at, synthetic_scene, to_torch
    dt = torch.bfloat16 if a.dtype == "bf16" else torch.float32
    sc = synthetic_scene(a.gaussians, seed=1, mode=a.mode, rank=a.rank)
    st = to_torch(sc, "cuda", dt)
    cam = look_at((0.0, -8.0, 0.0), width=a.width, height=a.height, device="cuda")
    K = 5
    if a.mode == "full":
        kw = dict(shs=st["shs"].requires_grad_())
        params = _lib.PaletteParams(_lib.WEIGHTS_FULL, _lib.DTYPE_BF16 if dt == torch.bfloat16
                                    else _lib.DTYPE_F32, K, 0, 0, 0, st["shs"].data_ptr(), None,
                                    None)
    else:
        kw = dict(dc=st["dc"].requires_grad_(), A=st["A"].requires_grad_(),
                  B=st["B"].requires_grad_())
        params = _lib.PaletteParams(_lib.WEIGHTS_LOWRANK, _lib.DTYPE_BF16 if dt == torch.bfloat16
                                    else _lib.DTYPE_F32, K, 5, 15, a.rank, st["dc"].data_ptr(),
                                    st["A"].data_ptr(), st["B"].data_ptr())
    alphas = st["alphas"].reshape(-1).contiguous()
    g = torch.rand((K, a.height, a.width), device="cuda")

    def fwd():
        with torch.no_grad():
            render_palette(st["pws"], st["rots"], st["scales"], alphas, cam, **kw)

    def fwd_bwd():
        for v in kw.values():
            v.grad = None
        layer, _, _ = render_palette(st["pws"], st["rots"], st["scales"], alphas, cam, **kw)
        layer.backward(g)

    n = a.gaussians
    L = _lib.lib()
    state = torch.empty(int(L.gsb_splat_state_bytes(n, K, a.height, a.width)), dtype=torch.uint8,
                        device="cuda")
    camst, _keep = camera_struct(cam)

    def pre():
        _lib.call("perf", "gsb_render_preprocess", n, C.byref(camst), _lib.ptr(st["pws"]),
                  _lib.ptr(st["rots"]), _lib.ptr(st["scales"]), _lib.ptr(alphas), C.byref(params),
                  _lib.ptr(state), None, _lib.stream_of(st["pws"]))

    out = dict(mode=a.mode, rank=a.rank if a.mode == "lowrank" else None, dtype=a.dtype,
               gaussians=n, width=a.width, height=a.height,
               preprocess_ms=round(median_ms(pre, a.reps), 4),
               forward_ms=round(median_ms(fwd, a.reps), 4),
               fwd_bwd_ms=round(median_ms(fwd_bwd, a.reps), 4))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
