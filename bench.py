#!/usr/bin/env python
"""Benchmark of the palette-weight rasterizer on B200.

Workload (one step): a finetune step of ReparamGS-Palette's low-rank path
(WeightGSFunctionFast, gsplat/gsmodel.py:151-200) over 1,000,000 synthetic
Gaussians at 1920x1080 with rank-3 factors A [N,5,3], B [N,3,15] (P=5, Q=15,
K=5, SH order 3, FP32 storage): forward through the gsplatcu operators
(project, computeCov3D, computeCov2D, sh2Weight_fast, inverseCov2D,
splat_weight; palette_b200.weights.splat_palette_weights), the finetune loss
(finetune.py:356-389) against a seeded random target image -- L1 between the
rendered weights and the target's barycentric weights in the palette,
clamped to non-negative and renormalised, plus 0.5 * mean(relu(-weights))
(one fused kernel, palette_b200.loss) -- and the backward (splat_weight_B,
then one kernel from dL/dweights to the dc, A, B gradients; palette
gradient).  `value` is whole-job fwd+bwd iterations per second with the
scene resident in HBM; `frames_per_s` is the forward alone; `fused_path` the
same step through the one-kernel preprocess (palette_b200.render).
`multiview` is the differentiation workload on the same scene: steps of 8
views at 1920x1080 from BF16 rank-3 factors, loss 0.8 L1 + 0.2 (1 - SSIM) +
0.5 mean(relu(-W)) per view (fused render + fused loss kernel).
`gpu_baseline` times the reference's own gsplatcu extension (built from its
sources) on the same GPU through the reference's own autograd functions,
beside this build's paths on the same scenes, in a subprocess.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 (under torchrun): independent replicas, one per GPU (the path has no
exchange step); rank 0 prints the line with the max-over-ranks time.
--impl reference times the reference algorithm's CPU implementation (the
CPU oracle port, every tile of every step composited) on this host's cores,
and, as a labelled extra, the reference's own numpy rasterizer
(gsplat/gausplat.py) on the 20k-Gaussian 256x256 workload.
"""
import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "reparamgs-palette_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "1080p frames/s & fwd+bwd iters/s at 1M Gaussians; p50/p99 palette-edit latency"
# The finetune step's loss on the rendered weights (finetune.py:356-389): L1
# against the barycentric target of the target image in the palette, clamped
# to non-negative and renormalised, plus the negative-weight penalty.
LOSS = dict(clamp=True, lambda_pos=0.5, kind="l1")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--gaussians", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--rank", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="length of the palette-edit serving stream (0: skip)")
    ap.add_argument("--no-gpu-baseline", action="store_true",
                    help="skip the reference-extension timing leg")
    ap.add_argument("--gpu-baseline-leg", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--serve-rate", type=float, default=400.0)
    ap.add_argument("--serve-scale", type=float, default=1.0,
                    help="scale of the resident scene sizes (1: 100k..3M)")
    return ap.parse_args()


# ---------------------------------------------------------------- workload
def make_workload(a, device):
    from palette_b200.scene import look_at, synthetic_scene
    sc = synthetic_scene(a.gaussians, seed=a.seed, mode="lowrank", rank=a.rank)
    cam = look_at((0.0, -8.0, 0.0), width=a.width, height=a.height, device=device)
    t = lambda x: torch.from_numpy(x).to(device).contiguous()
    wl = dict(sc=sc, cam=cam, K=5, Q=15, pws=t(sc["pws"]), rots=t(sc["rots"]),
              scales=t(sc["scales"]), alphas=t(sc["alphas"]),
              dc=t(sc["dc"]).requires_grad_(), A=t(sc["A"]).requires_grad_(),
              B=t(sc["B"]).requires_grad_(), chroma=t(sc["palette"][2:]).requires_grad_())
    g = torch.Generator(device="cpu").manual_seed(a.seed)
    target = torch.rand((3, a.height, a.width), generator=g)
    wl["target_host"] = target.pin_memory() if device.type == "cuda" else target
    wl["target"] = target.to(device)
    wl["param_bytes"] = sum(int(x.numel()) * 4 for x in (wl["pws"], wl["rots"], wl["scales"],
                                                         wl["alphas"], wl["dc"], wl["A"], wl["B"]))
    return wl


def step(wl, cam=None, target=None, backward=True):
    from palette_b200.loss import palette_geo_loss
    from palette_b200.weights import splat_palette_weights
    cam = cam or wl["cam"]
    target = wl["target"] if target is None else target
    for p in (wl["dc"], wl["A"], wl["B"], wl["chroma"]):
        p.grad = None
    layer, _ = splat_palette_weights(wl["pws"], wl["alphas"], wl["scales"], wl["rots"], cam,
                                     dc=wl["dc"], A=wl["A"], B=wl["B"])
    loss = palette_geo_loss(layer, wl["chroma"], target, **LOSS)
    if backward:
        loss.backward()
    return loss


def step_fused(wl, backward=True):
    """The same step through the fused render path (palette_b200.render): one
    preprocess kernel instead of five operators; weights-only backward, as
    the reference's backward (only dc, A, B and the palette need gradients)."""
    from palette_b200.loss import palette_geo_loss
    from palette_b200.render import render_palette
    for p in (wl["dc"], wl["A"], wl["B"], wl["chroma"]):
        p.grad = None
    layer, _, _ = render_palette(wl["pws"], wl["rots"], wl["scales"], wl["alphas"], wl["cam"],
                                 dc=wl["dc"], A=wl["A"], B=wl["B"])
    loss = palette_geo_loss(layer, wl["chroma"], wl["target"], **LOSS)
    if backward:
        loss.backward()
    return loss


VIEWS = 8  # views per step of the multi-view finetune leg


def make_views(wl, a, device):
    """The multi-view leg's inputs: the scene's low-rank factors in BF16, a
    learnt palette, VIEWS cameras on a sphere of radius 8 and one seeded
    random target image per view."""
    from palette_b200.scene import look_at, sphere_poses
    sc = wl["sc"]
    bf = lambda x: torch.from_numpy(x).to(device, torch.bfloat16).contiguous().requires_grad_()
    g = torch.Generator(device="cpu").manual_seed(a.seed + 1)
    return dict(dc=bf(sc["dc"]), A=bf(sc["A"]), B=bf(sc["B"]),
                palette=torch.from_numpy(sc["palette"]).to(device).requires_grad_(),
                cams=[look_at(e, width=a.width, height=a.height, device=device)
                      for e in sphere_poses(VIEWS, 8.0, seed=a.seed)],
                targets=[torch.rand((3, a.height, a.width), generator=g).to(device)
                         for _ in range(VIEWS)])


def step_views(wl, mv, backward=True):
    """One step of the multi-view finetune workload: VIEWS views rendered
    through the fused path from BF16 rank-3 factors (FP32 arithmetic,
    palette_b200.render.render_palette_views), each with 0.8 L1 + 0.2 (1 -
    SSIM) of its palette colour image against its target plus 0.5
    mean(relu(-weights)) (one fused kernel per view,
    palette_b200.loss.palette_l1_ssim_loss), averaged over the views; the
    backward sums the views' dc, A, B gradients in FP32 and returns them in
    BF16, with the palette gradient."""
    from palette_b200.loss import palette_l1_ssim_loss
    from palette_b200.render import render_palette_views
    for p in (mv["dc"], mv["A"], mv["B"], mv["palette"]):
        p.grad = None
    layers, _, _ = render_palette_views(wl["pws"], wl["rots"], wl["scales"], wl["alphas"],
                                        mv["cams"], dc=mv["dc"], A=mv["A"], B=mv["B"])
    total = None
    for layer, tgt in zip(layers, mv["targets"]):
        loss = palette_l1_ssim_loss(layer, mv["palette"], tgt, lambda_ssim=0.2, lambda_pos=0.5)
        total = loss if total is None else total + loss
    total = total / len(mv["cams"])
    if backward:
        total.backward()
    return total


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi SM clock / throttle-reason samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc, self.path = index, None, None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def dist_setup(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def allreduce_max(v, world, device):
    if world == 1:
        return v
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_figure(kernel_tag, key):
    """A per-launch figure of a kernel from its committed ncu summary
    (profiles/<kernel_tag>.md, a line '<key>: N'): traffic_bytes_per_launch
    (dram__bytes_read.sum + dram__bytes_write.sum), warp_inst_per_launch
    (smsp__inst_executed.sum), inst_per_blended_pair."""
    p = os.path.join(ROOT, "profiles", kernel_tag + ".md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def timed(fn, reps, stream):
    """Device time (ms) of `reps` calls of fn on `stream` (after one untimed
    call), CUDA events, synced both sides."""
    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(reps):
        fn()
    e.record(stream)
    torch.cuda.synchronize()
    return s.elapsed_time(e)


# ------------------------------------------------------------- stage timing
def stage_breakdown(wl, reps=5):
    """Per-stage device times (ms) of one step, each stage run alone through the
    C ABI with CUDA events on the launching stream, plus the algorithmic bytes
    of the compositing kernels."""
    import gsplatcu as gsc
    from gsplatcu import _lib
    cam, K, Q = wl["cam"], wl["K"], wl["Q"]
    H, W = cam.height, cam.width
    st = torch.cuda.current_stream()
    L = _lib.lib()
    with torch.no_grad():
        dc, A, B = wl["dc"].detach(), wl["A"].detach(), wl["B"].detach()
        out = {}

        def pre():
            us, pcs, d = gsc.project(wl["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
            c3, = gsc.computeCov3D(wl["rots"], wl["scales"], d, False)
            c2, = gsc.computeCov2D(c3, pcs, cam.Rcw, d, cam.fx, cam.fy, W, H, False)
            w, = gsc.sh2Weight_fast(dc, A, B, wl["pws"], cam.twc, False, K, Q)
            cinv, areas = gsc.inverseCov2D(c2, d, False)
            return us, cinv, d, areas, w
        out["preprocess"] = timed(pre, reps, st) / reps
        us, cinv, d, areas, w = pre()
        n = us.shape[0]
        state = torch.empty(int(L.gsb_splat_state_bytes(n, K, H, W)), dtype=torch.uint8,
                            device=us.device)
        import ctypes as C
        sp = _lib.stream_of(us)
        def pack():
            _lib.call("bench", "gsb_splat_pack", n, H, W, K, _lib.ptr(us), _lib.ptr(cinv),
                      _lib.ptr(wl["alphas"]), _lib.ptr(w), 0, _lib.ptr(d), _lib.ptr(areas),
                      _lib.ptr(state), sp)
        # the pack's in-place updates (depth and extent of Gaussians with an
        # empty tile rectangle) are idempotent: after this first call every
        # timed call sees the same inputs and writes the same outputs
        pack()
        out["bin_pack_scan"] = timed(pack, reps, st) / reps
        plan = _lib.SplatPlan()
        _lib.call("bench", "gsb_splat_counts", n, H, W, _lib.ptr(state), C.byref(plan), sp)
        M = int(plan.patches)
        ws = torch.empty(int(L.gsb_splat_sort_bytes(n, H, W, C.byref(plan))), dtype=torch.uint8,
                         device=us.device)
        gx, gy = (W + 15) // 16, (H + 15) // 16
        gsid = torch.empty(M, dtype=torch.int32, device=us.device)
        ranges = torch.empty((gx * gy, 2), dtype=torch.int32, device=us.device)
        out["bin_sort"] = timed(lambda: _lib.call(
            "bench", "gsb_splat_sort", n, H, W, C.byref(plan), _lib.ptr(state), _lib.ptr(ws),
            _lib.ptr(gsid), _lib.ptr(ranges), sp), reps, st) / reps
        layer = torch.empty((K, H, W), device=us.device)
        contrib = torch.empty((H, W), dtype=torch.int32, device=us.device)
        ft = torch.empty((H, W), device=us.device)
        out["draw"] = timed(lambda: _lib.call(
            "bench", "gsb_splat_draw", n, H, W, K, _lib.ptr(ranges), _lib.ptr(gsid), _lib.ptr(state),
            0.0, _lib.ptr(layer), _lib.ptr(contrib), _lib.ptr(ft), sp), reps, st) / reps
        g = torch.rand((K, H, W), device=us.device)
        dW = torch.zeros((n, 1, K), device=us.device)
        out["draw_backward"] = timed(lambda: _lib.call(
            "bench", "gsb_splat_backward_packed", n, H, W, K, _lib.ptr(ranges), _lib.ptr(gsid),
            _lib.ptr(contrib), _lib.ptr(ft), _lib.ptr(g), None, _lib.ptr(state), _lib.ptr(dW), None,
            None, None, sp), reps, st) / reps
        from palette_b200.render import camera_struct
        camst, _keep = camera_struct(cam)
        params = _lib.PaletteParams(_lib.WEIGHTS_LOWRANK, _lib.DTYPE_F32, K, 5, Q, int(A.shape[2]),
                                    dc.data_ptr(), A.data_ptr(), B.data_ptr())
        gdc, gA, gB = torch.empty_like(dc), torch.empty_like(A), torch.empty_like(B)
        out["weights_backward"] = timed(lambda: _lib.call(
            "bench", "gsb_palette_weights_backward", n, C.byref(camst), _lib.ptr(wl["pws"]),
            C.byref(params), _lib.ptr(dW), _lib.ptr(gdc), _lib.ptr(gA), _lib.ptr(gB), sp),
            reps, st) / reps
        # fused path: one preprocess kernel (+ count scan), weights-only backward
        fstate = torch.empty_like(state)
        out["fused_preprocess"] = timed(lambda: _lib.call(
            "bench", "gsb_render_preprocess", n, C.byref(camst), _lib.ptr(wl["pws"]),
            _lib.ptr(wl["rots"]), _lib.ptr(wl["scales"]), _lib.ptr(wl["alphas"]), C.byref(params),
            _lib.ptr(fstate), None, sp), reps, st) / reps
        scratch = torch.empty(int(L.gsb_render_backward_bytes(n, K)), dtype=torch.uint8,
                              device=us.device)
        out["fused_backward"] = timed(lambda: _lib.call(
            "bench", "gsb_render_backward", n, C.byref(camst), _lib.ptr(wl["pws"]),
            _lib.ptr(wl["rots"]), _lib.ptr(wl["scales"]), _lib.ptr(wl["alphas"]), C.byref(params),
            _lib.ptr(state), _lib.ptr(ranges), _lib.ptr(gsid), _lib.ptr(contrib), _lib.ptr(ft),
            _lib.ptr(g), None, _lib.ptr(scratch), None, None, None, None, _lib.ptr(gdc),
            _lib.ptr(gA), _lib.ptr(gB), sp), reps, st) / reps
        from palette_b200.loss import palette_l1_ssim_loss
        pal = torch.from_numpy(wl["sc"]["palette"]).to(us.device)
        out["l1_ssim_loss"] = timed(lambda: palette_l1_ssim_loss(layer, pal, wl["target"]),
                                    reps, st) / reps
        visible = int((d > 0.2).sum())
        pix = H * W
        # algorithmic bytes: per patch 48 B record + 4 B id; per pixel K*4 + 8 B out;
        # backward: per pixel K*4 + 8 B in, per patch 52 B, per visible Gaussian K*4 B out
        bytes_draw = M * 52 + pix * (4 * K + 8)
        bytes_bwd = pix * (4 * K + 8) + M * 52 + visible * 4 * K
        return out, dict(M=M, visible=visible, bytes_draw=bytes_draw, bytes_bwd=bytes_bwd)


# ------------------------------------------------------------------ serving
SERVE_SIZES = (100_000, 250_000, 500_000, 1_000_000, 2_000_000, 3_000_000)
SERVE_RES = ((1280, 720), (1920, 1080), (3840, 2160))


def serve_bench(a, device):
    """Palette-edit serving (palette_b200.serve): 12 resident scenes of
    100k..3M Gaussians (two of each size; one with full SH weights in FP32,
    one with rank-3 low-rank factors in BF16), an open-loop Poisson stream of
    requests (random scene, camera on a sphere of radius 6..10, resolution
    720p / 1080p / 4K, the 3 chromatic palette anchors perturbed by
    N(0, 0.15) clipped to [0, 1]).  Latency = arrival to image complete in
    HBM, camera and palette copied from pinned host memory per request."""
    from palette_b200.scene import look_at, sphere_poses, synthetic_scene, to_torch
    from palette_b200.serve import PaletteServer, Request, Scene
    rng = np.random.default_rng(a.seed + 7)
    scenes, palettes = [], {}
    for j, size in enumerate(SERVE_SIZES):
        n = max(1000, int(size * a.serve_scale))
        for form in ("fp32_full", "bf16_lowrank"):
            sid = f"{form}_{n}"
            if form == "fp32_full":
                sc = synthetic_scene(n, seed=100 + j, mode="full")
                st = to_torch(sc, device, torch.float32)
                scenes.append(Scene(sid, st["pws"], st["rots"], st["scales"], st["alphas"],
                                    shs=st["shs"]))
            else:
                sc = synthetic_scene(n, seed=200 + j, mode="lowrank", rank=3)
                st = to_torch(sc, device, torch.bfloat16)
                scenes.append(Scene(sid, st["pws"], st["rots"], st["scales"], st["alphas"],
                                    dc=st["dc"], A=st["A"], B=st["B"]))
            palettes[sid] = sc["palette"]
            del sc, st
    res = []
    for W, H in SERVE_RES:
        c = look_at((0, -8, 0), width=W, height=H, device="cpu")
        res.append((W, H, c.fx, c.fy, c.cx, c.cy))
    probes = [(c.Rcw.numpy(), c.tcw.numpy()) for c in
              (look_at(e, device="cpu") for e in sphere_poses(8, 6.0, seed=3))]
    free, _ = torch.cuda.mem_get_info(device)
    srv = PaletteServer(hbm_budget=int(0.8 * free), slots=8, device=device, keep_images=False)
    t0 = time.perf_counter()
    for sc in scenes:
        if not srv.admit_scene(sc, res, probes):
            raise RuntimeError(f"serving: scene {sc.id} does not fit the HBM budget")
    admit_s = time.perf_counter() - t0
    nreq = max(1, int(a.serve_rate * a.serve_seconds))
    eyes = sphere_poses(nreq, (6.0, 10.0), seed=a.seed + 11)
    reqs = []
    for i in range(nreq):
        sc = scenes[int(rng.integers(len(scenes)))]
        W, H, fx, fy, cx, cy = res[int(rng.integers(len(res)))]
        cam = look_at(eyes[i], width=W, height=H, device="cpu")
        pal = np.array(palettes[sc.id], np.float32)
        pal[2:] = np.clip(pal[2:] + rng.normal(0, 0.15, pal[2:].shape), 0, 1)
        reqs.append(Request(sc.id, cam.Rcw.numpy(), cam.tcw.numpy(), fx, fy, cx, cy, W, H, pal,
                            tag=("bf16" if sc.id.startswith("bf16") else "fp32", W)))
    t1 = time.perf_counter()
    srv.prepare(reqs)
    prep_s = time.perf_counter() - t1
    n_batches0 = len(srv.batch_sizes)
    st = srv.run_open_loop(reqs, rate=a.serve_rate, seed=a.seed)
    st["mean_batch"] = round(float(np.mean(srv.batch_sizes[n_batches0:])), 2)
    lat = {}
    for r in srv.done:
        for key in (r.tag[0], f"{r.tag[1]}px"):
            lat.setdefault(key, []).append((r.done - r.arrival) * 1000.0)
    st["by_form"] = {k: dict(n=len(v), p50_ms=round(float(np.percentile(v, 50)), 3),
                             p99_ms=round(float(np.percentile(v, 99)), 3))
                     for k, v in sorted(lat.items())}
    # saturation (closed loop): every request of one storage form queued at
    # once, per form
    sat = {}
    for form in ("fp32", "bf16"):
        sub = [Request(r.scene_id, r.Rcw.numpy(), r.tcw.numpy(), r.fx, r.fy, r.cx, r.cy, r.width,
                       r.height, r.palette.numpy(), tag=r.tag)
               for r in reqs if r.tag[0] == form][:600]
        srv.run_closed_loop(sub[:50])  # warm
        res = srv.run_closed_loop(sub)
        sat[form] = dict(requests=res["requests"], frames_per_s=round(res["frames_per_s"], 1),
                         mean_batch=round(res["mean_batch"], 2), reruns=res["reruns"])
    st["saturation"] = sat
    st.update(scenes=len(scenes), gaussians=int(sum(s.n for s in scenes)),
              resident_gb=round(srv.resident_bytes() / 1e9, 2), slots=len(srv.slots),
              graphs=srv.graph_captures, seconds=a.serve_seconds, admit_s=round(admit_s, 1),
              capture_s=round(prep_s, 1),
              latency="arrival to image complete in HBM; camera/palette H2D per request",
              path=("per-request preparation graphs (fused preprocess + capacity sort) on 8 "
                    "slot streams; prepared requests composited together by one persistent "
                    "kernel per batch (captured graph, up to 3 batches in flight on their own streams)"))
    for k in ("p50_ms", "p99_ms", "mean_ms", "max_ms", "frames_per_s"):
        st[k] = round(st[k], 3)
    del srv, scenes
    torch.cuda.empty_cache()
    return st


# ----------------------------------------------------------- CPU baseline
def cpu_step(wl, orc):
    """One full step on the host cores (CPU oracle, FP32; the loss in FP64):
    preprocess and binning of all Gaussians, compositing of every tile, the
    loss on every pixel, the compositing adjoint and the factor gradients.
    Returns its seconds."""
    sc, cam, K, Q = wl["sc"], wl["cam"], wl["K"], wl["Q"]
    H, W = cam.height, cam.width
    t0 = time.perf_counter()
    pre = orc.preprocess(sc["pws"], sc["rots"], sc["scales"], cam, np.float32)
    w, _, ylm = orc.sh2weight_fast(sc["dc"], sc["A"], sc["B"], sc["pws"], pre["twc"], K, Q, True)
    b = orc.bin_gaussians(pre["us"], pre["areas"], pre["depths"], H, W)
    out, contrib, ft = orc.draw(H, W, K, b["ranges"], b["gsid"], pre["us"], pre["cinv"],
                                sc["alphas"], w, 0.0)
    tgt = wl["target_host"].numpy()
    lo = orc.palette_geo_loss(out, tgt, sc["palette"][2:], **LOSS)
    g = orc.draw_backward(H, W, K, b["ranges"], b["gsid"], pre["us"], pre["cinv"], sc["alphas"], w,
                          ft, contrib, lo["dlayer"].astype(np.float32))
    orc.sh2weight_fast_b(sc["A"], sc["B"], ylm, g["dfeat"], K, Q)
    return time.perf_counter() - t0


def cpu_baseline(wl, steps, warmup):
    from oracle import oracle as orc
    orc.set_threads(os.cpu_count() or 1)
    for _ in range(max(0, warmup)):
        cpu_step(wl, orc)
    secs = [cpu_step(wl, orc) for _ in range(max(1, steps))]
    v = len(secs) / sum(secs)
    return dict(value=v, unit="iters/s", cores=orc.get_threads(), kind="port",
                sample=(f"CPU oracle (FP32, from-scratch restatement of gsplatcu's kernels) on "
                        f"{orc.get_threads()} host threads: {len(secs)} full steps (all "
                        f"{wl['sc']['pws'].shape[0]} Gaussians preprocessed and binned, every "
                        f"tile composited forward and backward, the loss on every pixel), "
                        f"{sum(secs):.1f} s timed after {max(0, warmup)} warm-up steps"),
                ms_per_step=1000.0 * sum(secs) / len(secs), seconds=sum(secs))


def numpy_reference_forward(seed=0):
    """The reference's own numpy rasterizer (gsplat/gausplat.py, executed
    unchanged from oracle/_ref) on the 20k-Gaussian, 256x256 workload: project
    -> compute_cov_3d -> compute_cov_2d -> inverse_cov2d, the SH weights by its
    sh2color (3 channels at a time, so twice for K = 5; it adds its +0.5 bias),
    then splat twice (it is fixed at 3 channels).  Single-threaded numpy; its
    maths differs from the CUDA extension (a timing baseline, not an oracle).
    Returns None when the numpy path is not staged."""
    import contextlib
    import io
    from oracle.build_ref import reference_numpy_path
    from palette_b200.scene import look_at, synthetic_scene
    gp = reference_numpy_path()
    if gp is None:
        return None
    n, W, H = 20000, 256, 256
    sc = synthetic_scene(n, seed=seed, mode="full")
    cam = look_at((0.0, -8.0, 0.0), width=W, height=H, device="cpu")
    R, t = cam.Rcw.numpy().astype(np.float64), cam.tcw.numpy().astype(np.float64)
    twc = -R.T @ t
    shs = sc["shs"].reshape(n, 16, 5).astype(np.float64)
    # the numpy path's colour layout: band b, channel c at 3 b + c
    groups = [shs[:, :, 0:3], np.concatenate([shs[:, :, 3:5], np.zeros((n, 16, 1))], 2)]
    t0 = time.perf_counter()
    with contextlib.redirect_stdout(io.StringIO()):
        u, pc = gp.project(sc["pws"].astype(np.float64), R, t, cam.fx, cam.fy, cam.cx, cam.cy)
        cov3 = gp.compute_cov_3d(sc["scales"].astype(np.float64), sc["rots"].astype(np.float64))
        cov2 = gp.compute_cov_2d(pc, cam.fx, cam.fy, W, H, cov3, R)
        cinv, areas = gp.inverse_cov2d(cov2)
        alpha = sc["alphas"].reshape(-1).astype(np.float64)
        for g in groups:
            col = gp.sh2color(g.reshape(n, 48), sc["pws"].astype(np.float64), twc)
            gp.splat(H, W, u, cinv, alpha, pc[:, 2], col, areas)
    sec = time.perf_counter() - t0
    return dict(workload=f"{n} Gaussians, {W}x{H}, full SH weights K=5 (forward only)",
                forward_s=round(sec, 3), frames_per_s=round(1.0 / sec, 4), threads=1,
                source="gsplat/gausplat.py of the reference, unchanged")


# ------------------------------------------------------------------- arms
def run_reference(a):
    world, rank, local = dist_setup(a)
    if rank != 0:
        return
    wl = make_workload(a, torch.device("cpu"))
    cb = cpu_baseline(wl, a.steps, a.warmup)
    try:
        npy = numpy_reference_forward(a.seed)
    except Exception as e:  # a labelled extra: report, never fail the arm
        npy = dict(error=f"{type(e).__name__}: {e}")
    line = dict(metric=METRIC, value=cb["value"], unit="iters/s", n_gpus=a.gpus, steps=a.steps,
                warmup=a.warmup, ms_per_step=cb["ms_per_step"], higher_is_better=True,
                scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
                config=config(a), impl="reference",
                cpu_baseline={k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
                timed_seconds=round(cb["seconds"], 2),
                e2e=dict(value=cb["value"], unit="iters/s", h2d_bytes_per_step=0,
                         d2h_bytes_per_step=0),
                numpy_reference=npy)
    print(json.dumps(line), flush=True)


# ------------------------------------------------- reference extension leg
def _per_call_ms(fn, warmup=20, reps=200):
    """Median device time (ms) of one call of fn, CUDA events around each call
    on the current stream, synchronised after each call (the reference's
    operators synchronise inside every call anyway)."""
    st = torch.cuda.current_stream()
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = []
    for _ in range(reps):
        s.record(st)
        fn()
        e.record(st)
        e.synchronize()
        out.append(s.elapsed_time(e))
    return statistics.median(out)


def gpu_baseline_leg(a):
    """Run in a subprocess of the b200 arm (so that the reference extension is
    never loaded into the timed process): time the reference's own gsplatcu
    extension, built from its sources, through the reference's own autograd
    functions (gsplat/gsmodel.py WeightGSFunctionTest for full SH weights,
    WeightGSFunctionFast for rank-1 factors -- the only rank it supports),
    forward and forward + backward (dL/dlayer a fixed random image), on the
    bench scene's Gaussians and camera; beside it, on the same scenes and with
    the same method, this build through the same reference caller (drop-in),
    through palette_b200.weights (operator forward, fused weight adjoint) and
    through palette_b200.render (fused preprocess, weights-only adjoint).
    Prints one JSON line."""
    import gsplatcu
    from oracle.build_ref import load_ref, reference_caller
    from palette_b200.render import render_palette
    from palette_b200.scene import look_at, synthetic_scene
    from palette_b200.weights import splat_palette_weights
    ref = load_ref()
    gm_ref = reference_caller(ref, "ref") if ref is not None else None
    if gm_ref is None:
        print(json.dumps(dict(unavailable="reference build or caller missing under oracle/_ref")))
        return
    gm_b200 = reference_caller(gsplatcu, "b200")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    W, H, n = a.width, a.height, a.gaussians
    cam = look_at((0.0, -8.0, 0.0), width=W, height=H, device=dev)
    G = torch.randn((5, H, W), device=dev, generator=torch.Generator(dev).manual_seed(a.seed))
    clocks = ClockSampler(0)
    clocks.start()
    res = {}
    for form in ("full_sh", "rank1"):
        sc = synthetic_scene(n, seed=a.seed, mode="full" if form == "full_sh" else "lowrank",
                             rank=1)
        t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
        geo = (t(sc["pws"]), t(sc["alphas"]), t(sc["scales"]), t(sc["rots"]))
        pws, alphas, scales, rots = geo
        if form == "full_sh":
            shs = t(sc["shs"]).requires_grad_()
            leaves = [shs]
            calls = {
                "reference": lambda gm=gm_ref: gm.WeightGSFunctionTest.apply(
                    pws, shs, alphas, scales, rots, cam, 5)[0],
                "dropin": lambda gm=gm_b200: gm.WeightGSFunctionTest.apply(
                    pws, shs, alphas, scales, rots, cam, 5)[0],
                "ops": lambda: splat_palette_weights(pws, alphas, scales, rots, cam, shs=shs)[0],
                "fused": lambda: render_palette(pws, rots, scales, alphas, cam, shs=shs)[0],
            }
        else:
            dc, A, B = (t(sc["dc"]).requires_grad_(), t(sc["A"][:, :, 0]).requires_grad_(),
                        t(sc["B"][:, 0, :]).requires_grad_())
            leaves = [dc, A, B]
            calls = {
                "reference": lambda gm=gm_ref: gm.WeightGSFunctionFast.apply(
                    pws, dc, A, B, alphas, scales, rots, cam, 5, 15)[0],
                "dropin": lambda gm=gm_b200: gm.WeightGSFunctionFast.apply(
                    pws, dc, A, B, alphas, scales, rots, cam, 5, 15)[0],
                "ops": lambda: splat_palette_weights(pws, alphas, scales, rots, cam, dc=dc, A=A,
                                                     B=B)[0],
                "fused": lambda: render_palette(pws, rots, scales, alphas, cam, dc=dc, A=A,
                                                B=B)[0],
            }
        out = {}
        for name, fwd in calls.items():
            def fwd_only(fwd=fwd):
                with torch.no_grad():
                    fwd()

            def fwd_bwd(fwd=fwd):
                for x in leaves:
                    x.grad = None
                fwd().backward(G.reshape(5, H, W))
            out[name] = dict(forward_ms=round(_per_call_ms(fwd_only), 4),
                             fwd_bwd_ms=round(_per_call_ms(fwd_bwd), 4))
        r = out["reference"]
        for name in ("dropin", "ops", "fused"):
            out[name]["forward_speedup"] = round(r["forward_ms"] / out[name]["forward_ms"], 2)
            out[name]["fwd_bwd_speedup"] = round(r["fwd_bwd_ms"] / out[name]["fwd_bwd_ms"], 2)
        res[form] = out
        del sc, geo, leaves, calls
        torch.cuda.empty_cache()
    res["clocks"] = clocks.stop()
    res["method"] = ("median of 200 per-call CUDA-event times after 20 warm-up calls; forward: "
                     "layer under no_grad; fwd_bwd: layer.backward(fixed random dL/dlayer)")
    res["workload"] = f"{n} Gaussians, {W}x{H}, K=5, camera at distance 8"
    print(json.dumps(res), flush=True)


def run_gpu_baseline(a):
    """The reference-extension leg in a subprocess; its JSON, or a reason."""
    cmd = [sys.executable, os.path.abspath(__file__), "--gpu-baseline-leg",
           "--gaussians", str(a.gaussians), "--width", str(a.width), "--height", str(a.height),
           "--seed", str(a.seed)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    except subprocess.TimeoutExpired:
        return dict(unavailable="reference-extension leg timed out")
    lines = [x for x in r.stdout.strip().splitlines() if x.startswith("{")]
    if r.returncode != 0 or not lines:
        return dict(unavailable=f"reference-extension leg failed (rc {r.returncode}): "
                                f"{r.stderr.strip().splitlines()[-1:] }")
    return json.loads(lines[-1])


def config(a):
    return dict(workload=(f"palette-weight finetune step, low-rank fused path: {a.gaussians} "
                          f"Gaussians, {a.width}x{a.height}, rank-{a.rank} factors P=5 Q=15, K=5, "
                          "SH order 3, FP32 storage, L1 loss against the clamped and renormalised "
                          "barycentric palette target + 0.5 negative-weight penalty"),
                gaussians=a.gaussians, width=a.width, height=a.height, rank=a.rank,
                parallelism="replicas" if a.gpus > 1 else "single-gpu",
                l2="inputs larger than L2 (scene parameters ~%d MB > 126 MB L2)"
                   % int(a.gaussians * 4 * (3 + 4 + 3 + 1 + 5 + 15 * a.rank + 5 * a.rank) / 1e6))


def run_b200(a):
    world, rank, local = dist_setup(a)
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: CUDA is required for --impl b200 (no CPU fallback)")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    from gsplatcu import _lib
    L = _lib.lib()
    wl = make_workload(a, device)
    stream = torch.cuda.current_stream()
    for _ in range(max(3, a.warmup)):
        step(wl)
    torch.cuda.synchronize()

    # timed region: K fwd+bwd steps
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = L.gsb_launch_count()
    ms = timed(lambda: step(wl), a.steps, stream)
    launches = int(L.gsb_launch_count() - l0)
    clk = clocks.stop()
    barrier(world)
    ms = allreduce_max(ms, world, device)
    ms_per_step = ms / a.steps
    value = world * a.steps / (ms / 1000.0)

    # forward only (its own warm-up: the first forward-only steps after the
    # training steps reallocate)
    with torch.no_grad():
        for _ in range(max(3, a.warmup)):
            step(wl, backward=False)
        fms = timed(lambda: step(wl, backward=False), a.steps, stream) / a.steps
    fms = allreduce_max(fms, world, device)

    # end to end: every step copies its inputs (camera, target image) from pinned
    # host memory and reads its loss back into pinned host memory.  The inputs
    # of step i+1 -- the camera (R, t and centre: 60 bytes in one pinned buffer)
    # and the target -- are copied on a side stream while step i computes (an
    # input pipeline that prefetches one step ahead, into the buffers step i-1
    # used), and each step's loss is read back on a third stream once the step
    # is done, so that no copy sits between two steps' kernels on the compute
    # stream.  All copies fall inside the timed region.
    cam = wl["cam"]
    cam_h = torch.cat([cam.Rcw.reshape(-1), cam.tcw.reshape(-1), cam.twc.reshape(-1)]).cpu()
    cam_h = cam_h.pin_memory()
    loss_h = torch.empty((), dtype=torch.float32).pin_memory()
    tgt_d = [torch.empty_like(wl["target"]) for _ in range(2)]
    cam_d = [torch.empty(cam_h.shape, dtype=cam_h.dtype, device=device) for _ in range(2)]
    copy_stream = torch.cuda.Stream(device)
    read_stream = torch.cuda.Stream(device)
    copied = [torch.cuda.Event() for _ in range(2)]
    used = [torch.cuda.Event() for _ in range(2)]
    from palette_b200.scene import Camera

    def prefetch(slot):
        with torch.cuda.stream(copy_stream):
            copy_stream.wait_event(used[slot])  # the step that last read these buffers
            cam_d[slot].copy_(cam_h, non_blocking=True)
            tgt_d[slot].copy_(wl["target_host"], non_blocking=True)
            copied[slot].record(copy_stream)

    def e2e_run(k, start=None):
        if start is not None:
            copy_stream.wait_event(start)
        prefetch(0)
        for i in range(k):
            slot = i % 2
            if i + 1 < k:
                prefetch((i + 1) % 2)
            stream.wait_event(copied[slot])
            cd = cam_d[slot]
            c = Camera(0, cam.width, cam.height, cam.fx, cam.fy, cam.cx, cam.cy,
                       cd[:9].view(3, 3), cd[9:12], twc=cd[12:15])
            loss = step(wl, cam=c, target=tgt_d[slot])
            used[slot].record(stream)
            with torch.cuda.stream(read_stream):
                read_stream.wait_event(used[slot])
                loss = loss.detach()
                loss.record_stream(read_stream)  # not recycled before the copy ran
                loss_h.copy_(loss, non_blocking=True)
        stream.wait_stream(read_stream)  # the last read-back inside the timed region
    for _ in range(2):
        e2e_run(2)
    torch.cuda.synchronize()
    barrier(world)
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    e2e_run(a.steps, e_start)
    e_end.record(stream)
    torch.cuda.synchronize()
    ems = allreduce_max(e_start.elapsed_time(e_end), world, device)
    h2d = int((cam_h.numel() + wl["target_host"].numel()) * 4)

    # the fused render path, same workload
    for _ in range(3):
        step_fused(wl)
    fu_ms = allreduce_max(timed(lambda: step_fused(wl), a.steps, stream), world, device) / a.steps
    with torch.no_grad():
        fu_fms = allreduce_max(timed(lambda: step_fused(wl, backward=False), a.steps, stream),
                               world, device) / a.steps

    # the multi-view finetune leg (8 views per step, BF16 factors, L1 + SSIM)
    mv = make_views(wl, a, device)
    for _ in range(3):
        step_views(wl, mv)
    mv_reps = max(2, a.steps // 4)
    mv_ms = allreduce_max(timed(lambda: step_views(wl, mv), mv_reps, stream), world, device) / mv_reps
    del mv

    stages, alg = stage_breakdown(wl)
    dom = max(("draw", "draw_backward"), key=lambda k: stages[k])
    dom_bytes = alg["bytes_draw"] if dom == "draw" else alg["bytes_bwd"]
    peak, peak_kind = measured_peaks()
    achieved = dom_bytes / (stages[dom] / 1000.0) / 1e9
    tag = {"draw": "k_draw_1M_1080p", "draw_backward": "k_draw_backward_1M_1080p"}[dom]
    roof = dict(bound="hbm", kernel=f"k_{dom}", achieved=round(achieved, 1), peak=peak,
                unit="GB/s", frac=round(achieved / peak, 4),
                traffic=profile_figure(tag, "traffic_bytes_per_launch"),
                algorithmic_bytes=int(dom_bytes), launch_ms=round(stages[dom], 4),
                warp_inst_per_launch=profile_figure(tag, "warp_inst_per_launch"),
                inst_per_blended_pair=profile_figure(tag, "inst_per_blended_pair"),
                bound_note="issue-bound: the HBM fraction is low by construction; "
                           "warp instructions per blended (pixel, Gaussian) pair is the figure "
                           "the kernel design moves",
                peak_source=f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s")

    # the serving loop is per GPU (replicas): measured on one GPU, not repeated
    # on every rank of a scaling run
    serving = serve_bench(a, device) if a.serve_seconds > 0 and world == 1 else None

    cb = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cb = cpu_baseline(wl, steps=3, warmup=1)
        cb = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    gb = None
    if rank == 0 and world == 1 and not a.no_gpu_baseline:
        gb = run_gpu_baseline(a)
    if rank == 0:
        line = dict(metric=METRIC, value=round(value, 3), unit="iters/s", n_gpus=world,
                    steps=a.steps, warmup=a.warmup, ms_per_step=round(ms_per_step, 4),
                    higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
                    data="synthetic (seeded; distributions of the benchmark configs)",
                    config=config(a),
                    frames_per_s=round(world * 1000.0 / fms, 2), forward_ms=round(fms, 4),
                    e2e=dict(value=round(world * a.steps / (ems / 1000.0), 3), unit="iters/s",
                             h2d_bytes_per_step=h2d, d2h_bytes_per_step=4,
                             input_pipeline="next step's camera and target copied on a side "
                                            "stream while this step computes; each loss read "
                                            "back on a third stream"),
                    gpu_launches=launches, clocks=clk, roofline=roof, cpu_baseline=cb,
                    fused_path=dict(iters_per_s=round(world * 1000.0 / fu_ms, 3),
                                    ms_per_step=round(fu_ms, 4), forward_ms=round(fu_fms, 4),
                                    frames_per_s=round(world * 1000.0 / fu_fms, 2)),
                    multiview=dict(views_per_step=VIEWS, storage="bf16 dc/A/B, FP32 arithmetic",
                                   loss="0.8 L1 + 0.2 (1 - SSIM) + 0.5 mean(relu(-W))",
                                   steps=mv_reps, ms_per_step=round(mv_ms, 4),
                                   iters_per_s=round(world * 1000.0 / mv_ms, 3),
                                   views_per_s=round(world * VIEWS * 1000.0 / mv_ms, 2)),
                    serving=serving, gpu_baseline=gb,
                    stages_ms={k: round(v, 4) for k, v in stages.items()},
                    patches=alg["M"],
                    # sort throughput and the compositing's nominal pixel work
                    # (every patch against the 256 pixels of its tile)
                    sort_keys_per_s=round(alg["M"] / (stages["bin_sort"] / 1000.0), 1),
                    draw_evaluations_per_s=round(alg["M"] * 256 / (stages["draw"] / 1000.0), 1))
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    a = parse()
    if a.gpu_baseline_leg:
        gpu_baseline_leg(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
