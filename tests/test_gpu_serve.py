"""GPU tests of the palette-edit serving path: the capacity-sized tile sort,
the palette-colour render against the reference's bake-and-render sequence
(gsplat/gsmodel.py:488-509 + 14-26, run through gsplatcu), continuous
batching through the persistent batched compositing kernel (each image
identical alone and in the mix), HBM admission, and re-rendering after a
capacity overflow.  Tolerances: sort outputs bit-exact;
images 1e-5 abs against the bake-and-render sequence (a different FP32
summation order of the same linear map); mix vs alone bit-exact (same kernels
and inputs, no atomics in the forward)."""
import ctypes as C

import numpy as np
import pytest
import torch

import gsplatcu as gsc
from gsplatcu import _lib
from palette_b200.scene import Camera, look_at, sphere_poses, synthetic_scene, to_torch
from palette_b200.serve import MAX_DEPTH_KEY, PaletteServer, Request, Scene
from helpers import max_abs

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5


def _scene(sid, n, seed, mode="full", dtype=torch.float32, rank=3):
    sc = synthetic_scene(n, seed=seed, mode=mode, rank=rank)
    st = to_torch(sc, "cuda", dtype)
    if mode == "full":
        return Scene(sid, st["pws"], st["rots"], st["scales"], st["alphas"], shs=st["shs"]), sc
    return Scene(sid, st["pws"], st["rots"], st["scales"], st["alphas"], dc=st["dc"], A=st["A"],
                 B=st["B"]), sc


def _request(sid, eye, W, H, palette, tag=None):
    cam = look_at(eye, width=W, height=H, device="cpu")
    return Request(sid, cam.Rcw.numpy(), cam.tcw.numpy(), cam.fx, cam.fy, cam.cx, cam.cy, W, H,
                   palette, tag=tag)


def _res(W, H):
    cam = look_at((0, -8, 0), width=W, height=H, device="cpu")
    return (W, H, cam.fx, cam.fy, cam.cx, cam.cy)


def _probes(radius=6.0):
    out = []
    for eye in sphere_poses(6, radius, seed=9):
        c = look_at(eye, device="cpu")
        out.append((c.Rcw.numpy(), c.tcw.numpy()))
    return out


def _edit(palette, seed):
    rng = np.random.default_rng(seed)
    p = np.array(palette, np.float32)
    p[2:] = np.clip(p[2:] + rng.normal(0, 0.15, p[2:].shape), 0, 1)
    return p


def _bake_and_render(scene, req):
    """The reference's palette-edit render through gsplatcu: bake the palette
    into RGB SH coefficients, then sh2Color + splat_color (render_vanilla)."""
    K = scene.K
    if scene.mode == _lib.WEIGHTS_FULL:
        shs_w = scene.shs.float().reshape(scene.n, 16, K)
    else:
        A = scene.A.float() if scene.A.dim() == 3 else scene.A.float()[:, :, None]
        B = scene.B.float() if scene.B.dim() == 3 else scene.B.float()[:, None, :]
        Cm = torch.bmm(A, B).reshape(scene.n, 15, K)
        shs_w = torch.cat([scene.w0.float()[:, None, :], Cm], dim=1)
    P = req.palette.cuda()
    baked = torch.einsum("nlk,kc->nlc", shs_w, P).reshape(scene.n, 48).contiguous()
    cam = Camera(0, req.width, req.height, req.fx, req.fy, req.cx, req.cy, req.Rcw.cuda(),
                 req.tcw.cuda(), twc=req.twc.cuda())
    us, pcs, depths = gsc.project(scene.pws, cam.Rcw, cam.tcw, req.fx, req.fy, req.cx, req.cy, False)
    cov3, = gsc.computeCov3D(scene.rots, scene.scales, depths, False)
    cov2, = gsc.computeCov2D(cov3, pcs, cam.Rcw, depths, req.fx, req.fy, req.width, req.height,
                             False)
    colors, = gsc.sh2Color(baked, scene.pws, cam.twc, False)
    cinv, areas = gsc.inverseCov2D(cov2, depths, False)
    image, _, _, _, _ = gsc.splat_color(req.height, req.width, us, cinv, scene.alphas, depths,
                                        colors, areas)
    return image


def test_capacity_sort_matches_exact_sort_and_flags_overflow(cuda_ok):
    scene, sc = _scene("s", 20000, 3)
    n, W, H = scene.n, 256, 192
    cam = look_at((0.5, -7.0, 1.0), width=W, height=H, device="cuda")
    pal = torch.tensor(sc["palette"], device="cuda")
    camst = _lib.Camera(cam.Rcw.data_ptr(), cam.tcw.data_ptr(), cam.twc.data_ptr(), cam.fx, cam.fy,
                        cam.cx, cam.cy, W, H)
    params = scene.params(pal)
    L = _lib.lib()
    state = torch.empty(int(L.gsb_splat_state_bytes(n, 3, H, W)), dtype=torch.uint8, device="cuda")
    _lib.call("t", "gsb_render_preprocess", n, C.byref(camst), _lib.ptr(scene.pws),
              _lib.ptr(scene.rots), _lib.ptr(scene.scales), _lib.ptr(scene.alphas),
              C.byref(params), _lib.ptr(state), None, None)
    plan = _lib.SplatPlan()
    _lib.call("t", "gsb_splat_counts", n, H, W, _lib.ptr(state), C.byref(plan), None)
    M, tiles = int(plan.patches), ((W + 15) // 16) * ((H + 15) // 16)
    ws = torch.empty(int(L.gsb_splat_sort_bytes(n, H, W, C.byref(plan))), dtype=torch.uint8,
                     device="cuda")
    g_ref = torch.empty(M, dtype=torch.int32, device="cuda")
    r_ref = torch.empty((tiles, 2), dtype=torch.int32, device="cuda")
    _lib.call("t", "gsb_splat_sort", n, H, W, C.byref(plan), _lib.ptr(state), _lib.ptr(ws),
              _lib.ptr(g_ref), _lib.ptr(r_ref), None)
    status = torch.full((4,), -1, dtype=torch.int32, device="cuda")
    for cap, dkey in ((M, MAX_DEPTH_KEY), (3 * M + 5000, MAX_DEPTH_KEY), (M, (1 << 30))):
        ws2 = torch.empty(int(L.gsb_splat_sort_capacity_bytes(n, H, W, cap, dkey)),
                          dtype=torch.uint8, device="cuda")
        g = torch.full((cap,), -3, dtype=torch.int32, device="cuda")
        r = torch.full((tiles, 2), -3, dtype=torch.int32, device="cuda")
        _lib.call("t", "gsb_splat_sort_capacity", n, H, W, cap, dkey, _lib.ptr(state),
                  _lib.ptr(ws2), _lib.ptr(g), _lib.ptr(r), _lib.ptr(status), None)
        assert int(status[0]) == 0 and int(status[1]) == M and int(status[2]) == 0
        assert torch.equal(g[:M], g_ref) and torch.equal(r, r_ref)
    # overflow: capacity below the patch count, and depth keys wider than allowed
    for cap, dkey, bit in ((M // 2, MAX_DEPTH_KEY, _lib.STATUS_PATCH_OVERFLOW),
                           (M, 3, _lib.STATUS_DEPTH_KEY_OVERFLOW)):
        ws2 = torch.empty(int(L.gsb_splat_sort_capacity_bytes(n, H, W, cap, dkey)),
                          dtype=torch.uint8, device="cuda")
        g = torch.empty((cap,), dtype=torch.int32, device="cuda")
        r = torch.full((tiles, 2), -3, dtype=torch.int32, device="cuda")
        _lib.call("t", "gsb_splat_sort_capacity", n, H, W, cap, dkey, _lib.ptr(state),
                  _lib.ptr(ws2), _lib.ptr(g), _lib.ptr(r), _lib.ptr(status), None)
        assert int(status[0]) & bit
        assert torch.count_nonzero(r) == 0


@pytest.mark.parametrize("mode,dtype", [("full", torch.float32), ("lowrank", torch.bfloat16),
                                        ("lowrank", torch.float32)])
def test_palette_edit_render_matches_bake_and_render(cuda_ok, mode, dtype):
    scene, sc = _scene("a", 30000, 5, mode, dtype)
    srv = PaletteServer(hbm_budget=4 << 30, slots=2)
    res = [_res(320, 240), _res(256, 256)]
    assert srv.admit_scene(scene, res, _probes())
    for i, (W, H) in enumerate(((320, 240), (256, 256))):
        req = _request("a", sphere_poses(4, 7.0, seed=i)[i], W, H, _edit(sc["palette"], i))
        img = srv.render_alone(req)
        ref = _bake_and_render(scene, req)
        assert img.shape == (3, H, W)
        assert max_abs(img, ref) < IMG_TOL
        assert torch.count_nonzero(img) > 0


def test_continuous_batching_mix_equals_alone(cuda_ok):
    scenes = [_scene("f32", 40000, 11, "full")[0],
              _scene("bf16", 60000, 12, "lowrank", torch.bfloat16)[0],
              _scene("lr32", 20000, 13, "lowrank", torch.float32, rank=1)[0]]
    res = [_res(320, 240), _res(480, 272)]
    srv = PaletteServer(hbm_budget=8 << 30, slots=3)
    for s in scenes:
        assert srv.admit_scene(s, res, _probes())
    base_pal = synthetic_scene(10, seed=1)["palette"]
    reqs = []
    rng = np.random.default_rng(0)
    eyes = sphere_poses(12, (6.0, 10.0), seed=4)
    for i in range(12):
        s = scenes[i % 3]
        W, H = res[(i // 3) % 2][:2]
        reqs.append(lambda i=i, s=s, W=W, H=H: _request(s.id, eyes[i], W, H, _edit(base_pal, i),
                                                        tag=i))
    alone = {}
    for mk in reqs:
        r = mk()
        alone[r.tag] = srv.render_alone(r).clone()
    srv.prepare([mk() for mk in reqs])
    mix = [mk() for mk in reqs]
    for r in mix:  # all arrive at once: slots fill, the rest queue
        srv.submit(r)
    n0 = len(srv.batch_sizes)
    busy = srv.poll()
    assert busy == 3 and len(srv.queue) == 9
    srv.drain()
    assert len({r.slot for r in mix}) == 3
    # the mix was composited in shared persistent launches (several requests
    # of different scenes and resolutions per batch)
    assert max(srv.batch_sizes[n0:]) > 1
    for r in mix:
        assert torch.equal(r.image, alone[r.tag]), r.tag


def test_admission_by_hbm_budget_and_eviction(cuda_ok):
    a, _ = _scene("a", 50000, 21)
    b, _ = _scene("b", 50000, 22)
    res = [_res(320, 240)]
    srv = PaletteServer(hbm_budget=1 << 30, slots=2)
    assert srv.admit_scene(a, res, _probes())
    used = srv.resident_bytes()
    srv.budget = used + b.bytes // 2  # too small for b
    assert not srv.admit_scene(b, res, _probes())
    assert "b" not in srv.scenes and srv.resident_bytes() == used
    srv.evict_scene("a")
    assert srv.admit_scene(b, res, _probes())
    with pytest.raises(KeyError):
        srv.render_alone(_request("b", (0, -8, 0), 640, 480, np.ones((5, 3), np.float32)))


def test_capacity_overflow_rerenders(cuda_ok):
    scene, sc = _scene("a", 30000, 31)
    res = [_res(320, 240)]
    big = PaletteServer(hbm_budget=4 << 30, slots=1)
    assert big.admit_scene(scene, res, _probes())
    small = PaletteServer(hbm_budget=4 << 30, slots=1, capacity_margin=0.05)
    assert small.admit_scene(scene, res, _probes(radius=12.0))
    req1 = _request("a", (0.3, -6.0, 0.4), 320, 240, sc["palette"])
    req2 = _request("a", (0.3, -6.0, 0.4), 320, 240, sc["palette"])
    img = small.render_alone(req1)
    assert req1.reruns >= 1
    assert torch.equal(img, big.render_alone(req2))


def test_open_loop_poisson_stream(cuda_ok):
    scenes = [_scene("x", 50000, 41)[0], _scene("y", 80000, 42, "lowrank", torch.bfloat16)[0]]
    res = [_res(320, 240), _res(640, 480)]
    srv = PaletteServer(hbm_budget=8 << 30, slots=4, keep_images=False)
    for s in scenes:
        assert srv.admit_scene(s, res, _probes())
    pal = synthetic_scene(10, seed=1)["palette"]
    eyes = sphere_poses(40, (6.0, 10.0), seed=5)
    reqs = [_request(scenes[i % 2].id, eyes[i], *res[(i // 2) % 2][:2], _edit(pal, i))
            for i in range(40)]
    srv.prepare(reqs)
    st = srv.run_open_loop(reqs, rate=400.0)
    assert st["requests"] == 40
    assert 0 < st["p50_ms"] <= st["p99_ms"] and st["frames_per_s"] > 0
