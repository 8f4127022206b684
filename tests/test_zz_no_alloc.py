"""GPU test of gsb_splat_sort_static, the tile sort for callers that cannot
allocate device memory where they render (device memory owned by another
runtime's pool, plug-ins handed only their buffers).  Its temporaries live in
a fixed device array inside the library; this checks, through the C ABI,
that two calls in a row -- different scenes, image sizes and key widths, so
the second runs over what the first left in the array -- give exactly the
tile lists and ranges of gsb_splat_sort with a caller workspace (sorting is
integer work: bit-exact), and that a plan beyond the array's size is refused
before anything runs.  Kept in a file that pytest collects last."""
import ctypes as C

import numpy as np
import pytest
import torch

import gsplatcu as gsc
from gsplatcu import _lib
from palette_b200.scene import look_at, synthetic_scene, to_torch

pytestmark = pytest.mark.gpu


def _packed(n, W, H, seed, scale):
    """A packed splat state for a synthetic scene (the splat_weight inputs of
    the reference op sequence), plus its plan."""
    sc = synthetic_scene(n, seed=seed)
    sc["pws"] = sc["pws"] * scale
    sc["scales"] = sc["scales"] * scale
    st = to_torch(sc, "cuda")
    cam = look_at((0.0, -8.0 * scale, 0.0), width=W, height=H, device="cuda")
    us, pcs, depths = gsc.project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy,
                                  False)
    cov3, = gsc.computeCov3D(st["rots"], st["scales"], depths, False)
    cov2, = gsc.computeCov2D(cov3, pcs, cam.Rcw, depths, cam.fx, cam.fy, W, H, False)
    cinv, areas = gsc.inverseCov2D(cov2, depths, False)
    w, = gsc.sh2Weight(st["shs"], st["pws"], cam.twc, False, 5)
    L = _lib.lib()
    state = torch.empty(int(L.gsb_splat_state_bytes(n, 5, H, W)), dtype=torch.uint8,
                        device="cuda")
    s = _lib.stream_of(us)
    _lib.call("pack", "gsb_splat_pack", n, H, W, 5, _lib.ptr(us), _lib.ptr(cinv),
              _lib.ptr(st["alphas"]), _lib.ptr(w), _lib.DTYPE_F32, _lib.ptr(depths),
              _lib.ptr(areas), _lib.ptr(state), s)
    plan = _lib.SplatPlan()
    _lib.call("counts", "gsb_splat_counts", n, H, W, _lib.ptr(state), C.byref(plan), s)
    return state, plan, s


def _sort_with_workspace(n, W, H, state, plan, s):
    L = _lib.lib()
    M, tiles = int(plan.patches), ((W + 15) // 16) * ((H + 15) // 16)
    ws = torch.empty(max(1, int(L.gsb_splat_sort_bytes(n, H, W, C.byref(plan)))),
                     dtype=torch.uint8, device="cuda")
    gsid = torch.empty((M,), dtype=torch.int32, device="cuda")
    ranges = torch.empty((tiles, 2), dtype=torch.int32, device="cuda")
    _lib.call("sort", "gsb_splat_sort", n, H, W, C.byref(plan), _lib.ptr(state), _lib.ptr(ws),
              _lib.ptr(gsid), _lib.ptr(ranges), s)
    return gsid, ranges


def _sort_static(n, W, H, state, plan, s):
    M, tiles = int(plan.patches), ((W + 15) // 16) * ((H + 15) // 16)
    gsid = torch.full((M,), -7, dtype=torch.int32, device="cuda")
    ranges = torch.full((tiles, 2), -7, dtype=torch.int32, device="cuda")
    _lib.call("sort_static", "gsb_splat_sort_static", n, H, W, C.byref(plan), _lib.ptr(state),
              _lib.ptr(gsid), _lib.ptr(ranges), s)
    return gsid, ranges


def _key_bits(W, H, plan):
    tiles = ((W + 15) // 16) * ((H + 15) // 16)
    return int(tiles - 1).bit_length() + int(plan.max_depth_key).bit_length()


def test_static_sort_matches_workspace_sort_twice_in_a_row(cuda_ok):
    L = _lib.lib()
    cases = [  # (n, W, H, seed, scale): 32-bit keys, then 64-bit keys at another size
        (20000, 256, 256, 3, 1.0),
        (60000, 1920, 1080, 4, 400.0),
    ]
    widths = []
    for n, W, H, seed, scale in cases:
        state, plan, s = _packed(n, W, H, seed, scale)
        assert plan.patches > 0
        assert L.gsb_splat_sort_bytes(n, H, W, C.byref(plan)) <= L.gsb_splat_sort_static_max_bytes()
        g_ref, r_ref = _sort_with_workspace(n, W, H, state, plan, s)
        g, r = _sort_static(n, W, H, state, plan, s)
        torch.cuda.synchronize()
        assert torch.equal(g, g_ref)
        assert torch.equal(r, r_ref)
        widths.append(_key_bits(W, H, plan) > 32)
    assert widths == [False, True]


def test_static_sort_allocates_no_device_memory(cuda_ok):
    """The defining property: after one warm-up call (which looks up the
    array's address), a further call changes neither the device's free
    memory nor what torch's caching allocator holds."""
    n, W, H = 20000, 256, 256
    state, plan, s = _packed(n, W, H, 11, 1.0)
    M, tiles = int(plan.patches), ((W + 15) // 16) * ((H + 15) // 16)
    gsid = torch.empty((M,), dtype=torch.int32, device="cuda")
    ranges = torch.empty((tiles, 2), dtype=torch.int32, device="cuda")
    args = (n, H, W, C.byref(plan), _lib.ptr(state), _lib.ptr(gsid), _lib.ptr(ranges), s)
    _lib.call("sort_static", "gsb_splat_sort_static", *args)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    res0, alloc0 = torch.cuda.memory_reserved(), torch.cuda.memory_allocated()
    _lib.call("sort_static", "gsb_splat_sort_static", *args)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_reserved() == res0 and torch.cuda.memory_allocated() == alloc0
    g_ref, r_ref = _sort_with_workspace(n, W, H, state, plan, s)
    assert torch.equal(gsid, g_ref) and torch.equal(ranges, r_ref)


def test_static_sort_refuses_plans_beyond_its_array(cuda_ok):
    L = _lib.lib()
    n, W, H = 1000, 1920, 1080
    state = torch.zeros(int(L.gsb_splat_state_bytes(n, 5, H, W)), dtype=torch.uint8,
                        device="cuda")
    plan = _lib.SplatPlan(patches=3_000_000, max_depth_key=20000, reserved=0)
    assert L.gsb_splat_sort_bytes(n, H, W, C.byref(plan)) > L.gsb_splat_sort_static_max_bytes()
    gsid = torch.empty((1,), dtype=torch.int32, device="cuda")
    ranges = torch.empty((8160, 2), dtype=torch.int32, device="cuda")
    l0 = L.gsb_launch_count()
    with pytest.raises(_lib.GsplatError, match="sort scratch"):
        _lib.call("sort_static", "gsb_splat_sort_static", n, H, W, C.byref(plan),
                  _lib.ptr(state), _lib.ptr(gsid), _lib.ptr(ranges), None)
    assert L.gsb_launch_count() == l0
