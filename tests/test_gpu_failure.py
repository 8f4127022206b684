"""Failure detection without a GPU fault.

* Bounded device waits: ``gsb_debug_expire_bulk_wait`` arms an mbarrier for a
  transaction that no copy delivers and waits a short, bounded number of
  polls; the wait runs out and the kernel sets the same status bit the
  staging kernels set when a bulk copy never completes, then returns (no copy
  is in flight, the context stays usable).  The operators must then raise
  ``GsplatError`` with ``status == GSB_ERR_DEVICE_TIMEOUT`` at their next
  read-back -- where the reference printed CUDA errors and went on
  (gsplatcu/common.cuh:19-25) -- and work normally once it has been reported.
* Serving admission under host-side allocation failure: an allocator that
  fails part-way through growing the slot workspaces makes ``admit_scene``
  refuse the scene and leave the server consistent; a later admission with a
  working allocator renders exactly as a server that never failed."""
import ctypes as C

import numpy as np
import pytest
import torch

import gsplatcu as gsc
from gsplatcu import _lib
from gsplatcu._lib import GsplatError
from palette_b200.scene import look_at, synthetic_scene, to_torch
from palette_b200.serve import PaletteServer, Request, Scene
from helpers import forward_ops

pytestmark = pytest.mark.gpu


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _expire():
    _lib.call("test", "gsb_debug_expire_bulk_wait", 64, _stream())


def _device_bits():
    v = C.c_uint32(0)
    _lib.call("test", "gsb_device_status", C.byref(v), 0, _stream())
    return int(v.value)


def test_expired_wait_sets_status_and_check_raises(cuda_ok):
    gsc.check_device_status()  # clean start
    _expire()
    assert _device_bits() & _lib.STATUS_BULK_TIMEOUT
    _lib.fetch_device_status(torch.device("cuda", torch.cuda.current_device()), _stream())
    with pytest.raises(GsplatError) as e:
        gsc.check_device_status()
    assert e.value.status == _lib.GSB_ERR_DEVICE_TIMEOUT
    # reported once, then cleared on the device and the host
    assert _device_bits() == 0
    gsc.check_device_status()


def test_forward_raises_at_its_readback_then_recovers(cuda_ok):
    sc = synthetic_scene(20000, seed=4, mode="lowrank", rank=3)
    st = to_torch(sc, "cuda")
    cam = look_at((0.0, -8.0, 0.0), width=256, height=256)
    gsc.check_device_status()
    clean = forward_ops(gsc, st, cam, "lowrank")
    _expire()
    # sh2Weight_fast's status fetch picks the bit up; splat_weight raises
    # at its patch-count read-back
    with pytest.raises(GsplatError) as e:
        forward_ops(gsc, st, cam, "lowrank")
    assert e.value.status == _lib.GSB_ERR_DEVICE_TIMEOUT
    again = forward_ops(gsc, st, cam, "lowrank")
    for k in ("layer", "contrib", "final_tau", "gsid", "ranges"):
        assert torch.equal(clean[k], again[k]), k
    gsc.check_device_status()


def test_fused_render_raises_then_recovers(cuda_ok):
    from palette_b200.render import render_palette
    sc = synthetic_scene(20000, seed=5, mode="full")
    st = to_torch(sc, "cuda")
    cam = look_at((1.0, -7.0, 1.0), width=200, height=120)
    gsc.check_device_status()
    ref = render_palette(st["pws"], st["rots"], st["scales"], st["alphas"], cam, shs=st["shs"])
    _expire()
    with pytest.raises(GsplatError) as e:
        render_palette(st["pws"], st["rots"], st["scales"], st["alphas"], cam, shs=st["shs"])
    assert e.value.status == _lib.GSB_ERR_DEVICE_TIMEOUT
    out = render_palette(st["pws"], st["rots"], st["scales"], st["alphas"], cam, shs=st["shs"])
    assert torch.equal(out[0], ref[0]) and torch.equal(out[1], ref[1])


def _serve_scene(sid, n, seed):
    sc = synthetic_scene(n, seed=seed, mode="full")
    st = to_torch(sc, "cuda")
    return Scene(sid, st["pws"], st["rots"], st["scales"], st["alphas"], shs=st["shs"]), sc


def _res(W, H):
    cam = look_at((0, -8, 0), width=W, height=H, device="cpu")
    return (W, H, cam.fx, cam.fy, cam.cx, cam.cy)


def _probes():
    c = look_at((0.0, -7.0, 0.5), device="cpu")
    return [(c.Rcw.numpy(), c.tcw.numpy())]


def _req(sid, palette, W, H):
    cam = look_at((0.0, -7.0, 0.5), width=W, height=H, device="cpu")
    return Request(sid, cam.Rcw.numpy(), cam.tcw.numpy(), cam.fx, cam.fy, cam.cx, cam.cy, W, H,
                   palette)


class _FailingAlloc:
    """torch.empty on the GPU that raises torch.OutOfMemoryError on the
    `fail_at`-th call (host-side fault injection)."""

    def __init__(self, fail_at):
        self.calls, self.fail_at = 0, fail_at

    def __call__(self, shape, dtype):
        self.calls += 1
        if self.calls == self.fail_at:
            raise torch.OutOfMemoryError("injected allocation failure")
        return torch.empty(shape, dtype=dtype, device="cuda")


@pytest.mark.parametrize("fail_at", [1, 3, 9])
def test_serve_admission_survives_allocation_failure(cuda_ok, fail_at):
    W, H = 640, 360
    scene, sc = _serve_scene("s0", 50000, 7)
    alloc = _FailingAlloc(fail_at)
    srv = PaletteServer(8 << 30, slots=2, alloc=alloc)
    before = srv.resident_bytes()
    assert not srv.admit_scene(scene, [_res(W, H)], _probes())
    assert "allocation failed" in srv.last_admit_error
    assert "s0" not in srv.scenes and not srv.buckets
    # slots are whole: either their old (empty) buffers or a complete new set
    for sl in srv.slots:
        assert sl.bytes() == 0 or set(sl.buf) == {"state", "sort", "gsid", "ranges", "image",
                                                   "contrib", "final_tau"}
    assert srv.resident_bytes() >= before
    # the allocator works again: admission succeeds, the render matches a
    # server that never failed
    alloc.fail_at = -1
    assert srv.admit_scene(scene, [_res(W, H)], _probes())
    pal = sc["palette"]
    img = srv.render_alone(_req("s0", pal, W, H))
    good = PaletteServer(8 << 30, slots=2)
    assert good.admit_scene(scene, [_res(W, H)], _probes())
    ref = good.render_alone(_req("s0", pal, W, H))
    assert torch.equal(img, ref)


def test_serve_reports_expired_wait(cuda_ok):
    gsc.check_device_status()  # clean start
    W, H = 320, 180
    scene, sc = _serve_scene("s1", 20000, 8)
    srv = PaletteServer(4 << 30, slots=1)
    assert srv.admit_scene(scene, [_res(W, H)], _probes())
    pal = sc["palette"]
    ok = srv.render_alone(_req("s1", pal, W, H))
    _expire()
    with pytest.raises(GsplatError) as e:
        srv.render_alone(_req("s1", pal, W, H))
    assert e.value.status == _lib.GSB_ERR_DEVICE_TIMEOUT
    srv.queue.clear()
    again = srv.render_alone(_req("s1", pal, W, H))
    assert torch.equal(ok, again)
