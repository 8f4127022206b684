"""Palette-edit render serving on one GPU.

A ``PaletteServer`` keeps finetuned scenes resident in HBM and renders
palette-edit requests -- (scene, camera, resolution, edited palette) -> RGB
image -- with continuous batching:

* Scenes are admitted by their HBM footprint (parameters plus the growth of
  the per-slot render workspaces they need) against a byte budget, and can be
  evicted to make room.  Admission survives a failed workspace allocation
  (the scene is refused, the slots stay whole).
* A request is prepared in one of ``slots`` execution slots.  A slot owns a
  CUDA stream, device buffers for the camera and palette, and render
  workspaces sized for the largest (scene, resolution) bucket it serves.
  Each bucket's preparation -- fused preprocess with palette-colour records
  (gsb_render_preprocess), capacity-sized tile sort with no host read-back
  (gsb_splat_sort_capacity) and the copy of the sort's overflow words to
  pinned host memory -- is captured once per slot as a CUDA graph; a request
  copies its camera and palette into the slot's buffers and replays it on
  the slot's stream, so the preparations of different requests overlap.
* Prepared requests are composited together: a batch packs their images
  into a job table (gsb_draw_batch_pack) and one persistent kernel
  (gsb_draw_batch) claims (image, tile) items from all of them until every
  tile is done, so tiles of large and small images, of different scenes
  and resolutions, share the SMs.  The table copy, the kernel and the fetch
  and copy of the device status bits are one captured CUDA graph per batch
  table, replayed on the table's own stream after it waits for the members'
  preparations.  Up to ``batches`` batches are in flight and overlap on the
  device; requests that arrive meanwhile are prepared at once and join the
  next batch.
* A render whose patch count or depth key exceeded the bucket's capacity
  (status words) is re-run after the bucket's capacity grows (its graphs are
  recaptured); its latency includes the re-run.  A bounded device wait that
  ran out (status bits) raises GsplatError(GSB_ERR_DEVICE_TIMEOUT).

The palette-edit image equals the reference's bake-and-render path
(gsplat/gsmodel.py:488-509 bakes palette colours into RGB SH coefficients,
14-26 renders them with sh2Color / splat_color): sum_k P_k w_k(dir) is the
same linear map, summed in a different FP32 order.
"""
import collections
import ctypes as C
import math
import time

import numpy as np
import torch
from cuda.bindings import runtime as _rt

from gsplatcu import _lib

_F32 = torch.float32
MAX_DEPTH_KEY = (1 << 17) - 1  # depth keys uint32(depth*1000): scenes within 131 m


def _nbytes(*ts):
    return sum(int(t.numel()) * t.element_size() for t in ts if t is not None)


class Scene:
    """A finetuned scene: geometry (FP32) and palette weights, full SH order 3
    (``shs`` [N,16K]) or low-rank (``dc`` [N,K], ``A`` [N,P,r], ``B`` [N,r,Q]),
    FP32 or BF16, all on the device."""

    def __init__(self, scene_id, pws, rots, scales, alphas, shs=None, dc=None, A=None, B=None):
        self.id = scene_id
        self.pws, self.rots, self.scales = pws.contiguous(), rots.contiguous(), scales.contiguous()
        self.alphas = alphas.reshape(-1).contiguous()
        self.n = int(pws.shape[0])
        if shs is not None:
            self.mode, self.shs = _lib.WEIGHTS_FULL, shs.contiguous()
            self.K = int(shs.shape[1]) // 16
            self.P = self.Q = self.rank = 0
            self.w0, self.A, self.B = self.shs, None, None
        else:
            self.mode = _lib.WEIGHTS_LOWRANK
            self.w0, self.A, self.B = dc.contiguous(), A.contiguous(), B.contiguous()
            self.K = int(dc.shape[1])
            if A.dim() == 2:
                self.P, self.rank, self.Q = int(A.shape[1]), 1, int(B.shape[1])
            else:
                self.P, self.rank, self.Q = int(A.shape[1]), int(A.shape[2]), int(B.shape[2])
        self.dtype = self.w0.dtype
        self.bytes = _nbytes(self.pws, self.rots, self.scales, self.alphas, self.w0, self.A, self.B)

    def params(self, palette):
        return _lib.PaletteParams(self.mode, _lib.DTYPE_BF16 if self.dtype == torch.bfloat16
                                  else _lib.DTYPE_F32, self.K, self.P, self.Q, self.rank,
                                  self.w0.data_ptr(),
                                  self.A.data_ptr() if self.A is not None else None,
                                  self.B.data_ptr() if self.B is not None else None,
                                  palette.data_ptr())


class Request:
    """A palette-edit render: scene id, camera pose (Rcw [3,3], tcw [3]),
    intrinsics and resolution, and the [K,3] palette to render with."""
    __slots__ = ("scene_id", "Rcw", "tcw", "twc", "fx", "fy", "cx", "cy", "width", "height",
                 "palette", "arrival", "start", "done", "image", "reruns", "slot", "tag")

    def __init__(self, scene_id, Rcw, tcw, fx, fy, cx, cy, width, height, palette, tag=None):
        self.scene_id = scene_id
        R = np.asarray(Rcw, np.float32).reshape(3, 3)
        t = np.asarray(tcw, np.float32).reshape(3)
        self.Rcw = torch.from_numpy(R.copy()).pin_memory()
        self.tcw = torch.from_numpy(t.copy()).pin_memory()
        twc = (-np.linalg.inv(R.astype(np.float64)) @ t.astype(np.float64)).astype(np.float32)
        self.twc = torch.from_numpy(twc).pin_memory()
        self.fx, self.fy, self.cx, self.cy = float(fx), float(fy), float(cx), float(cy)
        self.width, self.height = int(width), int(height)
        self.palette = torch.from_numpy(np.asarray(palette, np.float32).copy()).pin_memory()
        self.arrival = self.start = self.done = None
        self.image = None
        self.reruns = 0
        self.slot = None
        self.tag = tag

    @property
    def bucket(self):
        return (self.scene_id, self.width, self.height, self.fx, self.fy, self.cx, self.cy)


class _Bucket:
    """Render sizes of one (scene, resolution, intrinsics)."""

    def __init__(self, scene, W, H, capacity):
        self.scene, self.W, self.H = scene, W, H
        self.tiles = ((W + 15) // 16) * ((H + 15) // 16)
        self.capacity = int(capacity)
        L = _lib.lib()
        self.state_bytes = int(L.gsb_splat_state_bytes(scene.n, 3, H, W))
        self.sort_bytes = int(L.gsb_splat_sort_capacity_bytes(scene.n, H, W, self.capacity,
                                                              MAX_DEPTH_KEY))
        self.pixels = W * H


class _Slot:
    """One execution slot: stream, input buffers, workspaces, graphs.
    `alloc(shape, dtype)` allocates its device buffers (torch.empty on the
    slot's device unless the server was given another allocator)."""

    def __init__(self, device, K_max, alloc=None):
        self.device = device
        self.alloc = alloc or (lambda shape, dtype: torch.empty(shape, dtype=dtype, device=device))
        self.stream = torch.cuda.Stream(device)
        self.Rcw = torch.zeros((3, 3), dtype=_F32, device=device)
        self.tcw = torch.zeros((3,), dtype=_F32, device=device)
        self.twc = torch.zeros((3,), dtype=_F32, device=device)
        self.palette = torch.zeros((K_max, 3), dtype=_F32, device=device)
        # overflow bits and patch count of the capacity sort
        self.status = torch.zeros((4,), dtype=torch.int32, device=device)
        self.status_host = torch.zeros((4,), dtype=torch.int32).pin_memory()
        self.sizes = dict(state=0, sort=0, gsid=0, tiles=0, pixels=0)
        self.buf = {}
        self.graphs = {}
        self.req = None
        self.event = None  # the preparation's completion
        self.batch = None  # the batch compositing the request, once launched

    def bytes(self):
        s = self.sizes
        return s["state"] + s["sort"] + 4 * s["gsid"] + 8 * s["tiles"] + 20 * s["pixels"]

    def ensure(self, b):
        """Grow the workspaces to fit bucket b (drops graphs that captured
        the old buffers)."""
        need = dict(state=b.state_bytes, sort=b.sort_bytes, gsid=b.capacity, tiles=b.tiles,
                    pixels=b.pixels)
        if all(need[k] <= self.sizes[k] for k in need):
            return False
        s = {k: max(self.sizes[k], need[k]) for k in need}
        a = self.alloc
        u8 = lambda nb: a((max(256, nb),), torch.uint8)
        # all new buffers first: if one allocation fails the slot keeps its
        # old buffers, sizes and graphs
        buf = dict(state=u8(s["state"]), sort=u8(s["sort"]),
                   gsid=a((max(1, s["gsid"]),), torch.int32),
                   ranges=a((s["tiles"], 2), torch.int32),
                   image=a((3 * s["pixels"],), _F32),
                   contrib=a((s["pixels"],), torch.int32),
                   final_tau=a((s["pixels"],), _F32))
        self.sizes, self.buf = s, buf
        self.graphs.clear()
        return True

    def image_view(self, W, H):
        return self.buf["image"][:3 * W * H].view(3, H, W)

    def launch_prep(self, b, fx, fy, cx, cy):
        """Enqueue one request's preparation for bucket b on the current
        stream (capturable): preprocess, capacity sort, status words."""
        sc, W, H = b.scene, b.W, b.H
        cam = _lib.Camera(self.Rcw.data_ptr(), self.tcw.data_ptr(), self.twc.data_ptr(), fx, fy,
                          cx, cy, W, H)
        params = sc.params(self.palette)
        st = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        bf, n = self.buf, sc.n
        _lib.call("serve", "gsb_render_preprocess", n, C.byref(cam), _lib.ptr(sc.pws),
                  _lib.ptr(sc.rots), _lib.ptr(sc.scales), _lib.ptr(sc.alphas), C.byref(params),
                  _lib.ptr(bf["state"]), None, st)
        _lib.call("serve", "gsb_splat_sort_capacity", n, H, W, b.capacity, MAX_DEPTH_KEY,
                  _lib.ptr(bf["state"]), _lib.ptr(bf["sort"]), _lib.ptr(bf["gsid"]),
                  _lib.ptr(bf["ranges"]), _lib.ptr(self.status), st)
        # overflow status -> pinned host words, read once the request's batch is
        # done (the device status bits are fetched by the batch, after its
        # members' preparations and the compositing)
        err, = _rt.cudaMemcpyAsync(self.status_host.data_ptr(), self.status.data_ptr(), 12,
                                   _rt.cudaMemcpyKind.cudaMemcpyDeviceToHost, st.value)
        if err != _rt.cudaError_t.cudaSuccess:
            raise _lib.GsplatError(f"serve: status copy failed ({err})")

    def job(self, b):
        """The slot's image as an entry of a batched compositing launch."""
        bf = self.buf
        return _lib.DrawJob(bf["state"].data_ptr(), b.scene.n, b.H, b.W, 3,
                            bf["ranges"].data_ptr(), bf["gsid"].data_ptr(), 1.0,
                            bf["image"].data_ptr(), bf["contrib"].data_ptr(),
                            bf["final_tau"].data_ptr())


class _Batch:
    """One batch table: pinned host table, device table, status words and
    the captured graph (table copy, persistent compositing, status copy)."""

    def __init__(self, device, max_jobs):
        L = _lib.lib()
        self.device = device
        self.max_jobs = max_jobs
        self.nbytes = int(L.gsb_draw_batch_bytes(max_jobs))
        self.host = torch.zeros((self.nbytes,), dtype=torch.uint8).pin_memory()
        self.dev = torch.zeros((self.nbytes,), dtype=torch.uint8, device=device)
        self.status = torch.zeros((1,), dtype=torch.int32, device=device)
        self.status_host = torch.zeros((1,), dtype=torch.int32).pin_memory()
        self.stream = torch.cuda.Stream(device)  # batches overlap on the device
        self.graph = None
        self.event = None
        self.slots = []

    def pack(self, jobs):
        arr = (_lib.DrawJob * max(1, len(jobs)))(*jobs)
        _lib.call("serve", "gsb_draw_batch_pack", arr, len(jobs), C.c_void_p(self.host.data_ptr()),
                  self.nbytes)

    def enqueue(self):
        """Table copy, batched compositing, status fetch and copy on the
        current stream (capturable: a replay copies the host table's
        contents at that time)."""
        st = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        err, = _rt.cudaMemcpyAsync(self.dev.data_ptr(), self.host.data_ptr(), self.nbytes,
                                   _rt.cudaMemcpyKind.cudaMemcpyHostToDevice, st.value)
        if err != _rt.cudaError_t.cudaSuccess:
            raise _lib.GsplatError(f"serve: table copy failed ({err})")
        _lib.call("serve", "gsb_draw_batch", _lib.ptr(self.dev), 3, st)
        # the library's device status bits (a bounded wait of the members'
        # preprocess ran out), fetched into a word cleared first
        self.status.zero_()
        _lib.call("serve", "gsb_device_status_fetch", _lib.ptr(self.status), st)
        err, = _rt.cudaMemcpyAsync(self.status_host.data_ptr(), self.status.data_ptr(), 4,
                                   _rt.cudaMemcpyKind.cudaMemcpyDeviceToHost, st.value)
        if err != _rt.cudaError_t.cudaSuccess:
            raise _lib.GsplatError(f"serve: status copy failed ({err})")


class PaletteServer:
    """Resident scenes + slots + request queue (see the module docstring).

    hbm_budget: bytes the server may hold (scenes + slot workspaces).
    slots: concurrent renders.  use_graphs: replay captured CUDA graphs
    (False: launch the same kernels directly, for comparison).  keep_images:
    copy each finished image out of its slot (off for throughput runs)."""

    def __init__(self, hbm_budget, slots=8, device="cuda", use_graphs=True, K_max=8,
                 capacity_margin=1.5, keep_images=True, alloc=None, batches=3):
        self.device = torch.device(device)
        self.last_admit_error = None
        self.keep_images = keep_images
        self.budget = int(hbm_budget)
        self.use_graphs = use_graphs
        self.margin = capacity_margin
        self.scenes = collections.OrderedDict()
        self.buckets = {}
        self.slots = [_Slot(self.device, K_max, alloc) for _ in range(slots)]
        self.batches = [_Batch(self.device, slots) for _ in range(batches)]
        self.queue = collections.deque()
        self.done = []
        self.graph_captures = 0
        self.batch_sizes = []

    # ------------------------------------------------------------ memory
    def resident_bytes(self):
        return sum(s.bytes for s in self.scenes.values()) + sum(s.bytes() for s in self.slots)

    def _slot_growth(self, b):
        grow = 0
        for sl in self.slots:
            s = sl.sizes
            need = dict(state=b.state_bytes, sort=b.sort_bytes, gsid=b.capacity, tiles=b.tiles,
                        pixels=b.pixels)
            new = {k: max(s[k], need[k]) for k in s}
            grow += (new["state"] + new["sort"] + 4 * new["gsid"] + 8 * new["tiles"] +
                     20 * new["pixels"]) - sl.bytes()
        return grow

    def admit_scene(self, scene, resolutions, probe_cameras):
        """Admit `scene` if its parameters plus the workspace growth for its
        render buckets fit the budget.  `resolutions`: [(W, H, fx, fy, cx,
        cy)] it will be rendered at; `probe_cameras`: poses [(Rcw, tcw)] used
        to size each bucket's patch capacity (the largest count seen, times
        the margin).  Returns False (nothing kept) when it does not fit."""
        if scene.id in self.scenes:
            raise ValueError(f"scene {scene.id!r} already resident")
        buckets = {}
        for (W, H, fx, fy, cx, cy) in resolutions:
            m = max(self._count_patches(scene, R, t, fx, fy, cx, cy, W, H)
                    for R, t in probe_cameras)
            cap = max(1024, int(math.ceil(m * self.margin)))
            buckets[(scene.id, W, H, fx, fy, cx, cy)] = _Bucket(scene, W, H, cap)
        growth = 0
        saved = [dict(sl.sizes) for sl in self.slots]
        for b in buckets.values():
            growth += self._slot_growth(b)
            for sl in self.slots:  # account cumulatively
                for k, v in dict(state=b.state_bytes, sort=b.sort_bytes, gsid=b.capacity,
                                 tiles=b.tiles, pixels=b.pixels).items():
                    sl.sizes[k] = max(sl.sizes[k], v)
        for sl, s in zip(self.slots, saved):
            sl.sizes = s
        if self.resident_bytes() + scene.bytes + growth > self.budget:
            self.last_admit_error = "over the HBM budget"
            return False
        try:
            for b in buckets.values():
                for sl in self.slots:
                    sl.ensure(b)
        except torch.OutOfMemoryError as e:
            # a workspace could not be allocated: the scene is not admitted; slots
            # that already grew keep their (larger, valid) buffers
            self.last_admit_error = f"workspace allocation failed: {e}"
            return False
        self.scenes[scene.id] = scene
        self.buckets.update(buckets)
        self.last_admit_error = None
        return True

    def evict_scene(self, scene_id):
        """Drop a scene (waits for its in-flight renders).  Slot workspaces
        keep their size until the server is rebuilt."""
        if any(sl.req is not None and sl.req.scene_id == scene_id for sl in self.slots):
            self.drain()
        self.scenes.pop(scene_id)
        for key in [k for k in self.buckets if k[0] == scene_id]:
            del self.buckets[key]
        for sl in self.slots:
            for key in [k for k in sl.graphs if k[0] == scene_id]:
                del sl.graphs[key]

    def _count_patches(self, scene, Rcw, tcw, fx, fy, cx, cy, W, H):
        """Exact patch count of one view (host read-back; admission only)."""
        dev = self.device
        Rd = torch.as_tensor(np.asarray(Rcw, np.float32), device=dev).reshape(3, 3).contiguous()
        td = torch.as_tensor(np.asarray(tcw, np.float32), device=dev).reshape(3).contiguous()
        cd = (-torch.linalg.inv(Rd.double()) @ td.double()).float().contiguous()
        cam = _lib.Camera(Rd.data_ptr(), td.data_ptr(), cd.data_ptr(), fx, fy, cx, cy, W, H)
        pal = torch.zeros((scene.K, 3), dtype=_F32, device=dev)
        params = scene.params(pal)
        L = _lib.lib()
        state = torch.empty((int(L.gsb_splat_state_bytes(scene.n, 3, H, W)),), dtype=torch.uint8,
                            device=dev)
        st = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        _lib.call("serve", "gsb_render_preprocess", scene.n, C.byref(cam), _lib.ptr(scene.pws),
                  _lib.ptr(scene.rots), _lib.ptr(scene.scales), _lib.ptr(scene.alphas),
                  C.byref(params), _lib.ptr(state), None, st)
        plan = _lib.SplatPlan()
        _lib.call("serve", "gsb_splat_counts", scene.n, H, W, _lib.ptr(state), C.byref(plan), st)
        if plan.max_depth_key > MAX_DEPTH_KEY:
            raise ValueError(f"scene {scene.id!r}: depth beyond {MAX_DEPTH_KEY / 1000:.0f} m")
        return int(plan.patches)

    # ----------------------------------------------------------- execute
    def _graph(self, sl, b, req):
        key = req.bucket
        g = sl.graphs.get(key)
        if g is None:
            with torch.cuda.stream(sl.stream):
                sl.launch_prep(b, req.fx, req.fy, req.cx, req.cy)  # warm (function attributes)
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=sl.stream):
                sl.launch_prep(b, req.fx, req.fy, req.cx, req.cy)
            sl.graphs[key] = g
            self.graph_captures += 1
        return g

    def _batch_graph(self, bt):
        """The batch table's graph, captured on first use (with an empty table:
        call it before packing the batch)."""
        if bt.graph is None:
            bt.pack([])
            with torch.cuda.stream(bt.stream):
                bt.enqueue()  # warm (function attributes, status-word addresses)
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=bt.stream):
                bt.enqueue()
            bt.graph = g
            self.graph_captures += 1
        return bt.graph

    def prepare(self, requests):
        """Capture every (bucket, slot) preparation graph these requests need
        and the batch graphs, before a timed run (a service does this at
        start-up)."""
        if not self.use_graphs:
            return
        seen = set()
        for r in requests:
            if r.bucket in seen:
                continue
            seen.add(r.bucket)
            b = self.buckets[r.bucket]
            for sl in self.slots:
                self._graph(sl, b, r)
        for bt in self.batches:
            self._batch_graph(bt)
        torch.cuda.synchronize(self.device)

    def _start(self, sl, req):
        b = self.buckets.get(req.bucket)
        if b is None:
            raise KeyError(f"no render bucket for scene {req.scene_id!r} at "
                           f"{req.width}x{req.height}; admit the scene with this resolution")
        sl.ensure(b)  # (workspaces grew: graphs are recaptured below)
        K = b.scene.K
        g = self._graph(sl, b, req) if self.use_graphs else None
        with torch.cuda.stream(sl.stream):
            sl.Rcw.copy_(req.Rcw, non_blocking=True)
            sl.tcw.copy_(req.tcw, non_blocking=True)
            sl.twc.copy_(req.twc, non_blocking=True)
            sl.palette[:K].copy_(req.palette, non_blocking=True)
            if g is not None:
                g.replay()
            else:
                sl.launch_prep(b, req.fx, req.fy, req.cx, req.cy)
            sl.event = torch.cuda.Event()
            sl.event.record(sl.stream)
        if req.start is None:
            req.start = time.perf_counter()
        req.slot = self.slots.index(sl)
        sl.req = req
        sl.batch = None

    def _launch_batch(self):
        """Composite every prepared request not yet in a batch in one
        persistent kernel, if a batch table is free."""
        ready = [sl for sl in self.slots if sl.req is not None and sl.batch is None]
        if not ready:
            return False
        bt = next((b for b in self.batches if not b.slots), None)
        if bt is None:
            return False
        ready = ready[:bt.max_jobs]
        g = self._batch_graph(bt) if self.use_graphs else None  # (captured before packing)
        bt.pack([sl.job(self.buckets[sl.req.bucket]) for sl in ready])
        with torch.cuda.stream(bt.stream):
            for sl in ready:
                bt.stream.wait_event(sl.event)
            if g is not None:
                g.replay()
            else:
                bt.enqueue()
            bt.event = torch.cuda.Event()
            bt.event.record(bt.stream)
        bt.slots = ready
        for sl in ready:
            sl.batch = bt
        self.batch_sizes.append(len(ready))
        return True

    def _retire_batch(self, bt):
        members, bt.slots = bt.slots, []
        bits = int(bt.status_host[0])
        if bits:
            # a bounded wait of a member's preprocess or of the compositing ran
            # out: the batch's images are incomplete.  Clear the bits, report.
            for sl in members:
                sl.req, sl.batch = None, None
            cleared = C.c_uint32(0)
            _lib.call("serve", "gsb_device_status", C.byref(cleared), 1,
                      C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream))
            bt.status_host[0] = 0
            raise _lib.GsplatError(f"serve: a bounded device wait ran out in a batch of "
                                   f"{len(members)} request(s) (status bits {bits:#x})",
                                   _lib.GSB_ERR_DEVICE_TIMEOUT)
        for sl in members:
            sl.batch = None
            self._retire(sl)

    def _retire(self, sl):
        req, b = sl.req, self.buckets[sl.req.bucket]
        sl.req = None
        status = int(sl.status_host[0])
        if status & (_lib.STATUS_PATCH_OVERFLOW | _lib.STATUS_DEPTH_KEY_OVERFLOW):
            if status & _lib.STATUS_DEPTH_KEY_OVERFLOW:
                raise RuntimeError(f"scene {req.scene_id!r}: depth key above {MAX_DEPTH_KEY}")
            # grow this bucket's capacity and render again
            nb = _Bucket(b.scene, b.W, b.H, b.capacity * 2)
            self.buckets[req.bucket] = nb
            for s2 in self.slots:
                s2.graphs.pop(req.bucket, None)
            req.reruns += 1
            self.queue.appendleft(req)
            return None
        req.done = time.perf_counter()
        if self.keep_images:
            req.image = sl.image_view(req.width, req.height).clone()
        self.done.append(req)
        return req

    def poll(self):
        """Retire finished batches, prepare queued requests on free slots and
        launch a batch of the prepared ones.  Returns the number of busy
        slots."""
        for bt in self.batches:
            if bt.slots and bt.event.query():
                self._retire_batch(bt)
        for sl in self.slots:
            if sl.req is None and self.queue:
                self._start(sl, self.queue.popleft())
        self._launch_batch()
        return sum(sl.req is not None for sl in self.slots)

    def submit(self, req, now=None):
        req.arrival = time.perf_counter() if now is None else now
        self.queue.append(req)

    def drain(self):
        while self.queue or any(sl.req is not None for sl in self.slots):
            self.poll()

    def render_alone(self, req):
        """Render one request by itself (nothing else in flight) and return
        the image."""
        self.drain()
        self.submit(req)
        self.drain()
        return req.image

    def run_open_loop(self, requests, rate, seed=0):
        """Serve `requests` arriving as a Poisson stream of `rate` per second
        (open loop: arrivals do not wait for completions).  Returns latency
        statistics in ms and the frames per second served."""
        rng = np.random.default_rng(seed)
        gaps = rng.exponential(1.0 / rate, size=len(requests))
        t0 = time.perf_counter() + 0.01
        arrivals = t0 + np.cumsum(gaps)
        i = 0
        self.done = []
        while i < len(requests) or self.queue or any(sl.req is not None for sl in self.slots):
            now = time.perf_counter()
            while i < len(requests) and arrivals[i] <= now:
                self.submit(requests[i], now=float(arrivals[i]))
                i += 1
            self.poll()
        t_end = max(r.done for r in self.done)
        lat = np.array([(r.done - r.arrival) * 1000.0 for r in self.done])
        return dict(requests=len(self.done), p50_ms=float(np.percentile(lat, 50)),
                    p99_ms=float(np.percentile(lat, 99)), mean_ms=float(lat.mean()),
                    max_ms=float(lat.max()), frames_per_s=len(self.done) / (t_end - t0),
                    offered_rate=rate, reruns=int(sum(r.reruns for r in self.done)))

    def run_closed_loop(self, requests):
        """Saturation: all `requests` queued at once, served as fast as the
        slots and batches allow.  Returns frames per second and the mean
        batch size."""
        self.done = []
        n0 = len(self.batch_sizes)
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        for r in requests:
            self.submit(r, now=t0)
        self.drain()
        t1 = time.perf_counter()
        sizes = self.batch_sizes[n0:]
        return dict(requests=len(self.done), seconds=t1 - t0,
                    frames_per_s=len(self.done) / (t1 - t0),
                    mean_batch=float(np.mean(sizes)) if sizes else 0.0,
                    reruns=int(sum(r.reruns for r in self.done)))
