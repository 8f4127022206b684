"""GPU tests of the fused render path (palette_b200.render.render_palette):
the per-Gaussian state it packs and the image it renders against the
reference operator sequence run through gsplatcu, and its full adjoint
(means, rotations, scales, opacities, weight parameters, final-transmittance
term) against the oracle's FP64 chain rule, which is itself pinned to finite
differences on the CPU (test_oracle_chain.py).  Tolerances: images 1e-5 abs
(FP32 storage); gradients 1e-4 relative, norm-wise per gradient tensor."""
import ctypes as C

import numpy as np
import pytest
import torch

import gsplatcu as gsc
from gsplatcu import _lib
from oracle import oracle as orc
from palette_b200.render import camera_struct, render_palette
from palette_b200.scene import look_at, synthetic_scene, to_torch
from helpers import forward_ops, max_abs, np_of, rel_err

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
GRAD_REL = 1e-4
GEOM = ("pws", "rots", "scales", "alphas")

VARIANTS = [  # (mode, rank, param dtype)
    ("full", 0, torch.float32),
    ("full", 0, torch.bfloat16),
    ("lowrank", 1, torch.float32),
    ("lowrank", 3, torch.float32),
    ("lowrank", 3, torch.bfloat16),
]


def _setup(mode, rank, dtype, n=2000, W=64, H=64, eye=(0.0, -8.0, 0.0), seed=11):
    sc = synthetic_scene(n, seed=seed, mode=mode, rank=max(rank, 1))
    st = to_torch(sc, "cuda", dtype)
    if mode == "lowrank" and rank == 1:  # the reference's 2-D factor shapes
        st["A"], st["B"] = st["A"][:, :, 0].contiguous(), st["B"][:, 0, :].contiguous()
    cam = look_at(eye, width=W, height=H, device="cuda")
    return sc, st, cam


def _render(st, cam, mode, requires_grad=False, grad_names=None):
    names = list(GEOM) + (["shs"] if mode == "full" else ["dc", "A", "B"])
    grad_names = names if grad_names is None else grad_names
    leaf = {k: st[k].detach().clone().requires_grad_(requires_grad and k in grad_names)
            for k in names}
    if mode == "full":
        out = render_palette(leaf["pws"], leaf["rots"], leaf["scales"], leaf["alphas"], cam,
                             shs=leaf["shs"])
    else:
        out = render_palette(leaf["pws"], leaf["rots"], leaf["scales"], leaf["alphas"], cam,
                             dc=leaf["dc"], A=leaf["A"], B=leaf["B"])
    return out, leaf


def _state_sections(n, K, H, W):
    al = lambda x: (x + 255) & ~255
    nb = (n + 255) // 256
    tiles = ((W + 15) // 16) * ((H + 15) // 16)
    o = [0]
    for size in (n * 8, n * 4, n * 4, nb * 4, 64, tiles * 4):
        o.append(o[-1] + al(size))
    del o[5]  # (the tile launch order, written by the compositing launches)
    return o  # rects, dkeys, counts, block sums, stats, records


def _packed_states(st, cam, mode, rank):
    """(compat state packed by gsb_splat_pack from the operator outputs,
    fused state from gsb_render_preprocess) as numpy byte arrays."""
    n, K, H, W = st["pws"].shape[0], 5, int(cam.height), int(cam.width)
    L = _lib.lib()
    nbytes = int(L.gsb_splat_state_bytes(n, K, H, W))
    r = forward_ops(gsc, st, cam, mode)
    us, pcs, depths = gsc.project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
    cov3, = gsc.computeCov3D(st["rots"], st["scales"], depths, False)
    cov2, = gsc.computeCov2D(cov3, pcs, cam.Rcw, depths, cam.fx, cam.fy, W, H, False)
    cinv, areas = gsc.inverseCov2D(cov2, depths, False)
    s = _lib.stream_of(us)
    s1 = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    _lib.call("t", "gsb_splat_pack", n, H, W, K, _lib.ptr(us), _lib.ptr(cinv),
              _lib.ptr(st["alphas"]), _lib.ptr(r["weights"]), _lib.DTYPE_F32, _lib.ptr(depths),
              _lib.ptr(areas), _lib.ptr(s1), s)
    s2 = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    camst, keep = camera_struct(cam)
    full = mode == "full"
    w0 = st["shs"] if full else st["dc"]
    A, B = (None, None) if full else (st["A"], st["B"])
    P, Q = (0, 0) if full else (5, 15)
    params = _lib.PaletteParams(_lib.WEIGHTS_FULL if full else _lib.WEIGHTS_LOWRANK,
                                _lib.DTYPE_BF16 if w0.dtype == torch.bfloat16 else _lib.DTYPE_F32,
                                K, P, Q, rank, w0.data_ptr(), A.data_ptr() if A is not None else None,
                                B.data_ptr() if B is not None else None)
    d2 = torch.empty(n, device="cuda")
    _lib.call("t", "gsb_render_preprocess", n, C.byref(camst), _lib.ptr(st["pws"]),
              _lib.ptr(st["rots"]), _lib.ptr(st["scales"]), _lib.ptr(st["alphas"]),
              C.byref(params), _lib.ptr(s2), _lib.ptr(d2), s)
    torch.cuda.synchronize()
    return s1.cpu().numpy(), s2.cpu().numpy(), np_of(depths), np_of(d2)


@pytest.mark.parametrize("mode,rank,dtype", VARIANTS)
def test_fused_preprocess_state_matches_operator_sequence(cuda_ok, mode, rank, dtype):
    """Per-Gaussian counts, depth keys, rectangles, block sums, depths and
    records: the fused kernel against gsb_splat_pack on the operators'
    outputs.  Integer fields and depths bit-exact; record floats within
    1e-5 of each field's magnitude (the fused kernel keeps its intermediates
    in registers, where the compiler may pair multiplies and adds into FMAs
    differently than across separate kernels)."""
    sc, st, cam = _setup(mode, rank, dtype, n=20000, W=200, H=120, eye=(5.0, -5.0, 2.0))
    n, K, H, W = 20000, 5, 120, 200
    a1, a2, dep1, dep2 = _packed_states(st, cam, mode, max(rank, 1))
    o = _state_sections(n, K, H, W)
    cnt1, cnt2 = (a[o[2]:o[2] + 4 * n].view(np.uint32) for a in (a1, a2))
    assert np.array_equal(cnt1, cnt2)
    live = cnt1 > 0
    assert live.sum() > 1000
    dk1, dk2 = (a[o[1]:o[1] + 4 * n].view(np.uint32) for a in (a1, a2))
    assert np.array_equal(dk1, dk2)
    rc1, rc2 = (a[o[0]:o[0] + 8 * n].view(np.uint32).reshape(n, 2)[live] for a in (a1, a2))
    assert np.array_equal(rc1, rc2)
    nb = (n + 255) // 256
    assert np.array_equal(a1[o[3]:o[3] + 4 * nb], a2[o[3]:o[3] + 4 * nb])
    assert np.array_equal(a1[o[4]:o[4] + 16], a2[o[4]:o[4] + 16])
    assert np.array_equal(dep1, dep2)
    V = (11 + K + 3) // 4
    r1, r2 = (a[o[5]:o[5] + n * V * 16].view(np.float32).reshape(n, V * 4)[live] for a in (a1, a2))
    names = ["ux", "uy", "qa", "qb", "qc", "c2", "alpha", "w0", "hx", "hy", "ia", "ic"] + \
            [f"w{k}" for k in range(1, K)]
    report = {}
    fin = np.isfinite(r1) & np.isfinite(r2)
    assert np.array_equal(np.isfinite(r1), np.isfinite(r2))
    for j, nm in enumerate(names):
        d = (r1[:, j] != r2[:, j]) & fin[:, j]
        if d.any():
            scale = max(np.abs(r1[fin[:, j], j]).max(), 1e-30)
            report[nm] = (int(d.sum()), float(np.abs(r1[d, j] - r2[d, j]).max() / scale))
    print(f"record fields differing ({mode}, rank {rank}, {dtype}):", report)
    for nm in ("ux", "uy", "alpha"):
        assert nm not in report, report
    assert all(v[1] < 1e-5 for v in report.values()), report


@pytest.mark.parametrize("mode,rank,dtype", VARIANTS)
def test_fused_forward_matches_operator_sequence(cuda_ok, mode, rank, dtype):
    sc, st, cam = _setup(mode, rank, dtype, n=20000, W=200, H=120, eye=(5.0, -5.0, 2.0))
    ref = forward_ops(gsc, st, cam, mode)
    (layer, ft, depths), _ = _render(st, cam, mode)
    assert torch.equal(depths, ref["depths"].reshape(-1))
    assert max_abs(layer, ref["layer"]) < IMG_TOL
    assert max_abs(ft, ref["final_tau"]) < IMG_TOL


def test_fused_forward_edge_cases(cuda_ok):
    # nothing in front of the camera, and an empty scene
    sc, st, cam = _setup("full", 0, torch.float32, n=500)
    st["pws"] = st["pws"] - torch.tensor([0.0, 100.0, 0.0], device="cuda")
    (layer, ft, depths), _ = _render(st, cam, "full")
    assert torch.count_nonzero(layer) == 0 and torch.count_nonzero(ft) == 0
    assert torch.all(depths == -1)
    st0 = {k: (v[:0].contiguous() if isinstance(v, torch.Tensor) else v) for k, v in st.items()}
    (layer, ft, depths), _ = _render(st0, cam, "full")
    assert layer.shape == (5, 64, 64) and torch.count_nonzero(layer) == 0 and depths.numel() == 0


def _fp64_chain(st, cam, mode, lists, dout, dT):
    f = lambda t: t.detach().double().cpu().numpy()
    lr = None if mode == "full" else (f(st["dc"]), f(st["A"]), f(st["B"]))
    return orc.render_weights_backward(f(st["pws"]), f(st["rots"]), f(st["scales"]),
                                       f(st["alphas"]), cam, f(cam.twc), 5,
                                       shs=f(st["shs"]) if mode == "full" else None,
                                       lowrank=lr, lists=lists, dout=dout, dT=dT)


@pytest.mark.parametrize("mode,rank,dtype", VARIANTS)
def test_fused_backward_matches_fp64_chain(cuda_ok, mode, rank, dtype):
    """2000 Gaussians at 64x64 (the finite-difference subset size): every
    gradient against the FP64 chain rule on the same (for BF16: rounded)
    parameter values and the same tile lists."""
    sc, st, cam = _setup(mode, rank, dtype, seed=12 + rank)
    (layer, ft, depths), leaf = _render(st, cam, mode, requires_grad=True)
    gen = torch.Generator("cuda").manual_seed(5)
    dout = torch.randn(layer.shape, device="cuda", generator=gen)
    dT = torch.randn(ft.shape, device="cuda", generator=gen)
    ((layer * dout).sum() + (ft * dT).sum()).backward()
    ref = forward_ops(gsc, st, cam, mode)
    lists = (np_of(ref["ranges"]), np_of(ref["gsid"]))
    r = _fp64_chain(st, cam, mode, lists, np_of(dout), np_of(dT))
    assert np.abs(np_of(layer) - r["layer"]).max() < IMG_TOL
    pairs = dict(pws="dpws", rots="drots", scales="dscales", alphas="dalphas")
    pairs.update(shs="dshs") if mode == "full" else pairs.update(dc="ddc", A="dA", B="dB")
    # BF16 parameters get BF16 gradients: rounding to 8 mantissa bits bounds
    # the norm-wise error by about 2^-9
    tol = GRAD_REL if dtype == torch.float32 else 4e-3
    for name, gname in pairs.items():
        g = leaf[name].grad
        assert g is not None and g.shape == leaf[name].shape and g.dtype == leaf[name].dtype
        e = rel_err(g.float().reshape(len(g), -1), r[gname].reshape(len(g), -1))
        assert e < tol, (name, e)


@pytest.mark.parametrize("mode,rank", [("full", 0), ("lowrank", 3)])
def test_fused_weights_only_backward(cuda_ok, mode, rank):
    """With no geometry input requiring a gradient the backward computes the
    weight gradients alone (the reference backward's scope); they match the
    full adjoint's."""
    sc, st, cam = _setup(mode, rank, torch.float32, seed=60 + rank)
    wn = ["shs"] if mode == "full" else ["dc", "A", "B"]
    g = torch.randn((5, 64, 64), device="cuda", generator=torch.Generator("cuda").manual_seed(2))
    (l1, _, _), full = _render(st, cam, mode, requires_grad=True)
    (l1 * g).sum().backward()
    (l2, _, _), wo = _render(st, cam, mode, requires_grad=True, grad_names=wn)
    assert torch.equal(l1, l2)
    (l2 * g).sum().backward()
    for k in GEOM:
        assert wo[k].grad is None
    for k in wn:
        assert rel_err(wo[k].grad, full[k].grad) < 1e-6, k


@pytest.mark.parametrize("rank", [1, 3])
def test_fused_weight_gradients_match_reference_backward(cuda_ok, rank):
    """d dc, dA, dB of the fused path equal the reference backward's formula
    (gsplat/gsmodel.py:182-200: splat_weight_B, dc' = dW * dweight_ddc,
    sh2Weight_fast_B) evaluated with the gsplatcu operators, and those of
    splat_palette_weights, up to FP32 summation order."""
    from palette_b200.weights import splat_palette_weights
    sc, st, cam = _setup("lowrank", rank, torch.float32, seed=40 + rank)
    (layer, ft, _), leaf = _render(st, cam, "lowrank", requires_grad=True,
                                   grad_names=["dc", "A", "B"])
    g = torch.randn(layer.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(9))
    (layer * g).sum().backward()
    # the reference's backward, written out with the operators
    H, W = cam.height, cam.width
    us, pcs, d = gsc.project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
    c3, = gsc.computeCov3D(st["rots"], st["scales"], d, False)
    c2, = gsc.computeCov2D(c3, pcs, cam.Rcw, d, cam.fx, cam.fy, W, H, False)
    w, ddc, ylm = gsc.sh2Weight_fast(st["dc"], st["A"], st["B"], st["pws"], cam.twc, True, 5, 15)
    cinv, areas = gsc.inverseCov2D(c2, d, False)
    ref_layer, contrib, rft, ranges, gsid = gsc.splat_weight(H, W, 5, us, cinv, st["alphas"], d, w,
                                                             areas)
    assert max_abs(ref_layer.reshape(layer.shape), layer) < IMG_TOL
    dW, = gsc.splat_weight_B(H, W, 5, us, cinv, st["alphas"], d, w, contrib, rft, ranges, gsid,
                             g.reshape(ref_layer.shape).contiguous())
    dw = dW.squeeze(1)
    dA, dB = gsc.sh2Weight_fast_B(st["A"], st["B"], ylm, dw, 5, 15)
    expect = dict(dc=dw * ddc, A=dA, B=dB)
    for k in ("dc", "A", "B"):
        assert rel_err(leaf[k].grad, expect[k]) < 1e-5, k
    ops_in = {k: st[k].detach().clone().requires_grad_(True) for k in ("dc", "A", "B")}
    ol, _ = splat_palette_weights(st["pws"], st["alphas"], st["scales"], st["rots"], cam,
                                  dc=ops_in["dc"], A=ops_in["A"], B=ops_in["B"])
    (ol.reshape(layer.shape) * g).sum().backward()
    for k in ("dc", "A", "B"):
        assert rel_err(ops_in[k].grad, expect[k]) < 1e-5, k


def test_fused_forward_overlapped_count_and_overflow(cuda_ok):
    """Repeated renders of one size enqueue the sort before the patch count is
    read back; a view with more patches than the stored capacity is redone
    exactly.  All match the operator sequence."""
    sc, st, cam_far = _setup("full", 0, torch.float32, n=15000, W=160, H=96, eye=(0.0, -14.0, 0.0))
    cam_near = look_at((0.0, -5.0, 0.5), width=160, height=96, device="cuda")
    gsc._CAPACITY.pop((15000, 96, 160), None)
    for cam in (cam_far, cam_far, cam_near, cam_near):
        ref = forward_ops(gsc, st, cam, "full")
        (layer, ft, depths), _ = _render(st, cam, "full")
        assert max_abs(layer, ref["layer"]) < IMG_TOL and max_abs(ft, ref["final_tau"]) < IMG_TOL
        assert torch.equal(depths, ref["depths"].reshape(-1))
    assert gsc._CAPACITY[(15000, 96, 160)][0] >= int(ref["gsid"].numel())


@pytest.mark.parametrize("dtype,geom", [(torch.float32, False), (torch.float32, True),
                                        (torch.bfloat16, False)])
def test_render_views_sums_view_gradients_in_fp32(cuda_ok, dtype, geom):
    """render_palette_views: each view's forward equals render_palette's; the
    backward equals the sum of the single-view gradients taken in FP32 (first
    view through gsb_render_backward, the others through
    gsb_render_backward_accumulate), cast once to the parameters' dtype.  FP32
    sums are compared to 1e-6 relative (the adjoint's atomics may add in a
    different order); BF16 gradients to one BF16 rounding of the FP32 sum."""
    from palette_b200.render import render_palette_views
    sc, st, _ = _setup("lowrank", 3, dtype, n=20000, W=96, H=80, eye=(4.0, -6.0, 1.0))
    cams = [look_at(e, width=96, height=80, device="cuda")
            for e in ((4.0, -6.0, 1.0), (-5.0, -5.0, 2.0), (0.5, 7.0, -1.0))]
    g = torch.Generator("cuda").manual_seed(9)
    dls = [torch.randn((5, 80, 96), device="cuda", generator=g) for _ in cams]
    names = ["dc", "A", "B"] + (list(GEOM) if geom else [])

    def leaves(dt):
        return {k: st[k].detach().to(dt if k in ("dc", "A", "B") else torch.float32).clone()
                .requires_grad_(k in names) for k in list(GEOM) + ["dc", "A", "B"]}
    lv = leaves(dtype)
    layers, taus, depths = render_palette_views(lv["pws"], lv["rots"], lv["scales"], lv["alphas"],
                                                cams, dc=lv["dc"], A=lv["A"], B=lv["B"])
    torch.autograd.backward(layers, dls)
    # reference: single views with FP32 copies of the same parameter values
    ref = leaves(torch.float32)
    for v, cam in enumerate(cams):
        layer, ft, d = render_palette(ref["pws"], ref["rots"], ref["scales"], ref["alphas"], cam,
                                      dc=ref["dc"], A=ref["A"], B=ref["B"])
        if dtype == torch.float32:
            assert torch.equal(layers[v], layer) and torch.equal(taus[v], ft)
            assert torch.equal(depths[v], d)
        else:
            assert max_abs(layers[v], layer) < 1e-5
        layer.backward(dls[v])
    for k in names:
        got, want = lv[k].grad, ref[k].grad
        assert got.dtype == lv[k].dtype
        if dtype == torch.float32:
            assert rel_err(got, np_of(want).astype(np.float64)) < 1e-6, k
        else:  # the FP32 sum rounded once to BF16 (atomics order aside: within 1 BF16 ulp)
            assert rel_err(got.float(), np_of(want).astype(np.float64)) < 5e-3, k
            close = (got.float() - want.to(torch.bfloat16).float()).abs()
            assert bool((close <= want.abs() * 2.0 ** -7 + 1e-30).all()), k


@pytest.mark.parametrize("mode,K,dtype", [("full", 5, torch.float32), ("full", 5, torch.bfloat16),
                                          ("lowrank", 6, torch.float32)])
def test_render_views_accumulate_padded_rows(cuda_ok, mode, K, dtype):
    """The accumulating adjoint adds into the gradient rows it bulk-loads with
    its inputs (full blocks) or by a read-add-write (the partial last block).
    Full-SH rows (16K floats) and even-K rows are built at a padded stride and
    packed before the store, so both take the add in the packing step: the
    views' summed gradients equal the single-view gradients summed in FP32."""
    from palette_b200.render import render_palette_views
    n, W, H = 9000, 80, 64  # 70 full blocks of 128 and a partial one
    sc = synthetic_scene(n, seed=5, mode=mode, rank=3)
    st = to_torch(sc, "cuda", dtype)
    if mode == "lowrank":  # K = 6 palette weights, rank-3 factors A [n,6,3], B [n,3,15]
        gen = torch.Generator().manual_seed(6)
        st["dc"] = (0.3 * torch.randn((n, K), generator=gen)).to("cuda", dtype)
        st["A"] = (0.2 * torch.randn((n, K, 3), generator=gen)).to("cuda", dtype)
        st["B"] = (0.2 * torch.randn((n, 3, 15), generator=gen)).to("cuda", dtype)
    cams = [look_at(e, width=W, height=H, device="cuda")
            for e in ((4.0, -6.0, 1.0), (-5.0, -5.0, 2.0), (0.5, 7.0, -1.0))]
    g = torch.Generator("cuda").manual_seed(3)
    dls = [torch.randn((K, H, W), device="cuda", generator=g) for _ in cams]
    pnames = ["shs"] if mode == "full" else ["dc", "A", "B"]

    def leaves(dt):
        out = {k: st[k].detach().float() for k in GEOM}
        out.update({k: st[k].detach().to(dt).clone().requires_grad_() for k in pnames})
        return out

    def kw(lv):
        return {k: lv[k] for k in pnames}
    lv = leaves(dtype)
    layers, _, _ = render_palette_views(lv["pws"], lv["rots"], lv["scales"], lv["alphas"], cams,
                                        **kw(lv))
    torch.autograd.backward(layers, dls)
    ref = leaves(torch.float32)
    for v, cam in enumerate(cams):
        layer, _, _ = render_palette(ref["pws"], ref["rots"], ref["scales"], ref["alphas"], cam,
                                     **kw(ref))
        layer.backward(dls[v])
    for k in pnames:
        got, want = lv[k].grad.float(), ref[k].grad
        assert float(want.abs().max()) > 0, k
        if dtype == torch.float32:
            assert rel_err(got, np_of(want).astype(np.float64)) < 1e-6, k
        else:
            assert rel_err(got, np_of(want).astype(np.float64)) < 5e-3, k
