"""GPU parity: every gsplatcu operator against the CPU oracle on the same
seeded inputs.  Tolerances: tile lists, ranges, in-place depth/area updates
and sort order bit-exact; images within 1e-5 abs (FP32 storage); gradients
within 1e-4 relative (norm-wise); preprocess values within a few FP32 ulps.

Compositing decisions: the oracle evaluates exp() with the host C library and
the GPU with CUDA's expf.  The two may differ by an ulp, which changes a skip
(alpha' < 0.002) or stop (T < 1e-4) decision only where alpha' or T lies
within that ulp of its threshold.  Such pixels (a different contributor
index) are counted, printed and excluded from the image comparison; at most
``MAX_EXP_FLIPS`` per image are allowed (measured on a B200: 0 such pixels in
every case of this file).  Against the reference build itself,
which uses the same expf, contributor indices are compared bit for bit
(tests/test_gpu_reference.py, tests/test_gpu_fullsize.py)."""
import numpy as np
import pytest
import torch

import gsplatcu as gsc
from oracle import oracle as orc
from palette_b200.scene import look_at, synthetic_scene, to_torch
from helpers import forward_ops, max_abs, np_of, rel_err

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5
GRAD_REL = 1e-4
MAX_EXP_FLIPS = 2


def _compare_composite(name, img, contrib, ft, ref):
    """Contributor indices equal but for at most MAX_EXP_FLIPS pixels (an
    exp() ulp at a threshold, see the module docstring); images and final
    transmittance within IMG_TOL on every other pixel."""
    same = np_of(contrib) == ref["contrib"]
    flips = int((~same).sum())
    print(f"{name}: {flips} of {same.size} pixels with a different contributor index")
    assert flips <= MAX_EXP_FLIPS
    assert max_abs(np_of(img)[:, same], ref["out"][:, same]) < IMG_TOL
    assert max_abs(np_of(ft)[same], ref["ft"][same]) < IMG_TOL

CASES = [  # (N, W, H, eye)
    (2000, 64, 64, (0.0, -8.0, 0.0)),
    (20000, 256, 256, (0.0, -8.0, 0.0)),
    (5000, 200, 120, (5.0, -5.0, 2.0)),  # sizes not multiples of 16
]


def _scene(n, seed, mode="full", rank=3, dtype=torch.float32):
    sc = synthetic_scene(n, seed=seed, mode=mode, rank=rank)
    return sc, to_torch(sc, "cuda", dtype)


def _cam(W, H, eye, dev="cuda"):
    return look_at(eye, width=W, height=H, device=dev)


@pytest.mark.parametrize("case", CASES)
def test_preprocess_ops_match_oracle(cuda_ok, case):
    n, W, H, eye = case
    sc, st = _scene(n, seed=n)
    cam = _cam(W, H, eye)
    Rcw, tcw, twc = orc.camera_arrays(cam, np.float32)
    us, pcs, depths, du = gsc.project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, True)
    o_us, o_pcs, o_d, o_du = orc.project(sc["pws"], Rcw, tcw, cam.fx, cam.fy, cam.cx, cam.cy, True)
    assert np.array_equal(np_of(depths) < 0.2, o_d < 0.2)
    np.testing.assert_allclose(np_of(us), o_us, rtol=2e-6, atol=1e-4)
    np.testing.assert_allclose(np_of(pcs), o_pcs, rtol=2e-6, atol=1e-6)
    np.testing.assert_allclose(np_of(du), o_du, rtol=1e-5, atol=1e-4)
    c3, dq, ds = gsc.computeCov3D(st["rots"], st["scales"], depths, True)
    o_c3, o_dq, o_ds = orc.cov3d(sc["rots"], sc["scales"], o_d, True)
    np.testing.assert_allclose(np_of(c3), o_c3, rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(np_of(dq), o_dq, rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(np_of(ds), o_ds, rtol=1e-4, atol=1e-7)
    c2, d3, dp = gsc.computeCov2D(c3, pcs, cam.Rcw, depths, cam.fx, cam.fy, cam.width, cam.height, True)
    o_c2, o_d3, o_dp = orc.cov2d(o_c3, o_pcs, Rcw, o_d, cam.fx, cam.fy, cam.width, cam.height, True)
    np.testing.assert_allclose(np_of(c2), o_c2, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(np_of(d3), o_d3, rtol=1e-4, atol=1e-3)
    assert rel_err(dp, o_dp) < 1e-4
    cinv, areas, dci = gsc.inverseCov2D(c2, depths, True)
    o_cinv, o_areas, o_dci = orc.inverse_cov2d(o_c2, o_d, True)
    assert np.array_equal(np_of(depths) < 0.2, o_d < 0.2)
    assert rel_err(cinv, o_cinv) < 1e-5
    assert np.mean(np_of(areas) != o_areas) < 1e-3  # ceil() ties at FP32 ulps only
    assert rel_err(dci, o_dci) < 1e-4
    w, dshs, dpw = gsc.sh2Weight(st["shs"], st["pws"], cam.twc, True, 5)
    o_w, o_dshs, o_dpw = orc.sh2feat(sc["shs"], sc["pws"], twc, 5, True)
    np.testing.assert_allclose(np_of(w), o_w, rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(np_of(dshs), o_dshs, rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(np_of(dpw), o_dpw, rtol=1e-4, atol=1e-6)
    col, dcs, dcp = gsc.sh2Color(st["shs"][:, :48].contiguous(), st["pws"], cam.twc, True)
    o_col, o_dcs, o_dcp = orc.sh2feat(sc["shs"][:, :48], sc["pws"], twc, 3, True)
    np.testing.assert_allclose(np_of(col), o_col, rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(np_of(dcp), o_dcp, rtol=1e-4, atol=1e-6)


def _oracle_splat(H, W, K, pre, alphas, feats, tau_init):
    us, cinv = np_of(pre["us"]), np_of(pre["cinv"])
    depths, areas = np_of(pre["depths"]).copy(), np_of(pre["areas"]).astype(np.int32).copy()
    b = orc.bin_gaussians(us, areas, depths, H, W)
    out, contrib, ft = orc.draw(H, W, K, b["ranges"], b["gsid"], us, cinv, np_of(alphas),
                                np_of(feats), tau_init)
    return dict(b=b, out=out, contrib=contrib, ft=ft, depths=depths, areas=areas)


def _gpu_pre(st, cam):
    us, pcs, depths = gsc.project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
    c3, = gsc.computeCov3D(st["rots"], st["scales"], depths, False)
    c2, = gsc.computeCov2D(c3, pcs, cam.Rcw, depths, cam.fx, cam.fy, cam.width, cam.height, False)
    cinv, areas = gsc.inverseCov2D(c2, depths, False)
    return dict(us=us, cinv=cinv, depths=depths, areas=areas)


@pytest.mark.parametrize("case", CASES)
def test_splat_weight_lists_bitexact_and_image(cuda_ok, case):
    n, W, H, eye = case
    sc, st = _scene(n, seed=n + 1)
    cam = _cam(W, H, eye)
    pre = _gpu_pre(st, cam)
    w, = gsc.sh2Weight(st["shs"], st["pws"], cam.twc, False, 5)
    ref = _oracle_splat(H, W, 5, {k: v.clone() for k, v in pre.items()}, st["alphas"], w, 0.0)
    layer, contrib, ft, ranges, gsid = gsc.splat_weight(H, W, 5, pre["us"], pre["cinv"], st["alphas"],
                                                        pre["depths"], w, pre["areas"])
    # binning: bit-exact lists, ranges and in-place updates
    assert np.array_equal(np_of(gsid), ref["b"]["gsid"])
    assert np.array_equal(np_of(ranges), ref["b"]["ranges"])
    assert np.array_equal(np_of(pre["depths"]), ref["depths"])
    assert np.array_equal(np_of(pre["areas"]), ref["areas"])
    # compositing
    _compare_composite(f"splat_weight {case}", layer, contrib, ft, ref)
    assert np.mean(np.abs(np_of(layer) - ref["out"])) < 1e-7


def test_splat_weight_empty_tiles_and_determinism(cuda_ok):
    sc, st = _scene(300, seed=9)
    cam = _cam(160, 96, (0.0, -30.0, 0.0))  # far away: most tiles empty
    pre = _gpu_pre(st, cam)
    w, = gsc.sh2Weight(st["shs"], st["pws"], cam.twc, False, 5)
    outs = [gsc.splat_weight(96, 160, 5, pre["us"], pre["cinv"], st["alphas"], pre["depths"].clone(),
                             w, pre["areas"].clone()) for _ in range(2)]
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    layer, contrib, ft, ranges, gsid = outs[0]
    empty = np_of(ranges)[:, 1] == np_of(ranges)[:, 0]
    assert empty.any()
    gx = (160 + 15) // 16
    t = int(np.nonzero(empty)[0][0])
    ty, tx = divmod(t, gx)
    blk = np_of(ft)[ty * 16:(ty + 1) * 16, tx * 16:(tx + 1) * 16]
    assert np.all(blk == 0.0)  # splat_weight leaves final_tau at 0 in empty tiles
    img, _, ftc, _, _ = gsc.splat_color(96, 160, pre["us"], pre["cinv"], st["alphas"],
                                        pre["depths"].clone(), w[:, :3].contiguous(),
                                        pre["areas"].clone())
    assert np.all(np_of(ftc)[ty * 16:(ty + 1) * 16, tx * 16:(tx + 1) * 16] == 1.0)


def test_edge_cases(cuda_ok):
    dev = "cuda"
    cam = _cam(64, 64, (0.0, -8.0, 0.0))
    # N = 0
    z = torch.zeros((0, 2), device=dev)
    out = gsc.splat_weight(64, 64, 5, z, torch.zeros((0, 3), device=dev), torch.zeros((0, 1), device=dev),
                           torch.zeros((0,), device=dev), torch.zeros((0, 5), device=dev),
                           torch.zeros((0, 2), dtype=torch.int32, device=dev))
    assert out[4].numel() == 0 and float(out[0].abs().sum()) == 0.0
    # a single patch (M == 1): the reference never writes the end of the tile's range
    us = torch.tensor([[20.0, 20.0]], device=dev)
    cinv = torch.tensor([[1.0, 0.0, 1.0]], device=dev)
    al = torch.tensor([[0.9]], device=dev)
    d = torch.tensor([3.0], device=dev)
    ar = torch.tensor([[2, 2]], dtype=torch.int32, device=dev)
    w = torch.ones((1, 5), device=dev)
    layer, contrib, ft, ranges, gsid = gsc.splat_weight(64, 64, 5, us, cinv, al, d, w, ar)
    assert gsid.tolist() == [0] and ranges[5].tolist() == [0, 0]
    assert float(layer.abs().sum()) == 0.0
    # two patches: drawn
    ar2 = torch.tensor([[2, 2], [2, 2]], dtype=torch.int32, device=dev)
    layer, contrib, *_ = gsc.splat_weight(64, 64, 5, us.repeat(2, 1), cinv.repeat(2, 1), al.repeat(2, 1),
                                          d.repeat(2), w.repeat(2, 1), ar2)
    assert float(layer[0, 20, 20]) > 0.9
    # one Gaussian covering every tile of a 1x1 and a 17x33 image
    for H, W in ((1, 1), (17, 33)):
        big = gsc.splat_weight(H, W, 5, torch.tensor([[0.0, 0.0]], device=dev), cinv * 1e-3, al,
                               d.clone(), w, torch.tensor([[900, 900]], dtype=torch.int32, device=dev))
        assert big[4].numel() == ((W + 15) // 16) * ((H + 15) // 16)
        assert big[0].shape == (5, H, W)
    # bad inputs raise instead of computing anything
    with pytest.raises(ValueError):
        gsc.project(torch.zeros(4, 3), cam.Rcw.cpu(), cam.tcw.cpu(), 1, 1, 0, 0, False)
    with pytest.raises(TypeError):
        gsc.project(torch.zeros(4, 3, device=dev, dtype=torch.float64), cam.Rcw, cam.tcw, 1, 1, 0, 0, False)
    with pytest.raises(ValueError):
        gsc.sh2Weight(torch.zeros(4, 10, device=dev), torch.zeros(4, 3, device=dev), cam.twc, False, 5)


def test_noncontiguous_inputs_match_contiguous(cuda_ok):
    sc, st = _scene(1000, seed=11)
    cam = _cam(64, 64, (0.0, -8.0, 0.0))
    big = torch.zeros((1000, 6), device="cuda")
    big[:, ::2] = st["pws"]
    pws_nc = big[:, ::2]
    assert not pws_nc.is_contiguous()
    a = gsc.project(pws_nc, cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
    b = gsc.project(st["pws"], cam.Rcw, cam.tcw, cam.fx, cam.fy, cam.cx, cam.cy, False)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


@pytest.mark.parametrize("case", CASES[:2])
def test_splat_weight_backward_matches_oracle(cuda_ok, case):
    n, W, H, eye = case
    sc, st = _scene(n, seed=n + 2)
    cam = _cam(W, H, eye)
    pre = _gpu_pre(st, cam)
    w, = gsc.sh2Weight(st["shs"], st["pws"], cam.twc, False, 5)
    layer, contrib, ft, ranges, gsid = gsc.splat_weight(H, W, 5, pre["us"], pre["cinv"], st["alphas"],
                                                        pre["depths"], w, pre["areas"])
    g = torch.randn((5, H, W), device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    dW, = gsc.splat_weight_B(H, W, 5, pre["us"], pre["cinv"], st["alphas"], pre["depths"], w,
                             contrib, ft, ranges, gsid, g)
    ref = orc.draw_backward(H, W, 5, np_of(ranges), np_of(gsid), np_of(pre["us"]), np_of(pre["cinv"]),
                            np_of(st["alphas"]), np_of(w), np_of(ft), np_of(contrib), np_of(g))
    assert dW.shape == (n, 1, 5)
    assert rel_err(dW[:, 0], ref["dfeat"]) < GRAD_REL
    # full adjoint (opacity / centre / conic, plus the final-transmittance term)
    gT = torch.randn((H, W), device="cuda")
    dW2, du, dq, da = gsc.splat_weight_B_full(H, W, 5, pre["us"], pre["cinv"], st["alphas"],
                                              pre["depths"], w, contrib, ft, ranges, gsid, g, gT)
    ref2 = orc.draw_backward(H, W, 5, np_of(ranges), np_of(gsid), np_of(pre["us"]), np_of(pre["cinv"]),
                             np_of(st["alphas"]), np_of(w), np_of(ft), np_of(contrib), np_of(g),
                             np_of(gT))
    assert rel_err(dW2[:, 0], ref2["dfeat"]) < GRAD_REL
    assert rel_err(da.reshape(-1), ref2["dalpha"]) < GRAD_REL
    assert rel_err(du[:, 0], ref2["du"]) < GRAD_REL
    assert rel_err(dq[:, 0], ref2["dconic"]) < GRAD_REL


def test_splat_color_forward_backward_matches_oracle(cuda_ok):
    n, W, H, eye = CASES[1]
    sc, st = _scene(n, seed=21)
    cam = _cam(W, H, eye)
    pre = _gpu_pre(st, cam)
    col, = gsc.sh2Color(st["shs"][:, :48].contiguous(), st["pws"], cam.twc, False)
    ref = _oracle_splat(H, W, 3, {k: v.clone() for k, v in pre.items()}, st["alphas"], col, 1.0)
    img, contrib, ft, ranges, gsid = gsc.splat_color(H, W, pre["us"], pre["cinv"], st["alphas"],
                                                     pre["depths"], col, pre["areas"])
    assert np.array_equal(np_of(gsid), ref["b"]["gsid"])
    _compare_composite("splat_color", img, contrib, ft, ref)
    g = torch.randn((3, H, W), device="cuda")
    du, dq, da, dc = gsc.splat_color_B(H, W, pre["us"], pre["cinv"], st["alphas"], pre["depths"], col,
                                       contrib, ft, ranges, gsid, g)
    r = orc.draw_backward(H, W, 3, np_of(ranges), np_of(gsid), np_of(pre["us"]), np_of(pre["cinv"]),
                          np_of(st["alphas"]), np_of(col), np_of(ft), np_of(contrib), np_of(g))
    assert du.shape == (n, 1, 2) and dq.shape == (n, 1, 3) and da.shape == (n, 1, 1) and dc.shape == (n, 1, 3)
    assert rel_err(dc[:, 0], r["dfeat"]) < GRAD_REL
    assert rel_err(da.reshape(-1), r["dalpha"]) < GRAD_REL
    assert rel_err(du[:, 0], r["du"]) < GRAD_REL
    assert rel_err(dq[:, 0], r["dconic"]) < GRAD_REL


@pytest.mark.parametrize("rank", [1, 3])
@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_lowrank_weights_and_backward(cuda_ok, rank, dtype):
    n = 4000
    sc, st = _scene(n, seed=30 + rank, mode="lowrank", rank=rank, dtype=dtype)
    cam = _cam(64, 64, (1.0, -7.0, 0.5))
    A, B = st["A"], st["B"]
    if rank == 1:  # the reference's 2-D call
        A, B = A[:, :, 0].contiguous(), B[:, 0, :].contiguous()
    w, ddc, ylm = gsc.sh2Weight_fast(st["dc"], A, B, st["pws"], cam.twc, True, 5, 15)
    # the oracle sees the same (possibly bf16-rounded) parameter values
    f = lambda t: t.float().cpu().numpy()
    twc = orc.camera_arrays(cam, np.float32)[2]
    o_w, o_ddc, o_ylm = orc.sh2weight_fast(f(st["dc"]), f(A), f(B), sc["pws"], twc, 5, 15, True)
    np.testing.assert_allclose(np_of(w), o_w, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(np_of(ylm), o_ylm, rtol=1e-5, atol=1e-6)
    assert torch.all(ddc == np.float32(0.28209479177387814))
    dw = torch.randn((n, 5), device="cuda")
    dA, dB = gsc.sh2Weight_fast_B(A, B, ylm, dw, 5, 15)
    o_dA, o_dB = orc.sh2weight_fast_b(f(A), f(B), np_of(ylm), np_of(dw), 5, 15)
    assert dA.shape == A.shape and dB.shape == B.shape
    assert rel_err(dA, o_dA) < 1e-5 and rel_err(dB, o_dB) < 1e-5


def test_bf16_full_weights_match_rounded_oracle(cuda_ok):
    sc, st = _scene(3000, seed=40, dtype=torch.bfloat16)
    cam = _cam(64, 64, (0.0, -8.0, 0.0))
    w, = gsc.sh2Weight(st["shs"], st["pws"], cam.twc, False, 5)
    twc = orc.camera_arrays(cam, np.float32)[2]
    o_w, = orc.sh2feat(st["shs"].float().cpu().numpy(), sc["pws"], twc, 5, False)
    np.testing.assert_allclose(np_of(w), o_w, rtol=1e-5, atol=2e-7)


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
@pytest.mark.parametrize("nb,K", [(1, 3), (1, 8), (4, 3), (4, 5), (9, 5), (9, 8), (16, 3), (16, 5),
                                  (16, 8)])
def test_sh_every_band_count_with_jacobians(cuda_ok, nb, K, dtype):
    """The SH kernel is instantiated per band count (1, 4, 9, 16): weights
    (or colours for K = 3) and both Jacobian outputs for each, FP32 rows and
    BF16 rows (staged as raw element pairs when nb*K is even, read in place
    when it is odd), against the oracle on the same stored values: weights
    and basis within 1e-5 relative, direction derivatives within 1e-4
    (norm-wise)."""
    n = 3000
    g = torch.Generator().manual_seed(200 + nb * 10 + K)
    vals = (torch.randn((n, nb * K), generator=g) * 0.2).to(dtype)
    shs = vals.cuda()
    sc, st = _scene(n, seed=43)
    cam = _cam(64, 64, (0.5, -7.0, 1.0))
    twc = orc.camera_arrays(cam, np.float32)[2]
    if K == 3:
        f, dsh, dpw = gsc.sh2Color(shs, st["pws"], cam.twc, True)
        f0, = gsc.sh2Color(shs, st["pws"], cam.twc, False)
    else:
        f, dsh, dpw = gsc.sh2Weight(shs, st["pws"], cam.twc, True, K)
        f0, = gsc.sh2Weight(shs, st["pws"], cam.twc, False, K)
    assert torch.equal(f, f0)  # the Jacobian outputs leave the weights unchanged
    o_f, o_dsh, o_dpw = orc.sh2feat(vals.float().numpy(), sc["pws"], twc, K, True)
    np.testing.assert_allclose(np_of(f), o_f, rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(np_of(dsh), o_dsh, rtol=1e-5, atol=2e-7)
    if nb > 1:
        assert rel_err(dpw, o_dpw) < 1e-4
    else:
        assert float(dpw.abs().max()) == 0.0


@pytest.mark.parametrize("nb,K,offset", [(9, 5, 0), (9, 3, 0), (16, 5, 1), (16, 3, 1), (4, 5, 1),
                                         (9, 5, 1)])
def test_bf16_sh_rows_odd_length_or_misaligned(cuda_ok, nb, K, offset):
    """BF16 coefficient rows that the SH kernel cannot stage as 32-bit
    element pairs -- an odd row length (nb*K = 45, 27, 15) or a base
    address offset by one element (a contiguous view at an odd storage
    offset) -- are read in place; results match the oracle on the same
    BF16-rounded values.  FP32 arithmetic: 1e-5 relative."""
    n = 3000
    g = torch.Generator().manual_seed(100 + nb * 10 + K + offset)
    vals = (torch.randn((n, nb * K), generator=g) * 0.2).to(torch.bfloat16)
    if offset:
        buf = torch.empty((n * nb * K + 1,), dtype=torch.bfloat16, device="cuda")
        buf[1:] = vals.reshape(-1).cuda()
        shs = buf[1:].view(n, nb * K)
        assert shs.is_contiguous() and shs.data_ptr() % 4 == 2
    else:
        shs = vals.cuda()
    sc, st = _scene(n, seed=41)
    cam = _cam(64, 64, (1.0, -8.0, 0.5))
    twc = orc.camera_arrays(cam, np.float32)[2]
    if K == 3:
        f, dsh, dpw = gsc.sh2Color(shs, st["pws"], cam.twc, True)
    else:
        f, dsh, dpw = gsc.sh2Weight(shs, st["pws"], cam.twc, True, K)
    o_f, o_dsh, o_dpw = orc.sh2feat(vals.float().numpy(), sc["pws"], twc, K, True)
    np.testing.assert_allclose(np_of(f), o_f, rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(np_of(dsh), o_dsh, rtol=1e-5, atol=2e-7)
    assert rel_err(dpw, o_dpw) < 1e-4


@pytest.mark.parametrize("nb,K,offset", [(16, 5, 1), (16, 5, 2), (4, 5, 3), (16, 8, 1),
                                         (9, 5, 0), (16, 3, 0)])
def test_fp32_sh_staging_modes_agree(cuda_ok, nb, K, offset):
    """FP32 coefficient rows are staged by 16-byte copies when the row length
    is a multiple of 4 and the base 16-byte aligned, else by 4-byte copies.
    A contiguous view at a storage offset of 1-3 floats takes the 4-byte
    path; rows of 45 or 48 floats (9 x 5, 16 x 3) take it as well (or the
    16-byte one, 48). Every output equals that of the aligned call bit for
    bit, and matches the oracle."""
    n = 3000  # 46 full blocks of 64 rows and a last one of 56
    g = torch.Generator().manual_seed(300 + nb * 10 + K + offset)
    vals = torch.randn((n, nb * K), generator=g) * 0.2
    ref_shs = vals.cuda()
    assert ref_shs.data_ptr() % 16 == 0
    if offset:
        buf = torch.empty((n * nb * K + offset,), device="cuda")
        buf[offset:] = ref_shs.reshape(-1)
        shs = buf[offset:].view(n, nb * K)
        assert shs.is_contiguous() and shs.data_ptr() % 16 == 4 * offset
    else:
        shs = ref_shs
    sc, st = _scene(n, seed=44)
    cam = _cam(64, 64, (0.5, -7.5, 0.8))
    call = (lambda s, j: gsc.sh2Color(s, st["pws"], cam.twc, j)) if K == 3 else \
        (lambda s, j: gsc.sh2Weight(s, st["pws"], cam.twc, j, K))
    for jac in (False, True):
        got, want = call(shs, jac), call(ref_shs, jac)
        for x, y in zip(got, want):
            assert torch.equal(x, y)
    twc = orc.camera_arrays(cam, np.float32)[2]
    f, dsh, dpw = call(shs, True)
    o_f, o_dsh, o_dpw = orc.sh2feat(vals.numpy(), sc["pws"], twc, K, True)
    np.testing.assert_allclose(np_of(f), o_f, rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(np_of(dsh), o_dsh, rtol=1e-5, atol=2e-7)
    assert rel_err(dpw, o_dpw) < 1e-4


@pytest.mark.parametrize("rank", [1, 3])
def test_bf16_lowrank_unaligned_factors_agree(cuda_ok, rank):
    """BF16 low-rank factors are bulk-copied raw when a block's spans start on
    16-byte boundaries, else copied raw element by element. Factors in views
    at an odd storage offset (every block on the element path) give the same
    weights, basis and factor gradients bit for bit as aligned ones."""
    n = 4000
    sc, st = _scene(n, seed=50 + rank, mode="lowrank", rank=rank, dtype=torch.bfloat16)
    cam = _cam(64, 64, (0.8, -7.0, 0.4))
    A, B = st["A"], st["B"]
    if rank == 1:
        A, B = A[:, :, 0].contiguous(), B[:, 0, :].contiguous()

    def shifted(t):
        buf = torch.empty((t.numel() + 1,), dtype=t.dtype, device="cuda")
        buf[1:] = t.reshape(-1)
        v = buf[1:].view(t.shape)
        assert v.is_contiguous() and v.data_ptr() % 4 == 2
        return v

    dc_s, A_s, B_s = shifted(st["dc"]), shifted(A), shifted(B)
    got = gsc.sh2Weight_fast(dc_s, A_s, B_s, st["pws"], cam.twc, True, 5, 15)
    want = gsc.sh2Weight_fast(st["dc"], A, B, st["pws"], cam.twc, True, 5, 15)
    for x, y in zip(got, want):
        assert torch.equal(x, y)
    dw = torch.randn((n, 5), device="cuda", generator=torch.Generator("cuda").manual_seed(9))
    gA, gB = gsc.sh2Weight_fast_B(A_s, B_s, want[2], dw, 5, 15)
    wA, wB = gsc.sh2Weight_fast_B(A, B, want[2], dw, 5, 15)
    assert torch.equal(gA, wA) and torch.equal(gB, wB)


def test_lab2rgb_matches_oracle(cuda_ok):
    g = torch.Generator().manual_seed(0)
    lab = torch.stack([torch.rand(40, 50, generator=g), torch.rand(40, 50, generator=g) * 160 - 80,
                       torch.rand(40, 50, generator=g) * 160 - 80])
    rgb = gsc.lab2rgb(lab.cuda())
    np.testing.assert_allclose(np_of(rgb), orc.lab2rgb(lab.numpy()), rtol=1e-5, atol=1e-6)


def test_weight_function_sequence_end_to_end(cuda_ok):
    """The full WeightGSFunctionTest forward sequence (gsplat/gsmodel.py:107-118) on
    the GPU against the oracle's FP32 pipeline."""
    n, W, H, eye = CASES[1]
    sc, st = _scene(n, seed=50)
    cam = _cam(W, H, eye)
    r = forward_ops(gsc, st, cam, "full")
    twc = orc.camera_arrays(cam, np.float32)[2]
    o_w, = orc.sh2feat(sc["shs"], sc["pws"], twc, 5, False)
    o = orc.render_weights(sc["pws"], sc["rots"], sc["scales"], sc["alphas"], o_w, cam)
    assert np.mean(np_of(r["gsid"]) == o["gsid"]) > 0.999 if len(o["gsid"]) == r["gsid"].numel() else True
    assert np.mean(np.abs(np_of(r["layer"]) - o["layer"])) < 1e-6


@pytest.mark.parametrize("crowd", [300, 5000, 17000])
def test_sort_long_lists_and_ties_bitexact(cuda_ok, crowd):
    """Crowded tiles (up to 17k patches) and many equal depth keys: the sort
    gives the reference's order (ties by Gaussian id)."""
    rng = np.random.default_rng(crowd)
    n = 3000 + crowd
    us = np.concatenate([rng.uniform(0, 200, (3000, 2)), 40 + rng.uniform(-1, 1, (crowd, 2))])
    areas = np.concatenate([rng.integers(1, 30, (3000, 2)), np.full((crowd, 2), 3)]).astype(np.int32)
    depths = rng.uniform(0.1, 30.0, n).astype(np.float32)
    depths[::7] = depths[3]  # many equal depth keys: ties ordered by id
    cinv = np.tile(np.array([[0.3, 0.01, 0.2]], np.float32), (n, 1))
    al = rng.uniform(0.01, 0.9, (n, 1)).astype(np.float32)
    w = rng.uniform(0, 1, (n, 5)).astype(np.float32)
    H, W = 120, 200
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=a.dtype)).cuda()
    d_g, a_g = t(depths.copy()), t(areas.copy())
    layer, contrib, ft, ranges, gsid = gsc.splat_weight(H, W, 5, t(us.astype(np.float32)), t(cinv),
                                                        t(al), d_g, t(w), a_g)
    dd, aa = depths.copy(), areas.copy()
    b = orc.bin_gaussians(us.astype(np.float32), aa, dd, H, W)
    assert np.array_equal(np_of(gsid), b["gsid"])
    assert np.array_equal(np_of(ranges), b["ranges"])
    assert np.array_equal(np_of(d_g), dd) and np.array_equal(np_of(a_g), aa)
    counts = b["ranges"][:, 1] - b["ranges"][:, 0]
    assert counts.max() >= crowd


def test_splat_weight_overlapped_count_and_overflow_bitexact(cuda_ok):
    """After the first render of a size, the sort and compositing are enqueued
    before the patch count is read back (capacity from earlier renders); a
    view needing more patches is sorted and composited again exactly.  Every
    render's lists, ranges, in-place updates and image equal the oracle's."""
    n, W, H = 12000, 144, 112
    sc, st = _scene(n, seed=77)
    gsc._CAPACITY.pop((n, H, W), None)
    for eye in ((0.0, -15.0, 0.0), (1.0, -14.0, 0.5), (0.0, -5.0, 0.5), (0.5, -5.5, 0.0)):
        cam = _cam(W, H, eye)
        pre = _gpu_pre(st, cam)
        w, = gsc.sh2Weight(st["shs"], st["pws"], cam.twc, False, 5)
        ref = _oracle_splat(H, W, 5, {k: v.clone() for k, v in pre.items()}, st["alphas"], w, 0.0)
        layer, contrib, ft, ranges, gsid = gsc.splat_weight(H, W, 5, pre["us"], pre["cinv"],
                                                            st["alphas"], pre["depths"], w,
                                                            pre["areas"])
        assert (n, H, W) in gsc._CAPACITY
        assert np.array_equal(np_of(gsid), ref["b"]["gsid"])
        assert np.array_equal(np_of(ranges), ref["b"]["ranges"])
        assert np.array_equal(np_of(pre["depths"]), ref["depths"])
        assert np.array_equal(np_of(pre["areas"]), ref["areas"])
        _compare_composite(f"overlapped count {eye}", layer, contrib, ft, ref)


def test_backward_reuses_forward_records_only_when_inputs_unchanged(cuda_ok):
    """splat_weight_B takes the forward's packed records when it is handed the
    same, unmodified tensors; the result matches a fresh pack (up to the order
    of the float atomics that sum a Gaussian's gradient over tiles), and an
    input modified in place since the forward forces the fresh pack."""
    n, W, H, eye = CASES[1]
    sc, st = _scene(n, seed=44)
    cam = _cam(W, H, eye)
    pre = _gpu_pre(st, cam)
    w, = gsc.sh2Weight(st["shs"], st["pws"], cam.twc, False, 5)
    g = torch.randn((5, H, W), device="cuda", generator=torch.Generator("cuda").manual_seed(5))

    def fwd_bwd(release):
        out = gsc.splat_weight(H, W, 5, pre["us"], pre["cinv"], st["alphas"], pre["depths"], w,
                               pre["areas"].clone())
        if release:
            gsc.release_packed()
        else:
            assert len(gsc._PACKED) >= 1
        dW, = gsc.splat_weight_B(H, W, 5, pre["us"], pre["cinv"], st["alphas"], pre["depths"], w,
                                 *out[1:], g)
        return out, dW

    _, reused = fwd_bwd(release=False)
    _, fresh = fwd_bwd(release=True)
    assert rel_err(reused[:, 0], np_of(fresh[:, 0]).astype(np.float64)) < 1e-6
    # modify the opacities in place after the forward: the cached records hold
    # the old ones, so the backward must pack again (a fresh pack of the same
    # call, with the cache emptied, is the expected answer)
    out = gsc.splat_weight(H, W, 5, pre["us"], pre["cinv"], st["alphas"], pre["depths"], w,
                           pre["areas"].clone())
    alphas = st["alphas"]
    alphas.mul_(0.5)
    dW, = gsc.splat_weight_B(H, W, 5, pre["us"], pre["cinv"], alphas, pre["depths"], w,
                             *out[1:], g)
    gsc.release_packed()
    dW2, = gsc.splat_weight_B(H, W, 5, pre["us"], pre["cinv"], alphas, pre["depths"], w,
                              *out[1:], g)
    assert rel_err(dW[:, 0], np_of(dW2[:, 0]).astype(np.float64)) < 1e-6
    assert rel_err(dW[:, 0], np_of(fresh[:, 0]).astype(np.float64)) > 0.05


@pytest.mark.parametrize("K", [1, 2, 4, 6, 7, 8])
def test_splat_weight_channel_counts(cuda_ok, K):
    """Compositing and its weights adjoint for every channel count the
    kernels are built for other than the 5 of the benchmark and the 3 of the
    colour path (records take two overlapping Gaussians per step, and the
    adjoint sums their K-vectors in one half-warp transposition padded to a
    power of two): image, contributor indices and weight gradients against
    the oracle."""
    n, W, H, eye = CASES[2]
    sc, st = _scene(n, seed=40 + K)
    cam = _cam(W, H, eye)
    pre = _gpu_pre(st, cam)
    w = torch.rand((n, K), device="cuda", generator=torch.Generator("cuda").manual_seed(K)) - 0.3
    ref = _oracle_splat(H, W, K, {k: v.clone() for k, v in pre.items()}, st["alphas"], w, 0.0)
    layer, contrib, ft, ranges, gsid = gsc.splat_weight(H, W, K, pre["us"], pre["cinv"], st["alphas"],
                                                        pre["depths"], w, pre["areas"])
    assert np.array_equal(np_of(gsid), ref["b"]["gsid"])
    same = np_of(contrib) == ref["contrib"]
    assert same.mean() > 1 - 1e-4
    assert max_abs(np_of(layer)[:, same], ref["out"][:, same]) < IMG_TOL
    g = torch.randn((K, H, W), device="cuda", generator=torch.Generator("cuda").manual_seed(7))
    dW, = gsc.splat_weight_B(H, W, K, pre["us"], pre["cinv"], st["alphas"], pre["depths"], w,
                             contrib, ft, ranges, gsid, g)
    r = orc.draw_backward(H, W, K, np_of(ranges), np_of(gsid), np_of(pre["us"]), np_of(pre["cinv"]),
                          np_of(st["alphas"]), np_of(w), np_of(ft), np_of(contrib), np_of(g))
    assert dW.shape == (n, 1, K)
    assert rel_err(dW[:, 0], r["dfeat"]) < GRAD_REL
