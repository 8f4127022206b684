"""numpy front-end of the CPU oracle (gsplat_oracle.cpp) -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker or the timed CPU baseline; the product never does.
Each function mirrors one reference ``gsplatcu`` op (ReparamGS-Palette
``gsplatcu/ext.cpp:125-139``) on numpy arrays, in FP32 (``np.float32``) or in
FP64 (``np.float64``), chosen by the dtype argument.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
TILE = 16
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or (
                os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "gsplat_oracle.cpp"))):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.oracle_bin_count.restype = C.c_int64
        _lib.oracle_get_threads.restype = C.c_int
    return _lib


def set_threads(n):
    lib().oracle_set_threads(int(n))


def get_threads():
    return int(lib().oracle_get_threads())


def _p(a):
    """Raw pointer of a contiguous numpy array (or NULL for None)."""
    if a is None:
        return C.c_void_p(0)
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be contiguous"
    return C.c_void_p(a.ctypes.data)


def _sfx(dt):
    dt = np.dtype(dt)
    if dt == np.float32:
        return "f32", C.c_float
    if dt == np.float64:
        return "f64", C.c_double
    raise TypeError(f"oracle supports float32/float64, got {dt}")


def _arr(x, dt):
    return np.ascontiguousarray(np.asarray(x, dtype=dt))


def grid_dims(H, W):
    return (W + TILE - 1) // TILE, (H + TILE - 1) // TILE


# ------------------------------------------------------------------ geometry
def project(pws, Rcw, tcw, fx, fy, cx, cy, calc_J=False, dtype=np.float32):
    s, cf = _sfx(dtype)
    pws, Rcw, tcw = _arr(pws, dtype), _arr(Rcw, dtype), _arr(tcw, dtype)
    n = pws.shape[0]
    us = np.zeros((n, 2), dtype)
    pcs = np.zeros((n, 3), dtype)
    depths = np.zeros((n,), dtype)
    du = np.zeros((n, 2, 3), dtype) if calc_J else None
    getattr(lib(), f"oracle_project_{s}")(C.c_int64(n), _p(pws), _p(Rcw), _p(tcw), cf(fx), cf(fy),
                                           cf(cx), cf(cy), _p(us), _p(pcs), _p(depths), _p(du))
    return [us, pcs, depths] + ([du] if calc_J else [])


def cov3d(rots, scales, depths, calc_J=False, dtype=np.float32):
    s, _ = _sfx(dtype)
    rots, scales, depths = _arr(rots, dtype), _arr(scales, dtype), _arr(depths, dtype)
    n = rots.shape[0]
    out = np.zeros((n, 6), dtype)
    dr = np.zeros((n, 6, 4), dtype) if calc_J else None
    ds = np.zeros((n, 6, 3), dtype) if calc_J else None
    getattr(lib(), f"oracle_cov3d_{s}")(C.c_int64(n), _p(rots), _p(scales), _p(depths), _p(out),
                                         _p(dr), _p(ds))
    return [out] + ([dr, ds] if calc_J else [])


def tan_fov(width, height, fx, fy, dtype=np.float32):
    """tan of the half field of view as the reference host code computes it
    (gsplatcu/gausplat.cu:357-358): W / (2 fx) in the working precision."""
    dt = np.dtype(dtype).type
    return dt(width) / (dt(2) * dt(fx)), dt(height) / (dt(2) * dt(fy))


def cov2d(cov3ds, pcs, Rcw, depths, fx, fy, width, height, calc_J=False, dtype=np.float32):
    s, cf = _sfx(dtype)
    cov3ds, pcs, Rcw, depths = (_arr(x, dtype) for x in (cov3ds, pcs, Rcw, depths))
    n = pcs.shape[0]
    tx, ty = tan_fov(width, height, fx, fy, dtype)
    out = np.zeros((n, 3), dtype)
    d3 = np.zeros((n, 3, 6), dtype) if calc_J else None
    dp = np.zeros((n, 3, 3), dtype) if calc_J else None
    getattr(lib(), f"oracle_cov2d_{s}")(C.c_int64(n), _p(cov3ds), _p(pcs), _p(Rcw), _p(depths),
                                         cf(fx), cf(fy), cf(tx), cf(ty), _p(out), _p(d3), _p(dp))
    return [out] + ([d3, dp] if calc_J else [])


def inverse_cov2d(cov2ds, depths, calc_J=False, dtype=np.float32):
    """Returns [cinv, areas, (dcinv)]; `depths` (a numpy array of `dtype`) is
    updated in place, as the reference does."""
    s, _ = _sfx(dtype)
    cov2ds = _arr(cov2ds, dtype)
    assert depths.dtype == np.dtype(dtype) and depths.flags["C_CONTIGUOUS"]
    n = cov2ds.shape[0]
    cinv = np.zeros((n, 3), dtype)
    areas = np.zeros((n, 2), np.int32)
    dc = np.zeros((n, 3, 3), dtype) if calc_J else None
    getattr(lib(), f"oracle_inverse_cov2d_{s}")(C.c_int64(n), _p(cov2ds), _p(depths), _p(cinv),
                                                 _p(areas), _p(dc))
    return [cinv, areas] + ([dc] if calc_J else [])


# -------------------------------------------------------- spherical harmonics
def sh2feat(shs, pws, twc, K, calc_J=False, dtype=np.float32, ref_quirk=True):
    """sh2Weight (K palette weights) / sh2Color (K = 3).  shs [N, nb*K] band-major."""
    s, _ = _sfx(dtype)
    shs, pws, twc = _arr(shs, dtype), _arr(pws, dtype), _arr(twc, dtype).reshape(3)
    n = pws.shape[0]
    nb = shs.shape[1] // K
    assert nb in (1, 4, 9, 16)
    feat = np.zeros((n, K), dtype)
    dshs = np.zeros((n, 1, nb), dtype) if calc_J else None
    dpws = np.zeros((n, K, 3), dtype) if calc_J else None
    getattr(lib(), f"oracle_sh2feat_{s}")(C.c_int64(n), _p(shs), _p(pws), _p(twc), C.c_int(nb),
                                           C.c_int(K), _p(feat), _p(dshs), _p(dpws),
                                           C.c_int(1 if ref_quirk else 0))
    return [feat] + ([dshs, dpws] if calc_J else [])


def _lowrank_dims(A, B, K, Q):
    if A.ndim == 2:
        P, rank = A.shape[1], 1
        assert B.ndim == 2 and B.shape[1] == Q
    else:
        P, rank = A.shape[1], A.shape[2]
        assert B.shape[1] == rank and B.shape[2] == Q
    L = P * Q // K
    return P, rank, L


def sh2weight_fast(dc, A, B, pws, twc, K, Q, calc_J=True, dtype=np.float32):
    s, _ = _sfx(dtype)
    dc, A, B, pws = (_arr(x, dtype) for x in (dc, A, B, pws))
    twc = _arr(twc, dtype).reshape(3)
    n = pws.shape[0]
    P, rank, L = _lowrank_dims(A, B, K, Q)
    w = np.zeros((n, K), dtype)
    ddc = np.zeros((n, K), dtype)
    ylm = np.zeros((n, L), dtype)
    getattr(lib(), f"oracle_sh2weight_lowrank_{s}")(
        C.c_int64(n), _p(dc), _p(A), _p(B), _p(pws), _p(twc), C.c_int(K), C.c_int(P), C.c_int(Q),
        C.c_int(rank), C.c_int(L), _p(w), _p(ddc), _p(ylm))
    return [w, ddc, ylm] if calc_J else [w]


def sh2weight_fast_b(A, B, ylm, dw, K, Q, dtype=np.float32):
    s, _ = _sfx(dtype)
    A, B, ylm, dw = (_arr(x, dtype) for x in (A, B, ylm, dw))
    n = A.shape[0]
    P, rank, L = _lowrank_dims(A, B, K, Q)
    dA = np.zeros(A.shape, dtype)
    dB = np.zeros(B.shape, dtype)
    getattr(lib(), f"oracle_sh2weight_lowrank_b_{s}")(
        C.c_int64(n), _p(A), _p(B), _p(ylm), _p(dw), C.c_int(K), C.c_int(P), C.c_int(Q),
        C.c_int(rank), C.c_int(L), _p(dA), _p(dB))
    return [dA, dB]


# ------------------------------------------------------------------- binning
def bin_gaussians(us, areas, depths, H, W):
    """Rects, counts, scan, key emission, stable sort and ranges (FP32, bit-exact
    restatement).  `areas` (int32) and `depths` (float32) are updated in place.
    Returns dict(gsid, ranges, keys, M, counts, rects)."""
    us = _arr(us, np.float32)
    assert areas.dtype == np.int32 and depths.dtype == np.float32
    n = us.shape[0]
    gx, gy = grid_dims(H, W)
    rects = np.zeros((n, 4), np.uint32)
    counts = np.zeros((n,), np.uint32)
    offsets = np.zeros((n,), np.uint32)
    M = int(lib().oracle_bin_count(C.c_int64(n), _p(us), _p(areas), _p(depths), C.c_int(H),
                                   C.c_int(W), _p(rects), _p(counts), _p(offsets)))
    gsid = np.zeros((M,), np.int32)
    keys = np.zeros((M,), np.uint64)
    ranges = np.zeros((gx * gy, 2), np.int32)
    lib().oracle_bin_sort(C.c_int64(n), _p(depths), _p(rects), _p(offsets), C.c_int(H), C.c_int(W),
                          C.c_int64(M), _p(gsid), _p(ranges), _p(keys))
    return dict(gsid=gsid, ranges=ranges, keys=keys, M=M, counts=counts, rects=rects)


# -------------------------------------------------------------- compositing
def draw(H, W, K, ranges, gsid, us, cinv, alphas, feat, tau_init, dtype=np.float32):
    """Forward compositing; returns [out [K,H,W], contrib [H,W], final_tau [H,W]].
    `tau_init` is 0 for splat_weight and 1 for splat_color (the reference's
    initial value kept by empty tiles)."""
    s, _ = _sfx(dtype)
    us, cinv, feat = _arr(us, dtype), _arr(cinv, dtype), _arr(feat, dtype)
    alphas = _arr(alphas, dtype).reshape(-1)
    ranges, gsid = _arr(ranges, np.int32), _arr(gsid, np.int32)
    out = np.zeros((K, H, W), dtype)
    contrib = np.zeros((H, W), np.int32)
    ft = np.full((H, W), tau_init, dtype)
    getattr(lib(), f"oracle_draw_{s}")(C.c_int(H), C.c_int(W), C.c_int(K), _p(ranges), _p(gsid),
                                        _p(us), _p(cinv), _p(alphas), _p(feat), _p(out),
                                        _p(contrib), _p(ft))
    return [out, contrib, ft]


def draw_count(H, W, K, ranges, gsid, us, cinv, alphas, feat, tau_init):
    """draw() in FP32 plus the per-pixel number of blended Gaussians; returns
    [out, contrib, final_tau, blends [H,W] int32]."""
    us, cinv, feat = (_arr(x, np.float32) for x in (us, cinv, feat))
    alphas = _arr(alphas, np.float32).reshape(-1)
    ranges, gsid = _arr(ranges, np.int32), _arr(gsid, np.int32)
    out = np.zeros((K, H, W), np.float32)
    contrib = np.zeros((H, W), np.int32)
    ft = np.full((H, W), tau_init, np.float32)
    blends = np.zeros((H, W), np.int32)
    lib().oracle_draw_count_f32(C.c_int(H), C.c_int(W), C.c_int(K), _p(ranges), _p(gsid), _p(us),
                                _p(cinv), _p(alphas), _p(feat), _p(out), _p(contrib), _p(ft),
                                _p(blends))
    return [out, contrib, ft, blends]


def draw_backward(H, W, K, ranges, gsid, us, cinv, alphas, feat, final_tau, contrib, dout,
                  dT=None, dtype=np.float32):
    """Adjoint of draw(); returns dict(dfeat [N,K], dalpha [N], du [N,2], dconic [N,3])."""
    s, _ = _sfx(dtype)
    us, cinv, feat = _arr(us, dtype), _arr(cinv, dtype), _arr(feat, dtype)
    alphas = _arr(alphas, dtype).reshape(-1)
    final_tau, dout = _arr(final_tau, dtype), _arr(dout, dtype)
    dT = None if dT is None else _arr(dT, dtype)
    ranges, gsid, contrib = _arr(ranges, np.int32), _arr(gsid, np.int32), _arr(contrib, np.int32)
    n = us.shape[0]
    dfeat = np.zeros((n, K), dtype)
    dalpha = np.zeros((n,), dtype)
    du = np.zeros((n, 2), dtype)
    dq = np.zeros((n, 3), dtype)
    getattr(lib(), f"oracle_draw_backward_{s}")(
        C.c_int(H), C.c_int(W), C.c_int(K), _p(ranges), _p(gsid), _p(us), _p(cinv), _p(alphas),
        _p(feat), _p(final_tau), _p(contrib), _p(dout), _p(dT), _p(dfeat), _p(dalpha), _p(du), _p(dq))
    return dict(dfeat=dfeat, dalpha=dalpha, du=du, dconic=dq)


def lab2rgb(lab):
    lab = _arr(lab, np.float32)
    _, H, W = lab.shape
    out = np.zeros_like(lab)
    lib().oracle_lab2rgb(C.c_int(H), C.c_int(W), _p(lab), _p(out))
    return out


# ---------------------------------------------------- composite pipelines
def splat(H, W, K, us, cinv, alphas, depths, feat, areas, tau_init):
    """The reference's splat_weight / splat_color host sequence
    (gsplatcu/gausplat.cu:161-249): binning then compositing, FP32.  depths and
    areas are updated in place.  Returns [out, contrib, final_tau, ranges, gsid]."""
    b = bin_gaussians(us, areas, depths, H, W)
    out, contrib, ft = draw(H, W, K, b["ranges"], b["gsid"], us, cinv, alphas, feat, tau_init)
    return [out, contrib, ft, b["ranges"], b["gsid"]]


def camera_arrays(cam, dtype):
    """(Rcw [3,3], tcw [3], twc [3]) of a camera-like object as numpy arrays."""
    def npy(x):
        if hasattr(x, "detach"):
            x = x.detach().cpu().numpy()
        return np.asarray(x, dtype=np.float64)
    Rcw, tcw = npy(cam.Rcw), npy(cam.tcw).reshape(3)
    twc = -np.linalg.inv(Rcw) @ tcw
    return Rcw.astype(dtype), tcw.astype(dtype), twc.astype(dtype)


def preprocess(pws, rots, scales, cam, dtype=np.float32):
    """project -> cov3D -> cov2D -> inverse, as WeightGSFunctionTest does
    (gsplat/gsmodel.py:107-115).  Returns dict of per-Gaussian arrays."""
    Rcw, tcw, twc = camera_arrays(cam, dtype)
    us, pcs, depths = project(pws, Rcw, tcw, cam.fx, cam.fy, cam.cx, cam.cy, False, dtype)
    c3, = cov3d(rots, scales, depths, False, dtype)
    c2, = cov2d(c3, pcs, Rcw, depths, cam.fx, cam.fy, cam.width, cam.height, False, dtype)
    cinv, areas = inverse_cov2d(c2, depths, False, dtype)
    return dict(us=us, pcs=pcs, depths=depths, cov3d=c3, cov2d=c2, cinv=cinv, areas=areas,
                twc=twc, Rcw=Rcw, tcw=tcw)


def render_weights(pws, rots, scales, alphas, weights, cam, dtype=np.float32, lists=None):
    """Full forward of the palette-weight path.  Geometry and compositing run in
    `dtype`; binning always runs on the FP32 image of the projected values (it
    is integer work defined on FP32 inputs), unless `lists` = (ranges, gsid)
    supplies the tile lists to use.  Returns dict(layer, contrib, final_tau,
    ranges, gsid, pre)."""
    pre = preprocess(pws, rots, scales, cam, dtype)
    K = weights.shape[1]
    H, W = int(cam.height), int(cam.width)
    if lists is None:
        d32 = pre["depths"].astype(np.float32)
        a32 = pre["areas"].copy()
        b = bin_gaussians(pre["us"].astype(np.float32), a32, d32, H, W)
        ranges, gsid = b["ranges"], b["gsid"]
    else:
        ranges, gsid = lists
    out, contrib, ft = draw(H, W, K, ranges, gsid, pre["us"], pre["cinv"], alphas, weights, 0.0, dtype)
    return dict(layer=out, contrib=contrib, final_tau=ft, ranges=ranges, gsid=gsid, pre=pre)


def render_weights_backward(pws, rots, scales, alphas, cam, twc, K, shs=None, lowrank=None,
                            lists=None, dout=None, dT=None, dtype=np.float64):
    """Gradients of sum(dout * layer) + sum(dT * final_tau) with respect to
    every input of the palette-weight path, by the reference's own chain rule
    (vanilla_3dgs/gsplat/gsmodel.py:65-75: per-operator Jacobians composed
    with the compositing adjoint), with the weights' true view-direction
    derivative.  Weights come from full SH ``shs [N,16K]`` or from
    ``lowrank = (dc [N,K], A [N,P,r] or [N,P], B [N,r,Q] or [N,Q])``.
    `lists` = (ranges, gsid) fixes the tile lists.  Returns a dict of
    gradients plus the forward (layer, final_tau, contrib)."""
    dt = np.dtype(dtype).type
    Rcw, tcw, _ = camera_arrays(cam, dtype)
    twc = _arr(twc, dtype).reshape(3)
    H, W = int(cam.height), int(cam.width)
    us, pcs, depths, du_dpc = project(pws, Rcw, tcw, cam.fx, cam.fy, cam.cx, cam.cy, True, dtype)
    c3, dc3_dq, dc3_ds = cov3d(rots, scales, depths, True, dtype)
    c2, dc2_dc3, dc2_dpc = cov2d(c3, pcs, Rcw, depths, cam.fx, cam.fy, W, H, True, dtype)
    cinv, areas, dci_dc2 = inverse_cov2d(c2, depths, True, dtype)
    if lowrank is None:
        shs_eff = _arr(shs, dtype)
    else:  # C = A B; band l+1, channel k of the weights is C[g], g = l*K + k
        dc, A, B = (_arr(x, dtype) for x in lowrank)
        A3 = A[:, :, None] if A.ndim == 2 else A
        B3 = B[:, None, :] if B.ndim == 2 else B
        Cm = np.einsum("npr,nrq->npq", A3, B3).reshape(A.shape[0], -1)
        shs_eff = np.concatenate([dc, Cm], axis=1)
    feat, Y, dw_dpw = sh2feat(shs_eff, pws, twc, K, True, dtype, ref_quirk=False)
    if lists is None:
        b = bin_gaussians(us.astype(np.float32), areas.copy(), depths.astype(np.float32), H, W)
        lists = (b["ranges"], b["gsid"])
    ranges, gsid = lists
    layer, contrib, ft = draw(H, W, K, ranges, gsid, us, cinv, alphas, feat, 0.0, dtype)
    dout = np.zeros((K, H, W), dtype) if dout is None else _arr(dout, dtype)
    g = draw_backward(H, W, K, ranges, gsid, us, cinv, alphas, feat, ft, contrib, dout, dT, dtype)
    live = (np.any(g["dfeat"] != 0, axis=1) | np.any(g["du"] != 0, axis=1) |
            np.any(g["dconic"] != 0, axis=1))
    z = lambda a: np.where(live.reshape((-1,) + (1,) * (a.ndim - 1)), a, dt(0))
    dc2 = np.einsum("nj,nji->ni", g["dconic"], z(dci_dc2))
    dc3 = np.einsum("nj,nji->ni", dc2, z(dc2_dc3))
    dpc = np.einsum("nj,nji->ni", g["du"], z(du_dpc)) + np.einsum("nj,nji->ni", dc2, z(dc2_dpc))
    out = dict(layer=layer, final_tau=ft, contrib=contrib, dalphas=g["dalpha"],
               drots=np.einsum("nj,nji->ni", dc3, z(dc3_dq)),
               dscales=np.einsum("nj,nji->ni", dc3, z(dc3_ds)),
               dpws=dpc @ Rcw + np.einsum("nk,nki->ni", g["dfeat"], z(dw_dpw)),
               dfeat=g["dfeat"])
    dshs = (g["dfeat"][:, None, :] * Y.reshape(Y.shape[0], -1)[:, :, None]).reshape(len(feat), -1)
    if lowrank is None:
        out["dshs"] = dshs
    else:
        dC = dshs[:, K:].reshape(Cm.shape[0], A3.shape[1], B3.shape[2])
        out["ddc"] = dshs[:, :K]
        out["dA"] = np.einsum("npq,nrq->npr", dC, B3).reshape(A.shape)
        out["dB"] = np.einsum("npq,npr->nrq", dC, A3).reshape(B.shape)
    return out


# ------------------------------------------------------------- loss side
def _softplus(x):
    return np.where(x > 20.0, x, np.log1p(np.exp(np.minimum(x, 20.0))))


def _sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def palette_geo_loss(layer, target, chroma, clamp=True, lambda_pos=0.5, kind="mse", tau=1e-9,
                     eps=1e-12):
    """The finetune step's loss on the rendered palette weights (finetune.py:
    356-389 with gsplat/gsmodel.py:219-285 for the target), in FP64:

      W_bary = barycentric target of the colour image `target` [3,H,W] in the
               palette {black, white, chroma [Kc,3]}: for each tetrahedron
               (black, white, c_i, c_{i+1}) the barycentric coordinates of the
               pixel colour, their softplus-normalised projection's
               reconstruction error, and a softmax over the tetrahedra (tau)
               weighting the raw coordinates;
      clamp:   W_bary <- max(W_bary, 0) / max(sum_k max(W_bary, 0), 1e-8);
      loss   = mean((layer - W_bary)^2) (kind "mse") or mean(|layer - W_bary|)
               ("l1"), plus lambda_pos * mean(relu(-layer)).

    Returns dict(loss, target_weights [K,H,W], dlayer [K,H,W], dchroma [Kc,3])
    with the gradients of the loss (the target depends on the palette)."""
    layer = np.asarray(layer, np.float64)
    C = np.asarray(target, np.float64).reshape(3, -1).T  # [N,3]
    P = np.asarray(chroma, np.float64)
    Kc = P.shape[0]
    K = Kc + 2
    N = C.shape[0]
    Wt = layer.reshape(K, -1).T  # [N,K]
    e = np.ones(3)
    raws, errs, cache = [], [], []
    for i in range(Kc):
        j = (i + 1) % Kc
        A = np.stack([e, P[i], P[j]], axis=1)  # columns: white-black, P_i, P_j
        a = A
        det = (a[0, 0] * (a[1, 1] * a[2, 2] - a[1, 2] * a[2, 1])
               - a[0, 1] * (a[1, 0] * a[2, 2] - a[1, 2] * a[2, 0])
               + a[0, 2] * (a[1, 0] * a[2, 1] - a[1, 1] * a[2, 0]))
        adj = np.array([
            [a[1, 1] * a[2, 2] - a[1, 2] * a[2, 1], -(a[0, 1] * a[2, 2] - a[0, 2] * a[2, 1]),
             a[0, 1] * a[1, 2] - a[0, 2] * a[1, 1]],
            [-(a[1, 0] * a[2, 2] - a[1, 2] * a[2, 0]), a[0, 0] * a[2, 2] - a[0, 2] * a[2, 0],
             -(a[0, 0] * a[1, 2] - a[0, 2] * a[1, 0])],
            [a[1, 0] * a[2, 1] - a[1, 1] * a[2, 0], -(a[0, 0] * a[2, 1] - a[0, 1] * a[2, 0]),
             a[0, 0] * a[1, 1] - a[0, 1] * a[1, 0]]])
        dinv = 1.0 / (det + eps)
        co = (C @ adj.T) * dinv  # [N,3]: beta, gamma, delta
        beta, gamma, delta = co[:, 0], co[:, 1], co[:, 2]
        alpha = 1.0 - beta - gamma - delta
        raw = np.zeros((N, K))
        raw[:, 0] = alpha
        raw[:, 1] = beta
        raw[:, i + 2] += gamma
        raw[:, j + 2] += delta
        x = np.stack([alpha, beta, gamma, delta], 1)
        sp = _softplus(x)
        den = sp.sum(1) + eps
        pr = sp / den[:, None]
        recon = pr[:, 1:2] * e + pr[:, 2:3] * P[i] + pr[:, 3:4] * P[j]
        err = ((recon - C) ** 2).sum(1)
        raws.append(raw)
        errs.append(err)
        cache.append((i, j, A, co, x, sp, den, pr, recon))
    E = np.stack(errs, 1)  # [N,Kc]
    lg = -E / tau
    lg = lg - lg.max(1, keepdims=True)
    pe = np.exp(lg)
    probs = pe / pe.sum(1, keepdims=True)
    R = np.stack(raws, 1)  # [N,Kc,K]
    Wb = (probs[:, :, None] * R).sum(1)  # [N,K]
    if clamp:
        m = np.maximum(Wb, 0.0)
        s_raw = m.sum(1)
        s = np.maximum(s_raw, 1e-8)
        Wc = m / s[:, None]
    else:
        Wc = Wb
    diff = Wt - Wc
    n_el = K * N
    if kind == "mse":
        loss = (diff ** 2).sum() / n_el
        g = 2.0 * diff / n_el
    else:
        loss = np.abs(diff).sum() / n_el
        g = np.sign(diff) / n_el
    loss += lambda_pos * np.maximum(-Wt, 0.0).sum() / n_el
    dWt = g + lambda_pos * np.where(Wt < 0, -1.0, 0.0) / n_el
    gW = -g  # dL / d (clamped) target
    if clamp:
        gm = np.where(s_raw[:, None] > 1e-8,
                      gW / s[:, None] - (gW * m).sum(1, keepdims=True) / (s * s)[:, None],
                      gW / s[:, None])
        gWb = gm * (Wb > 0)
    else:
        gWb = gW
    # W = sum_i probs_i raw_i
    graw = probs[:, :, None] * gWb[:, None, :]  # [N,Kc,K]
    gprob = (R * gWb[:, None, :]).sum(2)  # [N,Kc]
    glog = probs * (gprob - (probs * gprob).sum(1, keepdims=True))
    gerr = -glog / tau
    dP = np.zeros_like(P)
    for (i, j, A, co, x, sp, den, pr, recon), ii in zip(cache, range(Kc)):
        gr = graw[:, ii, :]
        g_alpha, g_beta = gr[:, 0], gr[:, 1]
        g_gamma, g_delta = gr[:, i + 2], gr[:, j + 2]
        # error path: err = |recon - C|^2
        ge = gerr[:, ii]
        grec = 2.0 * (recon - C) * ge[:, None]  # [N,3]
        dP[i] += (grec * pr[:, 2:3]).sum(0)
        dP[j] += (grec * pr[:, 3:4]).sum(0)
        gpr = np.stack([np.zeros(N), grec.sum(1), (grec * P[i]).sum(1), (grec * P[j]).sum(1)], 1)
        gsp = gpr / den[:, None] - (gpr * sp).sum(1, keepdims=True) / (den * den)[:, None]
        gx = gsp * np.where(x > 20.0, 1.0, _sigmoid(np.minimum(x, 20.0)))
        g_alpha = g_alpha + gx[:, 0]
        g_beta = g_beta + gx[:, 1]
        g_gamma = g_gamma + gx[:, 2]
        g_delta = g_delta + gx[:, 3]
        gco = np.stack([g_beta - g_alpha, g_gamma - g_alpha, g_delta - g_alpha], 1)  # [N,3]
        # coords = A^-1 C: d coords = -A^-1 (dA) coords, dA columns 1, 2 = dP_i, dP_j
        Ainv_T_g = gco @ np.linalg.inv(A)  # rows: (A^-T g)^T
        dP[i] -= (Ainv_T_g * co[:, 1:2]).sum(0)
        dP[j] -= (Ainv_T_g * co[:, 2:3]).sum(0)
    return dict(loss=float(loss), target_weights=Wc.T.reshape(layer.shape),
                dlayer=dWt.T.reshape(layer.shape), dchroma=dP)


def ssim_window(window_size=11, sigma=1.5):
    """The SSIM window as the reference builds it (vanilla_3dgs/gsplat/
    pytorch_ssim.py:12-23), in FP32: g[x] = exp(-(x - size//2)^2 / (2 sigma^2))
    rounded to FP32 and divided by its FP32 sum, the 2-D window the FP32
    outer product g g^T.  Returns (g [size], window [size,size]) as float64
    arrays holding those FP32 values."""
    g = np.array([np.exp(-float(x - window_size // 2) ** 2 / (2.0 * sigma * sigma))
                  for x in range(window_size)], dtype=np.float32)
    g = (g / np.float32(g.astype(np.float64).sum())).astype(np.float32)
    return g.astype(np.float64), np.outer(g, g).astype(np.float32).astype(np.float64)


def _filter(a, w2):
    """Per-channel 2-D filtering of a [C,H,W] with the window w2 (zero padding of
    size//2 on every side, output the input's size): F.conv2d with groups=C and
    padding=window//2 (pytorch_ssim.py:27-39).  w2 is point-symmetric, so the
    same call is its own adjoint."""
    r = w2.shape[0] // 2
    C_, H, W = a.shape
    p = np.zeros((C_, H + 2 * r, W + 2 * r))
    p[:, r:r + H, r:r + W] = a
    out = np.zeros_like(a, dtype=np.float64)
    for i in range(w2.shape[0]):
        for j in range(w2.shape[1]):
            out += w2[i, j] * p[:, i:i + H, j:j + W]
    return out


def l1_ssim_loss(image, target, lambda_ssim=0.2, range_=1.0, window_size=11):
    """gau_loss (vanilla_3dgs/gsplat/pytorch_ssim.py:26-67) in FP64:
    loss = (1 - lambda) mean|x - y| + lambda (1 - mean SSIM(x, y)), the SSIM map
    from the 11x11 sigma 1.5 window with C1 = (0.01 range)^2, C2 = (0.03 range)^2.
    Returns dict(loss, l1, ssim, dimage) with dimage = d loss / d image.

    The gradient: with mu_x = G*x, s_xx = G*x^2, s_xy = G*(xy) and the SSIM map
    S = A1 A2 / (B1 B2), A1 = 2 mu_x mu_y + C1, A2 = 2 (s_xy - mu_x mu_y) + C2,
    B1 = mu_x^2 + mu_y^2 + C1, B2 = s_xx - mu_x^2 + s_yy - mu_y^2 + C2,
      dS/dmu_x = 2 mu_y (A2 - A1) / (B1 B2) - 2 mu_x S (1/B1 - 1/B2),
      dS/ds_xx = -S / B2,   dS/ds_xy = 2 A1 / (B1 B2),
    and d sum_p S(p) / dx(q) = (G*dS/dmu_x)(q) + 2 x(q) (G*dS/ds_xx)(q) +
    y(q) (G*dS/ds_xy)(q) (the window is point-symmetric, so its adjoint under
    zero padding is the same filter).  The window holds the reference's FP32
    values, so the FP64 result equals the reference module run in FP64."""
    x = np.asarray(image, np.float64)
    y = np.asarray(target, np.float64)
    _, g = ssim_window(window_size)
    C1, C2 = (0.01 * range_) ** 2, (0.03 * range_) ** 2
    mx, my = _filter(x, g), _filter(y, g)
    sxx, syy, sxy = _filter(x * x, g), _filter(y * y, g), _filter(x * y, g)
    A1 = 2 * mx * my + C1
    A2 = 2 * (sxy - mx * my) + C2
    B1 = mx * mx + my * my + C1
    B2 = (sxx - mx * mx) + (syy - my * my) + C2
    S = A1 * A2 / (B1 * B2)
    n = x.size
    l1 = np.abs(x - y).sum() / n
    ssim = S.sum() / n
    dmx = 2 * my * (A2 - A1) / (B1 * B2) - 2 * mx * S * (1 / B1 - 1 / B2)
    dsxx = -S / B2
    dsxy = 2 * A1 / (B1 * B2)
    dS = _filter(dmx, g) + 2 * x * _filter(dsxx, g) + y * _filter(dsxy, g)
    dimage = (1 - lambda_ssim) * np.sign(x - y) / n - lambda_ssim * dS / n
    return dict(loss=float((1 - lambda_ssim) * l1 + lambda_ssim * (1 - ssim)), l1=float(l1),
                ssim=float(ssim), dimage=dimage)


def palette_l1_ssim_loss(layer, palette, target, lambda_ssim=0.2, lambda_pos=0.5, range_=1.0):
    """The differentiation workload's finetune loss on the palette colour image
    img = sum_k palette[k] layer_k, in FP64: gau_loss(img, target) plus
    lambda_pos mean(relu(-layer)) (finetune.py:375,381).  Returns dict(loss, l1,
    ssim, penalty (lambda_pos-scaled), image [3,H,W], dlayer [K,H,W],
    dpalette [K,3])."""
    layer = np.asarray(layer, np.float64)
    P = np.asarray(palette, np.float64)
    img = np.einsum("kc,khw->chw", P, layer)
    r = l1_ssim_loss(img, target, lambda_ssim, range_)
    dimg = r["dimage"]
    pen = lambda_pos * np.maximum(-layer, 0.0).sum() / layer.size
    dlayer = np.einsum("kc,chw->khw", P, dimg) - lambda_pos * (layer < 0) / layer.size
    dpal = np.einsum("khw,chw->kc", layer, dimg)
    return dict(loss=r["loss"] + float(pen), l1=r["l1"], ssim=r["ssim"], penalty=float(pen),
                image=img, dlayer=dlayer, dpalette=dpal)
