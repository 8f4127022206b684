"""CPU check of the oracle's whole-path chain rule (oracle.render_weights_backward)
against central finite differences of its own FP64 forward, with the tile
lists held fixed.  This pins the FP64 gradients that the fused GPU backward is
compared with."""
import numpy as np
import pytest

from oracle import oracle as orc
from palette_b200.scene import look_at, synthetic_scene


def _setup(mode, rank=1, n=300, W=48, H=40, seed=7):
    sc = synthetic_scene(n, seed=seed, mode=mode, rank=rank)
    cam = look_at((0.5, -6.0, 0.8), width=W, height=H, device="cpu")
    twc = orc.camera_arrays(cam, np.float64)[2]
    rng = np.random.default_rng(seed)
    dout = rng.standard_normal((5, H, W))
    dT = rng.standard_normal((H, W))
    return sc, cam, twc, dout, dT


def _params(sc, mode):
    p = dict(pws=sc["pws"], rots=sc["rots"], scales=sc["scales"], alphas=sc["alphas"])
    if mode == "full":
        p["shs"] = sc["shs"]
    else:
        p.update(dc=sc["dc"], A=sc["A"], B=sc["B"])
    return {k: np.asarray(v, np.float64).copy() for k, v in p.items()}


def _run(p, cam, twc, mode, lists, dout, dT):
    lr = None if mode == "full" else (p["dc"], p["A"], p["B"])
    return orc.render_weights_backward(p["pws"], p["rots"], p["scales"], p["alphas"], cam, twc, 5,
                                       shs=p.get("shs"), lowrank=lr, lists=lists, dout=dout, dT=dT)


def _loss(r, dout, dT):
    return float(np.sum(dout * r["layer"]) + np.sum(dT * r["final_tau"]))


def _lists(p, cam):
    pre = orc.preprocess(p["pws"].astype(np.float32), p["rots"].astype(np.float32),
                         p["scales"].astype(np.float32), cam, np.float32)
    b = orc.bin_gaussians(pre["us"], pre["areas"], pre["depths"], int(cam.height), int(cam.width))
    return b["ranges"], b["gsid"]


@pytest.mark.parametrize("mode,rank", [("full", 0), ("lowrank", 1), ("lowrank", 3)])
def test_chain_rule_matches_finite_differences(mode, rank):
    sc, cam, twc, dout, dT = _setup(mode, rank=max(rank, 1))
    p = _params(sc, mode)
    lists = _lists(p, cam)
    r0 = _run(p, cam, twc, mode, lists, dout, dT)
    live = np.flatnonzero(np.any(r0["dfeat"] != 0, axis=1))
    assert live.size > 20
    # Gaussians well inside the frustum: the reference clamps x/z, y/z at
    # 1.3 tan(fov/2) and does not differentiate the clamp.
    Rcw, tcw, _ = orc.camera_arrays(cam, np.float64)
    pc = p["pws"] @ Rcw.T + tcw
    tx, ty = orc.tan_fov(cam.width, cam.height, cam.fx, cam.fy, np.float64)
    inside = (np.abs(pc[:, 0] / pc[:, 2]) < 1.2 * tx) & (np.abs(pc[:, 1] / pc[:, 2]) < 1.2 * ty)
    live = live[inside[live]]
    rng = np.random.default_rng(1)
    pick = rng.choice(live, size=min(12, live.size), replace=False)
    grads = dict(pws="dpws", rots="drots", scales="dscales", alphas="dalphas")
    grads.update(shs="dshs") if mode == "full" else grads.update(dc="ddc", A="dA", B="dB")
    checked = 0
    for name, gname in grads.items():
        g = r0[gname].reshape(p[name].shape[0], -1)
        for i in pick:
            cols = range(g.shape[1]) if g.shape[1] <= 4 else rng.choice(g.shape[1], 4, replace=False)
            for j in cols:
                eps = 1e-6 * max(1.0, abs(p[name].reshape(len(g), -1)[i, j]))
                vals = []
                for s in (1, -1):
                    q = {k: v.copy() for k, v in p.items()}
                    q[name].reshape(len(g), -1)[i, j] += s * eps
                    vals.append(_loss(_run(q, cam, twc, mode, lists, dout, dT), dout, dT))
                fd = (vals[0] - vals[1]) / (2 * eps)
                scale = max(1e-3, np.abs(g).max())
                assert abs(fd - g[i, j]) <= 1e-5 * scale + 1e-6 * abs(fd), (name, i, j, fd, g[i, j])
                checked += 1
    assert checked > 100


def test_chain_rule_sees_the_view_direction_term():
    """Dropping the weights' view-direction derivative breaks the FD check:
    the test above is sensitive to it (a mistake planted in the oracle)."""
    sc, cam, twc, dout, dT = _setup("full")
    p = _params(sc, "full")
    lists = _lists(p, cam)
    r = _run(p, cam, twc, "full", lists, dout, dT)
    _, _, dw = orc.sh2feat(p["shs"], p["pws"], twc, 5, True, np.float64, ref_quirk=False)
    view = np.einsum("nk,nki->ni", r["dfeat"], dw)
    i = int(np.argmax(np.abs(view).max(axis=1)))
    j = int(np.argmax(np.abs(view[i])))
    vals = []
    for s in (1, -1):
        q = {k: v.copy() for k, v in p.items()}
        q["pws"][i, j] += s * 1e-6
        vals.append(_loss(_run(q, cam, twc, "full", lists, dout, dT), dout, dT))
    fd = (vals[0] - vals[1]) / 2e-6
    scale = np.abs(r["dpws"]).max()
    assert abs(fd - r["dpws"][i, j]) <= 1e-5 * scale
    assert abs(fd - (r["dpws"][i, j] - view[i, j])) > 1e-3 * scale
