"""Cameras and seeded synthetic palette scenes.

``Camera`` mirrors the object the reference operators read
(gsplat/gausplat_dataset.py:21-33): ``Rcw``/``tcw`` are CUDA float32 tensors,
``twc = -Rcw^-1 tcw``, and ``fx, fy, cx, cy, width, height`` are Python
numbers.  Cameras follow the OpenCV convention the reference kernels assume
(x right, y down, +z forward, gsplatcu/kernel.cu:645-652).

``synthetic_scene`` draws Gaussians from the distributions used for the
benchmark workloads: means from a mixture of 8 isotropic Gaussians
(sigma 0.8) centred uniformly in [-3,3]^3, log-scales ~ N(-4.5, 0.8) per axis,
uniform random unit quaternions (w,x,y,z), opacity sigmoid(N(0,1.5)), a K=5
palette [black, white, 3 uniform colours], and view-dependent palette
weights at SH order 3 -- full [N,16,K] (DC ~ Dirichlet(1), higher orders
~ N(0, 0.05)) or low-rank (DC ~ Dirichlet(1); factors A [N,P,r], B [N,r,Q]
~ N(0, 0.1)).  Full weights are returned band-major as ``shs [N, 16*K]``
(index l*K + k), the layout of gsplat/utils.py:157-158.
"""
import math

import numpy as np
import torch


class Camera:
    def __init__(self, id, width, height, fx, fy, cx, cy, Rcw, tcw, path="", twc=None):
        self.id = id
        self.width = width
        self.height = height
        self.fx = fx
        self.fy = fy
        self.cx = cx
        self.cy = cy
        self.Rcw = Rcw
        self.tcw = tcw
        # camera centre; callers that already have it (e.g. computed on the host)
        # may pass it to skip the device-side 3x3 inverse
        self.twc = -torch.linalg.inv(Rcw) @ tcw if twc is None else twc
        self.path = path

    def to(self, device):
        return Camera(self.id, self.width, self.height, self.fx, self.fy, self.cx, self.cy,
                      self.Rcw.to(device), self.tcw.to(device), self.path)


def look_at(eye, target=(0.0, 0.0, 0.0), width=1920, height=1080, fov_y_deg=60.0,
            up=(0.0, 0.0, 1.0), device="cuda", id=0):
    """Pinhole camera at `eye` looking at `target`; vertical field of view
    `fov_y_deg`, fx = fy = (H/2)/tan(fov/2), principal point at the image centre."""
    eye = np.asarray(eye, np.float64)
    z = np.asarray(target, np.float64) - eye
    z /= np.linalg.norm(z)
    down = -np.asarray(up, np.float64)
    y = down - np.dot(down, z) * z
    if np.linalg.norm(y) < 1e-8:  # looking along the up axis
        y = np.array([0.0, 1.0, 0.0]) - z[1] * z
    y /= np.linalg.norm(y)
    x = np.cross(y, z)
    R = np.stack([x, y, z])  # rows: camera axes in world coordinates
    t = -R @ eye
    f = (height / 2.0) / math.tan(math.radians(fov_y_deg) / 2.0)
    Rcw = torch.tensor(R, dtype=torch.float32, device=device)
    tcw = torch.tensor(t, dtype=torch.float32, device=device)
    return Camera(id, int(width), int(height), float(f), float(f), width / 2.0, height / 2.0,
                  Rcw, tcw)


def sphere_poses(count, radius, seed=0, jitter=0.05):
    """`count` eye positions on a sphere (Fibonacci lattice with seeded jitter)."""
    rng = np.random.default_rng(seed)
    out = []
    golden = math.pi * (3.0 - math.sqrt(5.0))
    for i in range(count):
        zc = 1.0 - 2.0 * (i + 0.5) / count
        r = math.sqrt(max(0.0, 1.0 - zc * zc))
        th = golden * i + rng.normal(0.0, jitter)
        d = np.array([r * math.cos(th), r * math.sin(th), zc]) + rng.normal(0.0, jitter, 3)
        d /= np.linalg.norm(d)
        rad = radius if np.isscalar(radius) else rng.uniform(radius[0], radius[1])
        out.append(d * rad)
    return out


def synthetic_scene(n, seed=0, K=5, mode="full", rank=3, P=5, Q=15, sh_bands=16):
    """Seeded numpy scene (float32).  Returns a dict with pws [N,3], rots [N,4],
    scales [N,3], alphas [N,1], palette [K,3] and either shs [N, sh_bands*K]
    (mode "full") or dc [N,K], A [N,P,rank], B [N,rank,Q] (mode "lowrank")."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-3.0, 3.0, size=(8, 3))
    pick = rng.integers(0, 8, size=n)
    pws = centres[pick] + rng.normal(0.0, 0.8, size=(n, 3))
    scales = np.exp(rng.normal(-4.5, 0.8, size=(n, 3)))
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    alphas = 1.0 / (1.0 + np.exp(-rng.normal(0.0, 1.5, size=(n, 1))))
    palette = np.concatenate([np.zeros((1, 3)), np.ones((1, 3)), rng.uniform(0, 1, (K - 2, 3))])
    out = dict(pws=pws, rots=q, scales=scales, alphas=alphas, palette=palette, K=K, mode=mode)
    dc = rng.dirichlet(np.ones(K), size=n)
    if mode == "full":
        hi = rng.normal(0.0, 0.05, size=(n, sh_bands - 1, K))
        out["shs"] = np.concatenate([dc[:, None, :], hi], axis=1).reshape(n, sh_bands * K)
    elif mode == "lowrank":
        out["dc"] = dc
        out["A"] = rng.normal(0.0, 0.1, size=(n, P, rank))
        out["B"] = rng.normal(0.0, 0.1, size=(n, rank, Q))
        out.update(P=P, Q=Q, rank=rank)
    else:
        raise ValueError(mode)
    for k, v in list(out.items()):
        if isinstance(v, np.ndarray):
            out[k] = v.astype(np.float32)
    return out


def to_torch(scene, device="cuda", param_dtype=torch.float32):
    """Device tensors of a synthetic scene; colour parameters (shs / dc / A / B)
    in `param_dtype` (float32 or bfloat16), geometry in float32."""
    out = {}
    for k, v in scene.items():
        if isinstance(v, np.ndarray):
            t = torch.from_numpy(v).to(device)
            if k in ("shs", "dc", "A", "B"):
                t = t.to(param_dtype)
            out[k] = t.contiguous()
        else:
            out[k] = v
    return out
