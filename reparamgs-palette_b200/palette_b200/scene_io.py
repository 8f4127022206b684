"""Finetuned palette scenes on disk, and their upload into HBM.

Formats (those ReparamGS-Palette writes):

* the finetune checkpoint ``.npy`` (finetune.py:440-468): a pickled dict with
  ``palette`` [K,3] (black, white, chromatic), ``pw`` [N,3], ``rot`` [N,4]
  (w,x,y,z), ``scale`` [N,3] (linear), ``alpha`` [N] or [N,1] (after the
  sigmoid), and either ``shs_w`` [N,16K] (full weights, band-major) or
  ``low_shs_w`` [N,K] + ``high_shs_A`` [N,P] + ``high_shs_B`` [N,Q] with
  ``reshape_P``/``reshape_Q`` (rank-1 low-rank weights).  Loading it unpickles
  the file: only load checkpoints you trust.
* the geometry-only ``.pply`` + weight sidecar ``.gswp`` pair
  (convert_npy_ply/palette_npy_to_pply.py): a binary little-endian PLY with
  per-vertex float x, y, z, scale_0..2 (log of the linear scale), opacity
  (logit of alpha), rot_0..3; and a 32-byte header (``GSWP``, version 1, N,
  splat_dim, num_sh, low_rank, P, Q, all u32 after the magic) followed by the
  palette [splat_dim,3], the DC weights [N,splat_dim] and either the
  rest-band weights [N,splat_dim*(num_sh-1)] or the factors A [N,P], B [N,Q],
  all float32.

``to_scene`` uploads a checkpoint dict into a ``palette_b200.serve.Scene``
(geometry FP32; weights FP32 or BF16), the form the serving loop and
``render_palette`` use.
"""
import struct

import numpy as np
import torch

GSWP_MAGIC = b"GSWP"
GSWP_VERSION = 1
_PLY_FIELDS = ("x", "y", "z", "scale_0", "scale_1", "scale_2", "opacity", "rot_0", "rot_1",
               "rot_2", "rot_3")


def _f32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float32))


def validate(d):
    """Check a checkpoint dict's keys and shapes; returns (N, splat_dim,
    num_sh, low_rank)."""
    for k in ("pw", "rot", "scale", "alpha", "palette"):
        if k not in d:
            raise KeyError(f"scene is missing {k!r}")
    pal = np.asarray(d["palette"])
    if pal.ndim != 2 or pal.shape[1] != 3:
        raise ValueError(f"palette has shape {pal.shape}; expected (splat_dim, 3)")
    K = pal.shape[0]
    N = np.asarray(d["pw"]).shape[0]
    for k, shape in (("pw", (N, 3)), ("rot", (N, 4)), ("scale", (N, 3))):
        if np.asarray(d[k]).shape != shape:
            raise ValueError(f"{k} has shape {np.asarray(d[k]).shape}; expected {shape}")
    if np.asarray(d["alpha"]).reshape(-1).shape != (N,):
        raise ValueError("alpha must hold N values")
    low_rank = bool(d.get("low_rank", False))
    if low_rank:
        P, Q = int(d["reshape_P"]), int(d["reshape_Q"])
        if np.asarray(d["low_shs_w"]).shape != (N, K):
            raise ValueError("low_shs_w must be (N, splat_dim)")
        if np.asarray(d["high_shs_A"]).shape != (N, P) or np.asarray(d["high_shs_B"]).shape != (N, Q):
            raise ValueError("high_shs_A / high_shs_B must be (N, P) / (N, Q)")
        if (P * Q) % K:
            raise ValueError("P*Q must be a multiple of splat_dim")
        num_sh = P * Q // K + 1
    else:
        shs = np.asarray(d["shs_w"])
        if shs.ndim != 2 or shs.shape[0] != N or shs.shape[1] % K:
            raise ValueError("shs_w must be (N, splat_dim * num_sh)")
        num_sh = shs.shape[1] // K
    return N, K, num_sh, low_rank


def load_checkpoint(path):
    """The finetune checkpoint dict of a ``.npy`` (unpickles: trusted files only)."""
    obj = np.load(path, allow_pickle=True)
    if not (isinstance(obj, np.ndarray) and obj.dtype == object and obj.ndim == 0):
        raise ValueError(f"{path}: expected a pickled dict")
    d = obj.item()
    if not isinstance(d, dict):
        raise ValueError(f"{path}: expected a pickled dict, got {type(d)}")
    validate(d)
    return d


def save_checkpoint(path, d):
    validate(d)
    np.save(path, d, allow_pickle=True)


def write_pply(path, d):
    N = np.asarray(d["pw"]).shape[0]
    pw, rot = _f32(d["pw"]), _f32(d["rot"])
    log_scale = np.log(np.clip(_f32(d["scale"]), 1e-20, None)).astype(np.float32)
    a = np.clip(_f32(d["alpha"]).reshape(-1), 1e-6, 1 - 1e-6)
    opacity = np.log(a / (1 - a)).astype(np.float32)
    rec = np.empty(N, dtype=[(f, "<f4") for f in _PLY_FIELDS])
    for c, f in enumerate(("x", "y", "z")):
        rec[f] = pw[:, c]
    for c in range(3):
        rec[f"scale_{c}"] = log_scale[:, c]
    rec["opacity"] = opacity
    for c in range(4):
        rec[f"rot_{c}"] = rot[:, c]
    head = ["ply", "format binary_little_endian 1.0",
            "comment palette-based 3DGS - geometry only; pair with .gswp sidecar",
            f"element vertex {N}"] + [f"property float {f}" for f in _PLY_FIELDS] + ["end_header", ""]
    with open(path, "wb") as fh:
        fh.write("\n".join(head).encode("ascii"))
        fh.write(rec.tobytes())


def read_pply(path):
    """Geometry of a ``.pply``: dict(pw, rot, scale (linear), alpha (sigmoid))."""
    with open(path, "rb") as fh:
        data = fh.read()
    end = data.find(b"end_header\n")
    if not data.startswith(b"ply\n") or end < 0:
        raise ValueError(f"{path}: not a PLY file")
    header = data[:end].decode("ascii").splitlines()
    if "format binary_little_endian 1.0" not in header:
        raise ValueError(f"{path}: only binary little-endian PLY is read")
    n, props = None, []
    for line in header:
        t = line.split()
        if t[:2] == ["element", "vertex"]:
            n = int(t[2])
        elif t[:1] == ["property"]:
            if t[1] != "float":
                raise ValueError(f"{path}: property {t[-1]} is not float")
            props.append(t[2])
    missing = [f for f in _PLY_FIELDS if f not in props]
    if n is None or missing:
        raise ValueError(f"{path}: missing vertex count or properties {missing}")
    rec = np.frombuffer(data, dtype=[(f, "<f4") for f in props], count=n,
                        offset=end + len(b"end_header\n"))
    pw = np.stack([rec["x"], rec["y"], rec["z"]], 1)
    scale = np.exp(np.stack([rec[f"scale_{c}"] for c in range(3)], 1))
    alpha = 1.0 / (1.0 + np.exp(-rec["opacity"].astype(np.float64)))
    rot = np.stack([rec[f"rot_{c}"] for c in range(4)], 1)
    return dict(pw=_f32(pw), rot=_f32(rot), scale=_f32(scale), alpha=_f32(alpha))


def write_gswp(path, d):
    N, K, num_sh, low_rank = validate(d)
    P = int(d["reshape_P"]) if low_rank else 0
    Q = int(d["reshape_Q"]) if low_rank else 0
    with open(path, "wb") as fh:
        fh.write(GSWP_MAGIC + struct.pack("<7I", GSWP_VERSION, N, K, num_sh, int(low_rank), P, Q))
        fh.write(_f32(d["palette"]).tobytes())
        if low_rank:
            fh.write(_f32(d["low_shs_w"]).tobytes())
            fh.write(_f32(d["high_shs_A"]).tobytes())
            fh.write(_f32(d["high_shs_B"]).tobytes())
        else:
            shs = _f32(d["shs_w"])
            fh.write(np.ascontiguousarray(shs[:, :K]).tobytes())
            fh.write(np.ascontiguousarray(shs[:, K:]).tobytes())


def read_gswp(path):
    """Palette and weights of a ``.gswp`` sidecar, as checkpoint-dict keys."""
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) < 32 or data[:4] != GSWP_MAGIC:
        raise ValueError(f"{path}: not a GSWP file")
    ver, N, K, num_sh, low_rank, P, Q = struct.unpack_from("<7I", data, 4)
    if ver != GSWP_VERSION:
        raise ValueError(f"{path}: GSWP version {ver} is not supported")
    off = 32

    def take(count, shape):
        nonlocal off
        a = np.frombuffer(data, dtype="<f4", count=count, offset=off).reshape(shape)
        off += 4 * count
        return a.copy()
    d = dict(palette=take(K * 3, (K, 3)))
    low = take(N * K, (N, K))
    if low_rank:
        if P * Q != K * (num_sh - 1):
            raise ValueError(f"{path}: P*Q != splat_dim*(num_sh-1)")
        d.update(low_rank=True, low_shs_w=low, high_shs_A=take(N * P, (N, P)),
                 high_shs_B=take(N * Q, (N, Q)), reshape_P=P, reshape_Q=Q)
    else:
        high = take(N * K * (num_sh - 1), (N, K * (num_sh - 1)))
        d.update(low_rank=False, shs_w=np.concatenate([low, high], 1))
    if off != len(data):
        raise ValueError(f"{path}: {len(data) - off} trailing bytes")
    return d


def load_pply_gswp(pply_path, gswp_path):
    """A checkpoint dict from a ``.pply`` + ``.gswp`` pair."""
    d = read_pply(pply_path)
    w = read_gswp(gswp_path)
    if w.get("low_rank"):
        n = w["low_shs_w"].shape[0]
    else:
        n = w["shs_w"].shape[0]
    if n != d["pw"].shape[0]:
        raise ValueError("the .pply and .gswp hold different Gaussian counts")
    d.update(w)
    validate(d)
    return d


def to_scene(d, scene_id, device="cuda", weight_dtype=torch.float32):
    """Upload a checkpoint dict into a resident ``palette_b200.serve.Scene``:
    geometry FP32, weights (shs, or dc / A / B) in `weight_dtype`."""
    from palette_b200.serve import Scene
    validate(d)
    dev = torch.device(device)
    t = lambda x, dt=torch.float32: torch.from_numpy(_f32(x)).to(dev, dt).contiguous()
    geo = dict(pws=t(d["pw"]), rots=t(d["rot"]), scales=t(d["scale"]),
               alphas=t(np.asarray(d["alpha"]).reshape(-1)))
    if d.get("low_rank"):
        return Scene(scene_id, **geo, dc=t(d["low_shs_w"], weight_dtype),
                     A=t(d["high_shs_A"], weight_dtype), B=t(d["high_shs_B"], weight_dtype))
    return Scene(scene_id, **geo, shs=t(d["shs_w"], weight_dtype))
