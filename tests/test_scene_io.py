"""Scene files: the finetune checkpoint ``.npy`` and the ``.pply`` + ``.gswp``
pair round-trip (CPU); the writers produce the same bytes as the reference's
converter (convert_npy_ply/palette_npy_to_pply.py:176-272) and the readers
read its files (golden bytes in tests/golden/scene_formats.npz, made by
tests/golden/make_scene_golden.py from the reference's own convert());
on the GPU, a scene loaded from them renders like the same parameters passed
directly."""
import os
import sys
import numpy as np
import pytest
import torch

from palette_b200 import scene_io
from palette_b200.scene import synthetic_scene


def _ckpt(n=500, low_rank=False, seed=0):
    sc = synthetic_scene(n, seed=seed, mode="lowrank" if low_rank else "full", rank=1)
    d = dict(palette=sc["palette"], pw=sc["pws"], rot=sc["rots"], scale=sc["scales"],
             alpha=sc["alphas"])
    if low_rank:
        d.update(low_rank=True, low_shs_w=sc["dc"], high_shs_A=sc["A"][:, :, 0],
                 high_shs_B=sc["B"][:, 0, :], reshape_P=5, reshape_Q=15)
    else:
        d.update(low_rank=False, shs_w=sc["shs"])
    return d


@pytest.mark.parametrize("low_rank", [False, True])
def test_checkpoint_and_pply_gswp_round_trip(tmp_path, low_rank):
    d = _ckpt(low_rank=low_rank)
    scene_io.save_checkpoint(tmp_path / "s.npy", d)
    d2 = scene_io.load_checkpoint(tmp_path / "s.npy")
    for k in d:
        assert np.array_equal(np.asarray(d[k]), np.asarray(d2[k])), k
    scene_io.write_pply(tmp_path / "s.pply", d)
    scene_io.write_gswp(tmp_path / "s.gswp", d)
    d3 = scene_io.load_pply_gswp(tmp_path / "s.pply", tmp_path / "s.gswp")
    assert np.array_equal(d3["pw"], d["pw"]) and np.array_equal(d3["rot"], d["rot"])
    np.testing.assert_allclose(d3["scale"], d["scale"], rtol=1e-6)
    np.testing.assert_allclose(d3["alpha"], np.asarray(d["alpha"]).reshape(-1), rtol=1e-5,
                               atol=1e-6)
    assert np.array_equal(d3["palette"], d["palette"])
    keys = ("low_shs_w", "high_shs_A", "high_shs_B") if low_rank else ("shs_w",)
    for k in keys:
        assert np.array_equal(d3[k], d[k]), k
    # header: magic, version 1, N, splat_dim, num_sh, low_rank, P, Q
    head = (tmp_path / "s.gswp").read_bytes()[:32]
    assert head[:4] == b"GSWP"
    assert np.frombuffer(head[4:], "<u4").tolist() == \
        [1, 500, 5, 16, int(low_rank), 5 if low_rank else 0, 15 if low_rank else 0]


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scene_formats.npz")


def _golden_checkpoints():
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_scene_golden import checkpoints
    return checkpoints()


@pytest.mark.parametrize("name", ["dense", "lowrank"])
def test_writers_match_reference_converter_bytes(tmp_path, name):
    z = np.load(GOLDEN)
    d = _golden_checkpoints()[name]
    scene_io.write_pply(tmp_path / "s.pply", d)
    scene_io.write_gswp(tmp_path / "s.gswp", d)
    assert (tmp_path / "s.pply").read_bytes() == z[f"{name}_pply"].tobytes()
    assert (tmp_path / "s.gswp").read_bytes() == z[f"{name}_gswp"].tobytes()


@pytest.mark.parametrize("name", ["dense", "lowrank"])
def test_readers_load_reference_converter_files(tmp_path, name):
    z = np.load(GOLDEN)
    d = _golden_checkpoints()[name]
    (tmp_path / "r.pply").write_bytes(z[f"{name}_pply"].tobytes())
    (tmp_path / "r.gswp").write_bytes(z[f"{name}_gswp"].tobytes())
    r = scene_io.load_pply_gswp(tmp_path / "r.pply", tmp_path / "r.gswp")
    assert np.array_equal(r["pw"], d["pw"]) and np.array_equal(r["rot"], d["rot"])
    assert np.array_equal(r["palette"], d["palette"])
    np.testing.assert_allclose(r["scale"], d["scale"], rtol=1e-6)
    a = np.clip(np.asarray(d["alpha"]).reshape(-1), 1e-6, 1 - 1e-6)  # the converter's logit clip
    np.testing.assert_allclose(r["alpha"], a, rtol=1e-5, atol=1e-6)
    keys = ("low_shs_w", "high_shs_A", "high_shs_B") if d["low_rank"] else ("shs_w",)
    for k in keys:
        assert np.array_equal(r[k], d[k]), k
    assert bool(r["low_rank"]) == d["low_rank"]


def test_malformed_files_are_rejected(tmp_path):
    d = _ckpt()
    bad = dict(d)
    bad["rot"] = d["rot"][:, :3]
    with pytest.raises(ValueError):
        scene_io.validate(bad)
    (tmp_path / "x.gswp").write_bytes(b"NOPE" + bytes(28))
    with pytest.raises(ValueError):
        scene_io.read_gswp(tmp_path / "x.gswp")
    scene_io.write_gswp(tmp_path / "t.gswp", d)
    data = (tmp_path / "t.gswp").read_bytes()
    (tmp_path / "t2.gswp").write_bytes(data + b"\0\0\0\0")
    with pytest.raises(ValueError):
        scene_io.read_gswp(tmp_path / "t2.gswp")


@pytest.mark.gpu
@pytest.mark.parametrize("low_rank", [False, True])
def test_loaded_scene_renders_like_direct_parameters(cuda_ok, tmp_path, low_rank):
    from palette_b200.render import render_palette
    from palette_b200.scene import look_at
    d = _ckpt(n=20000, low_rank=low_rank, seed=4)
    scene_io.save_checkpoint(tmp_path / "s.npy", d)
    sc = scene_io.to_scene(scene_io.load_checkpoint(tmp_path / "s.npy"), "s")
    cam = look_at((0.0, -8.0, 1.0), width=128, height=96, device="cuda")
    kw = dict(shs=sc.shs) if not low_rank else dict(dc=sc.w0, A=sc.A, B=sc.B)
    with torch.no_grad():
        layer, _, _ = render_palette(sc.pws, sc.rots, sc.scales, sc.alphas, cam, **kw)
        t = lambda x: torch.from_numpy(np.asarray(x, np.float32)).cuda()
        kw2 = dict(shs=t(d["shs_w"])) if not low_rank else dict(
            dc=t(d["low_shs_w"]), A=t(d["high_shs_A"]), B=t(d["high_shs_B"]))
        ref, _, _ = render_palette(t(d["pw"]), t(d["rot"]), t(d["scale"]),
                                   t(np.asarray(d["alpha"]).reshape(-1)), cam, **kw2)
    assert torch.equal(layer, ref)
