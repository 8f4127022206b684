"""Golden files for the scene formats, from the REFERENCE's own converter.

ReparamGS-Palette's convert_npy_ply/palette_npy_to_pply.py is plain numpy: this
script imports it from the reference checkout (``--reference``, default
$GSB_REFERENCE_ROOT, else the location oracle/build_ref.py uses), writes two
small seeded finetune checkpoints (dense weights, and rank-1 low-rank factors
with the alpha stored as [N,1]), runs the reference's ``convert()`` on each
and stores the checkpoints' arrays with the exact bytes of the ``.pply`` and
``.gswp`` it wrote in tests/golden/scene_formats.npz.  tests/test_scene_io.py
checks this build's writers against those bytes and its readers on them.

    python tests/golden/make_scene_golden.py [--reference /path/to/ReparamGS-Palette]
"""
import argparse
import importlib.util
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def checkpoints():
    """The two seeded checkpoint dicts (the fields finetune.py saves)."""
    rng = np.random.default_rng(20)
    out = {}
    for name, n, low_rank in (("dense", 37, False), ("lowrank", 29, True)):
        K, nsh = 5, 16
        q = rng.normal(size=(n, 4))
        d = dict(pw=rng.normal(0, 2, (n, 3)).astype(np.float32),
                 rot=(q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32),
                 scale=np.exp(rng.normal(-4.5, 0.8, (n, 3))).astype(np.float32),
                 palette=np.concatenate([np.zeros((1, 3)), np.ones((1, 3)),
                                         rng.uniform(0, 1, (K - 2, 3))]).astype(np.float32),
                 low_rank=low_rank)
        a = 1 / (1 + np.exp(-rng.normal(0, 1.5, n)))
        a[0], a[1] = 0.0, 1.0  # clipped by the logit
        d["alpha"] = (a.reshape(n, 1) if low_rank else a).astype(np.float32)
        if low_rank:
            d.update(low_shs_w=rng.dirichlet(np.ones(K), n).astype(np.float32),
                     high_shs_A=rng.normal(0, 0.1, (n, K)).astype(np.float32),
                     high_shs_B=rng.normal(0, 0.1, (n, nsh - 1)).astype(np.float32),
                     reshape_P=K, reshape_Q=nsh - 1)
        else:
            d["shs_w"] = rng.normal(0, 0.05, (n, nsh * K)).astype(np.float32)
        out[name] = d
    return out


def main():
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.build_ref import reference_root
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=reference_root())  # the sources, read-only
    ap.add_argument("--out", default=os.path.join(HERE, "scene_formats.npz"))
    a = ap.parse_args()
    path = os.path.join(a.reference, "convert_npy_ply", "palette_npy_to_pply.py")
    spec = importlib.util.spec_from_file_location("ref_palette_npy_to_pply", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    arrays = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, d in checkpoints().items():
            npy = os.path.join(tmp, name + ".npy")
            np.save(npy, d, allow_pickle=True)
            pply = os.path.join(tmp, name + ".pply")
            mod.convert(npy, pply, verbose=False)
            for ext in ("pply", "gswp"):
                with open(os.path.join(tmp, f"{name}.{ext}"), "rb") as fh:
                    arrays[f"{name}_{ext}"] = np.frombuffer(fh.read(), np.uint8)
    np.savez_compressed(a.out, **arrays)
    print("wrote", a.out, {k: v.size for k, v in arrays.items()})


if __name__ == "__main__":
    main()
