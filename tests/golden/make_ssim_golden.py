"""Golden vectors for the L1 + SSIM loss, from the REFERENCE's own module.

ReparamGS-Palette's gau_loss (vanilla_3dgs/gsplat/pytorch_ssim.py:26-67) is
plain torch, so it runs on the CPU of the machine that holds the reference
sources: this script imports it from there, evaluates the loss and its autograd
gradient on small seeded images (FP64 and FP32, sizes that are not multiples
of the window or of a 32-pixel tile, one smaller than the window) and writes
tests/golden/ssim_gau_loss.npz.  tests/test_oracle_ssim.py pins the CPU oracle
to it.

    python tests/golden/make_ssim_golden.py [--reference /path/to/ReparamGS-Palette]

The reference checkout defaults to $GSB_REFERENCE_ROOT, else the location
oracle/build_ref.py uses.
"""
import argparse
import importlib.util
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [(3, 23, 37, 0), (3, 40, 33, 1), (3, 7, 5, 2), (3, 36, 44, 3)]


def main():
    ap = argparse.ArgumentParser()
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.build_ref import reference_root
    ap.add_argument("--reference", default=reference_root())  # the sources, read-only
    ap.add_argument("--out", default=os.path.join(HERE, "ssim_gau_loss.npz"))
    a = ap.parse_args()
    path = os.path.join(a.reference, "vanilla_3dgs", "gsplat", "pytorch_ssim.py")
    spec = importlib.util.spec_from_file_location("ref_pytorch_ssim", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for C_, H, W, seed in CASES:
        rng = np.random.default_rng(seed)
        x = rng.random((C_, H, W))
        y = rng.random((C_, H, W))
        # a few exact ties (|x - y| has a zero subgradient there)
        x.reshape(-1)[::17] = y.reshape(-1)[::17]
        key = f"{H}x{W}_s{seed}"
        out[key + "_x"], out[key + "_y"] = x, y
        for dt, name in ((torch.float64, "f64"), (torch.float32, "f32")):
            X = torch.tensor(x, dtype=dt, requires_grad=True)
            Y = torch.tensor(y, dtype=dt)
            loss = mod.gau_loss(X, Y)
            loss.backward()
            out[f"{key}_{name}_loss"] = np.array(loss.item())
            out[f"{key}_{name}_dx"] = X.grad.numpy()
    np.savez_compressed(a.out, **out)
    print("wrote", a.out, len(out), "arrays")


if __name__ == "__main__":
    main()
