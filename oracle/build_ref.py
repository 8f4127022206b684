"""Compile the reference ``gsplatcu`` extension into ``oracle/_ref/`` (test infrastructure).

This is a checker, not product code: the parity tests and the golden-fixture
script load the result to compare the B200 kernels against the reference's own
CUDA build on identical inputs.  The recipe compiles the reference's three
sources where they lie (``gsplatcu/ext.cpp``, ``gsplatcu/kernel.cu``,
``gsplatcu/gausplat.cu``) with ``torch.utils.cpp_extension.load`` under the
module name ``gsplatcu_ref`` (so it can be imported beside the drop-in
``gsplatcu``), targeting sm_100 SASS exactly as a ``TORCH_CUDA_ARCH_LIST=10.0``
build of the reference would.  The reference's own ``setup.py`` is not run.

Usage (in the build container, where the reference sources exist)::

    python oracle/build_ref.py [--src <reference>/gsplatcu]

Output: ``oracle/_ref/gsplatcu_ref.so`` and, from the stage-1 sources
``vanilla_3dgs/gsplatcu``, ``oracle/_ref/vanilla/gsplatcu_vanilla_ref.so``
(git-ignored; they travel with the tree to the GPU box, where ``load_ref()`` /
``load_vanilla_ref()`` import them without recompiling).
"""
import argparse
import importlib.machinery
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "gsplatcu_ref.so")
DEFAULT_SRC = "/root/reference/gsplatcu"


# The stage-1 (vanilla 3DGS) extension of the same project: its colour splat
# backward carries the final-transmittance gradient (splat / splatB).
VANILLA_DIR = os.path.join(REF_DIR, "vanilla")
VANILLA_SO = os.path.join(VANILLA_DIR, "gsplatcu_vanilla_ref.so")
DEFAULT_VANILLA_SRC = "/root/reference/vanilla_3dgs/gsplatcu"


def _compile(name, src, out_dir, verbose):
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference sources not found at {src}")
    os.makedirs(out_dir, exist_ok=True)
    os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0"
    os.environ.setdefault("MAX_JOBS", "8")
    from torch.utils.cpp_extension import load
    sources = [os.path.join(src, f) for f in ("ext.cpp", "kernel.cu", "gausplat.cu")]
    load(name=name, sources=sources, build_directory=out_dir, extra_cflags=["-O3"],
         extra_cuda_cflags=["-O3"], verbose=verbose)


def build(src=DEFAULT_SRC, verbose=False):
    _compile("gsplatcu_ref", src, REF_DIR, verbose)
    return REF_SO


def build_vanilla(src=DEFAULT_VANILLA_SRC, verbose=False):
    _compile("gsplatcu_vanilla_ref", src, VANILLA_DIR, verbose)
    return VANILLA_SO


def _load(name, path):
    if not os.path.exists(path):
        return None
    import torch  # noqa: F401  (the module links against libtorch)
    loader = importlib.machinery.ExtensionFileLoader(name, path)
    spec = importlib.util.spec_from_file_location(name, path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def load_ref():
    """Import the prebuilt reference module, or return None when it is absent."""
    return _load("gsplatcu_ref", REF_SO)


def load_vanilla_ref():
    """Import the prebuilt stage-1 reference module, or return None when absent."""
    return _load("gsplatcu_vanilla_ref", VANILLA_SO)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("--vanilla-src", default=DEFAULT_VANILLA_SRC)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.src, a.verbose))
    print(build_vanilla(a.vanilla_src, a.verbose))
    sys.exit(0)
