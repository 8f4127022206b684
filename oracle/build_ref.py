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

Output: ``oracle/_ref/gsplatcu_ref.so`` (git-ignored; travels with the tree to
the GPU box, where ``load_ref()`` imports it without recompiling).
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


def build(src=DEFAULT_SRC, verbose=False):
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference sources not found at {src}")
    os.makedirs(REF_DIR, exist_ok=True)
    os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0"
    os.environ.setdefault("MAX_JOBS", "8")
    from torch.utils.cpp_extension import load
    sources = [os.path.join(src, f) for f in ("ext.cpp", "kernel.cu", "gausplat.cu")]
    load(name="gsplatcu_ref", sources=sources, build_directory=REF_DIR,
         extra_cflags=["-O3"], extra_cuda_cflags=["-O3"], verbose=verbose)
    return REF_SO


def load_ref():
    """Import the prebuilt reference module, or return None when it is absent."""
    if not os.path.exists(REF_SO):
        return None
    import torch  # noqa: F401  (the module links against libtorch)
    loader = importlib.machinery.ExtensionFileLoader("gsplatcu_ref", REF_SO)
    spec = importlib.util.spec_from_file_location("gsplatcu_ref", REF_SO, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.src, a.verbose))
    sys.exit(0)
