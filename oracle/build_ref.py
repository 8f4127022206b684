"""Compile the reference ``gsplatcu`` extension into ``oracle/_ref/`` (test infrastructure).

This is a checker, not product code: the parity tests and the golden-fixture
script load the result to compare the B200 kernels against the reference's own
CUDA build on identical inputs.  The recipe compiles the reference's three
sources where they lie (``gsplatcu/ext.cpp``, ``gsplatcu/kernel.cu``,
``gsplatcu/gausplat.cu``) with ``torch.utils.cpp_extension.load`` under the
module name ``gsplatcu_ref`` (so it can be imported beside the drop-in
``gsplatcu``), targeting sm_100 SASS exactly as a ``TORCH_CUDA_ARCH_LIST=10.0``
build of the reference would.  The reference's own ``setup.py`` is not run.

It also stages, unmodified, the reference's Python caller --
``gsplat/gsmodel.py`` and the ``gsplat/utils.py`` it star-imports -- and its
numpy rasterizer ``gsplat/gausplat.py`` with the ``gsplat/sh_coef.py`` it
imports, as the package ``oracle/_ref/gsplat``: the drop-in test runs the
reference's own autograd functions (``WeightGSFunctionTest`` /
``WeightGSFunctionFast``, ``FinetuneModel``) on either ``gsplatcu`` build,
and the benchmark's reference arm times the numpy path on the host cores.

The reference checkout is ``--root``, else ``$GSB_REFERENCE_ROOT``, else the
build container's copy::

    python oracle/build_ref.py [--root <ReparamGS-Palette checkout>]

Output (git-ignored; it travels with the tree to the GPU box, where
``load_ref()`` / ``load_vanilla_ref()`` / ``reference_caller()`` use it
without recompiling): ``oracle/_ref/gsplatcu_ref.so``, from the stage-1
sources ``vanilla_3dgs/gsplatcu`` ``oracle/_ref/vanilla/gsplatcu_vanilla_ref.so``,
and ``oracle/_ref/gsplat/{gsmodel,utils,gausplat,sh_coef}.py``.
"""
import argparse
import importlib.machinery
import importlib.util
import os
import shutil
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "gsplatcu_ref.so")
CALLER_DIR = os.path.join(REF_DIR, "gsplat")
CALLER_FILES = ("gsmodel.py", "utils.py", "gausplat.py", "sh_coef.py")

# The stage-1 (vanilla 3DGS) extension of the same project: its colour splat
# backward carries the final-transmittance gradient (splat / splatB).
VANILLA_DIR = os.path.join(REF_DIR, "vanilla")
VANILLA_SO = os.path.join(VANILLA_DIR, "gsplatcu_vanilla_ref.so")


def reference_root():
    """Root of the read-only reference checkout (ReparamGS-Palette)."""
    return os.environ.get("GSB_REFERENCE_ROOT", "/root/reference")


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


def build(root=None, verbose=False):
    _compile("gsplatcu_ref", os.path.join(root or reference_root(), "gsplatcu"), REF_DIR, verbose)
    return REF_SO


def build_vanilla(root=None, verbose=False):
    _compile("gsplatcu_vanilla_ref", os.path.join(root or reference_root(), "vanilla_3dgs", "gsplatcu"),
             VANILLA_DIR, verbose)
    return VANILLA_SO


def stage_caller(root=None):
    """Copy the reference's gsplat/{gsmodel,utils,gausplat,sh_coef}.py, byte
    for byte, into oracle/_ref/gsplat (a namespace package, as in the
    reference)."""
    src = os.path.join(root or reference_root(), "gsplat")
    os.makedirs(CALLER_DIR, exist_ok=True)
    for f in CALLER_FILES:
        shutil.copyfile(os.path.join(src, f), os.path.join(CALLER_DIR, f))
    return CALLER_DIR


def caller_staged():
    return all(os.path.exists(os.path.join(CALLER_DIR, f)) for f in CALLER_FILES)


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


def _stub_matplotlib():
    """gsplat/utils.py and gsplat/gausplat.py import matplotlib.pyplot for
    plotting helpers the timed and tested paths never call; when matplotlib
    is absent an empty stand-in is installed (its pause() is a no-op)."""
    if "matplotlib" in sys.modules:
        return
    try:
        import matplotlib  # noqa: F401
    except ImportError:
        mpl = types.ModuleType("matplotlib")
        mpl.pyplot = types.ModuleType("matplotlib.pyplot")
        mpl.pyplot.pause = lambda *a, **k: None
        sys.modules["matplotlib"], sys.modules["matplotlib.pyplot"] = mpl, mpl.pyplot


def reference_numpy_path():
    """The reference's numpy rasterizer module ``gsplat/gausplat.py``
    (project, compute_cov_3d, compute_cov_2d, inverse_cov2d, sh2color,
    splat), executed unchanged; None when it has not been staged."""
    if not caller_staged():
        return None
    _stub_matplotlib()
    saved = {k: sys.modules.get(k) for k in ("gsplat", "gsplat.sh_coef")}
    try:
        pkg = types.ModuleType("gsplat")
        pkg.__path__ = [CALLER_DIR]
        sys.modules["gsplat"] = pkg
        sc_spec = importlib.util.spec_from_file_location(
            "gsplat.sh_coef", os.path.join(CALLER_DIR, "sh_coef.py"))
        sh_coef = importlib.util.module_from_spec(sc_spec)
        sys.modules["gsplat.sh_coef"] = sh_coef
        sc_spec.loader.exec_module(sh_coef)
        spec = importlib.util.spec_from_file_location(
            "gausplat_ref", os.path.join(CALLER_DIR, "gausplat.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        return mod
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v


def reference_caller(gsplatcu_module, tag):
    """The reference's own ``gsplat.gsmodel`` module, executed unchanged with
    ``import gsplatcu`` resolving to ``gsplatcu_module`` (this build's drop-in
    or the reference build).  Each call returns a fresh module object named
    ``gsmodel_<tag>``, so both builds' callers can live in one process.
    ``gsplat/utils.py`` imports matplotlib for a plotting helper the render
    path never calls; when matplotlib is absent an empty stand-in is
    installed.  Returns None when the caller has not been staged."""
    if not caller_staged():
        return None
    _stub_matplotlib()
    saved = {k: sys.modules.get(k) for k in ("gsplatcu", "gsplat", "gsplat.utils")}
    try:
        sys.modules["gsplatcu"] = gsplatcu_module
        pkg = types.ModuleType("gsplat")
        pkg.__path__ = [CALLER_DIR]
        sys.modules["gsplat"] = pkg
        sys.modules.pop("gsplat.utils", None)
        utils_spec = importlib.util.spec_from_file_location(
            "gsplat.utils", os.path.join(CALLER_DIR, "utils.py"))
        utils = importlib.util.module_from_spec(utils_spec)
        sys.modules["gsplat.utils"] = utils
        utils_spec.loader.exec_module(utils)
        pkg.utils = utils
        spec = importlib.util.spec_from_file_location(
            f"gsmodel_{tag}", os.path.join(CALLER_DIR, "gsmodel.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        return mod
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--root", default=None, help="reference checkout (default: $GSB_REFERENCE_ROOT)")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.root, a.verbose))
    print(build_vanilla(a.root, a.verbose))
    print(stage_caller(a.root))
    sys.exit(0)
