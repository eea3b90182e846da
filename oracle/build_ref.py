"""Test infrastructure: the reference's own CUDA extension, built from its sources as a second
comparison point for per-kernel timings (never the product).

Compiles the five files of voxneus/cuda/ of rishidevde/VoxNeus (adam_upd.cpp, adam_upd_kernel.cu,
gradient_interp.cu, eikonal_grad.cu, curvature_grad.cu), unmodified and where they lie in the
reference tree, with torch's extension builder for sm_100a into oracle/_ref/ (git-ignored; the
built module travels with the repository to a GPU box, the reference tree does not). The
reference's setup.py is not run (it builds only when a GPU is visible, setup.py:10-15).

    python oracle/build_ref.py [--reference <reference>/Code]
        (default: $VOXNEUS_REFERENCE, else the reference tree of the build container)

`load()` imports the built module: the pybind functions of voxneus.cuda._backend
(adam_upd.cpp:118-125).
"""

from __future__ import annotations

import argparse
import glob
import importlib.machinery
import importlib.util
import os

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
NAME = "voxneus_ref_cuda"
SOURCES = ("adam_upd.cpp", "adam_upd_kernel.cu", "gradient_interp.cu", "eikonal_grad.cu", "curvature_grad.cu")


def built_path():
    hits = sorted(glob.glob(os.path.join(OUT, NAME + "*.so")))
    return hits[0] if hits else None


def build(reference=None, verbose=False):
    """Build the module when the reference tree is present; returns the .so path or None."""
    ref = reference or os.environ.get("VOXNEUS_REFERENCE") or "/root/reference/Code"
    src = os.path.join(ref, "voxneus", "cuda")
    files = [os.path.join(src, f) for f in SOURCES]
    if not all(os.path.exists(f) for f in files):
        return None
    os.makedirs(OUT, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    from torch.utils.cpp_extension import load as cpp_load

    cpp_load(name=NAME, sources=files, build_directory=OUT, extra_cflags=["-O3"], extra_cuda_cflags=["-O3"],
             verbose=verbose)
    return built_path()


def load():
    """The built reference module (import torch first), or None when it was not built."""
    path = built_path()
    if path is None:
        return None
    import torch  # noqa: F401  (the module links against libtorch)

    loader = importlib.machinery.ExtensionFileLoader(NAME, path)
    spec = importlib.util.spec_from_loader(NAME, loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("VOXNEUS_REFERENCE"))
    args = ap.parse_args()
    print(build(args.reference, verbose=True))
