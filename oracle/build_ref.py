"""Compile the REFERENCE's CUDA voxelizer extension from its own two source
files into oracle/_ref/ -- TEST INFRASTRUCTURE (GPU cross-check and the
reference-kernel timing), never part of the product.

    python oracle/build_ref.py [--reference /path/to/GS_TMI]

The reference checkout is taken from --reference, else from the
GSV_REFERENCE_ROOT environment variable, else from DEFAULT_REFERENCE (where
this build's recipe finds it).

Sources (read in place, never copied):
    3DGS/3dgsVC/gaussian/cuda_ext/tile_voxelize_cuda.cpp
    3DGS/3dgsVC/gaussian/cuda_ext/tile_voxelize_cuda_kernel.cu
The reference builds them with torch.utils.cpp_extension.load and
nvcc "-O3 --use_fast_math" (gaussian/tile_voxelizer.py:58-66); this recipe
runs nvcc / g++ directly with the same optimisation flags, for sm_100a, and
links the objects into an importable Python extension module
``tile_voxelize_cuda_ref`` (pybind forward / backward, .cpp:33-36).
The output is git-ignored and travels with the working tree, so a machine
without the reference source can still load it.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
MODULE = "tile_voxelize_cuda_ref"
SO = os.path.join(OUT, MODULE + ".so")


DEFAULT_REFERENCE = "/root/reference"


def reference_root(reference: str | None = None) -> str:
    return reference or os.environ.get("GSV_REFERENCE_ROOT") or DEFAULT_REFERENCE


def sources(reference: str):
    base = os.path.join(reference, "3DGS", "3dgsVC", "gaussian", "cuda_ext")
    return (os.path.join(base, "tile_voxelize_cuda.cpp"), os.path.join(base, "tile_voxelize_cuda_kernel.cu"))


def build(reference: str | None = None, force: bool = False) -> str | None:
    cpp, cu = sources(reference_root(reference))
    if not (os.path.exists(cpp) and os.path.exists(cu)):
        return SO if os.path.exists(SO) else None
    if not force and os.path.exists(SO) and os.path.getmtime(SO) >= max(os.path.getmtime(cpp), os.path.getmtime(cu)):
        return SO
    import torch
    from torch.utils import cpp_extension as ce

    os.makedirs(OUT, exist_ok=True)
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    incs = [f"-I{p}" for p in ce.include_paths(device_type="cuda")] + [f"-I{sysconfig.get_paths()['include']}"]
    defs = [f"-DTORCH_EXTENSION_NAME={MODULE}", "-DTORCH_API_INCLUDE_EXTENSION_H", f"-D_GLIBCXX_USE_CXX11_ABI={abi}"]
    nvcc = os.path.join(ce.CUDA_HOME or "/usr/local/cuda", "bin", "nvcc")
    cu_o, cpp_o = os.path.join(OUT, "kernel.o"), os.path.join(OUT, "binding.o")
    subprocess.run([nvcc, "-O3", "--use_fast_math", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-Xcompiler", "-fPIC", "-D__CUDA_NO_HALF_OPERATORS__", "-D__CUDA_NO_HALF_CONVERSIONS__",
                    "-D__CUDA_NO_BFLOAT16_CONVERSIONS__", "-D__CUDA_NO_HALF2_OPERATORS__",
                    *defs, *incs, "-c", cu, "-o", cu_o], check=True)
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([gxx, "-O3", "-std=c++17", "-fPIC", *defs, *incs, "-c", cpp, "-o", cpp_o], check=True)
    libdirs = [f"-L{p}" for p in ce.library_paths(device_type="cuda")]
    subprocess.run([gxx, "-shared", cu_o, cpp_o, "-o", SO, *libdirs, "-lc10", "-lc10_cuda", "-ltorch",
                    "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python", "-lcudart",
                    f"-Wl,-rpath,{os.path.dirname(torch.__file__)}/lib"], check=True)
    return SO


PY_OUT = os.path.join(os.path.dirname(HERE), "baseline", "_ref")
PY_PACKAGES = ("configs", "data", "gaussian", "losses", "metrics", "trainers")


def stage_python(reference: str | None = None) -> str | None:
    """Stage the reference's Python package (3DGS/3dgsVC: its trainer, data
    loader, Gaussian model, losses, metrics and configs) unchanged into the
    git-ignored baseline/_ref/3dgsVC, where the drop-in test imports it and
    from where it travels with the working tree.  Returns the staged root,
    or None when neither the sources nor an earlier staging exist."""
    import shutil

    src = os.path.join(reference_root(reference), "3DGS", "3dgsVC")
    dst = os.path.join(PY_OUT, "3dgsVC")
    if not os.path.isdir(src):
        return dst if os.path.isdir(dst) else None
    os.makedirs(dst, exist_ok=True)
    for pkg in PY_PACKAGES:
        target = os.path.join(dst, pkg)
        if os.path.isdir(target):
            shutil.rmtree(target)
        shutil.copytree(os.path.join(src, pkg), target, ignore=shutil.ignore_patterns("build", "__pycache__", "*.so"))
    return dst


def load():
    """Import the compiled reference extension (None if it was never built)."""
    if not os.path.exists(SO):
        return None
    import importlib.util

    import torch  # noqa: F401  (the extension links against torch's libraries)

    spec = importlib.util.spec_from_file_location(MODULE, SO)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="reference checkout (default: $GSV_REFERENCE_ROOT, "
                                                         "else DEFAULT_REFERENCE)")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    out = build(a.reference, a.force)
    print(out if out else "reference sources not found; nothing built")
    staged = stage_python(a.reference)
    print(staged if staged else "reference Python package not found; nothing staged")
    sys.exit(0 if out else 1)
