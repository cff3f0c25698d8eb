"""Build recipe of the CUDA library (in-tree, sm_100a).

``python -m warpmpc_b200.build`` compiles ``csrc/*.cu`` with nvcc into
``warpmpc_b200/libwarpmpc_b200.so``.  The library is the product: the Python
layer only binds it with ctypes.
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_NAME = "libwarpmpc_b200.so"
LIB_PATH = PKG / LIB_NAME

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-fmad=false",  # keep every product and sum separately rounded (reference op order)
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O3",
    "-Xptxas",
    "-warn-spills",
]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build warpmpc_b200")
    return cand


def sources() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_rebuild() -> bool:
    if not LIB_PATH.exists():
        return True
    mtime = LIB_PATH.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "warpmpc_b200.h"]
    return any(p.stat().st_mtime > mtime for p in deps if p.exists())


def build(verbose: bool = False, extra_flags: list[str] | None = None, force: bool = False) -> pathlib.Path:
    if not force and not needs_rebuild():
        return LIB_PATH
    nvcc = nvcc_path()
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc, *ARCH_FLAGS, *NVCC_FLAGS, *(extra_flags or []), "-I", str(PKG.parent / "include"), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    path = build(verbose=True, force="--force" in sys.argv, extra_flags=["-Xptxas", "-v"] if "-v" in sys.argv else None)
    print(path)
