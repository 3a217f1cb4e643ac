"""Build libolcuda.so (the sm_100a kernels and the C ABI) in-tree with nvcc."""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
INCLUDE = PACKAGE.parent / "include"
LIB_DIR = PACKAGE / "_lib"
LIBRARY = LIB_DIR / "libolcuda.so"
SOURCES = ("olc_bvh.cu", "olc_wavefront.cu", "olc_restir.cu", "olc_motion.cu", "olc_api.cu", "olc_noalloc.cu")
ARCH = ("-gencode", "arch=compute_100a,code=sm_100a")
FLAGS = (
    "-O3", "-std=c++17", "-lineinfo",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
)


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc was not found; the CUDA toolkit is required to build libolcuda")
    return found


def _stale(target: Path, inputs) -> bool:
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(p.stat().st_mtime > mtime for p in inputs)


def build(verbose: bool = False, force: bool = False, extra_flags=()) -> Path:
    """Compile every CUDA source for sm_100a and link libolcuda.so."""
    LIB_DIR.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    objects = []
    compiler = nvcc()
    for name in SOURCES:
        src = CSRC / name
        obj = LIB_DIR / (src.stem + ".o")
        objects.append(obj)
        if force or _stale(obj, [src, *headers]):
            cmd = [compiler, *ARCH, *FLAGS, *extra_flags, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIBRARY, objects):
        cmd = [compiler, *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIBRARY


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
