"""Build of libedgpu.so (sm_100a) from ed-lgt_b200/csrc with nvcc.

The library is built in-tree (``edgpu/lib/libedgpu.so``) so that it travels
with the source tree; ``build_library`` is a no-op when the shared object is
newer than every source file.
"""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
SRC_DIR = PKG_DIR.parent / "csrc"
INCLUDE_DIR = PKG_DIR.parent.parent / "include"
LIB_DIR = PKG_DIR / "lib"
LIB_PATH = LIB_DIR / "libedgpu.so"

NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "--expt-relaxed-constexpr",
]


def _sources():
    return sorted(SRC_DIR.glob("*.cu"))


def _deps():
    return _sources() + sorted(SRC_DIR.glob("*.cuh")) + sorted(INCLUDE_DIR.glob("*.h"))


def library_is_current() -> bool:
    if not LIB_PATH.exists():
        return False
    t = LIB_PATH.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _deps())


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile every .cu file of csrc into libedgpu.so (sm_100a)."""
    if not force and library_is_current():
        return LIB_PATH
    nvcc = os.environ.get("NVCC", "nvcc")
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    obj_dir = LIB_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    objs = []
    for src in _sources():
        obj = obj_dir / (src.stem + ".o")
        cmd = [nvcc, *NVCC_FLAGS, "-I", str(INCLUDE_DIR), "-I", str(SRC_DIR), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB_DIR / "libedgpu.so.tmp"
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", str(tmp), "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build_library(force=True, verbose=True))
