"""Build the engine's shared library in-tree with nvcc for sm_100a.

    python -m xfdtd_cuda_b200.build        # builds xfdtd_cuda_b200/libxfdtd_b200.so

The library is plain C-ABI (include/xfdtd_b200.h); it links only the CUDA
runtime.  --fmad=false keeps every floating-point operation individually
rounded so the FP64 build reproduces an IEEE CPU evaluation of the same
expressions in the same order.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libxfdtd_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the engine needs the CUDA toolkit to build")


def sources() -> list[Path]:
    return [CSRC / "api.cu", CSRC / "scene_compile.cpp"]


def build(force: bool = False, verbose: bool = False) -> Path:
    deps = sources() + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "xfdtd_b200.h"]
    if LIB.exists() and not force:
        mt = LIB.stat().st_mtime
        if all(p.stat().st_mtime <= mt for p in deps):
            return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [
        nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "--fmad=false",
        "-Xcompiler", "-fPIC,-O3", "-shared", "-I", str(ROOT / "include"),
        "-cudart", "static", "-o", str(tmp), *[str(s) for s in sources()],
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libxfdtd_b200.so")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
