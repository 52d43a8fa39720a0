"""Build the engine's shared library in-tree with nvcc for sm_100a.

    python -m xfdtd_cuda_b200.build        # builds xfdtd_cuda_b200/libxfdtd_b200.so

The library is plain C-ABI (include/xfdtd_b200.h); it links only the CUDA
runtime (statically).  The FP64 engine and the C-ABI are compiled with
--fmad=false, which keeps every floating-point operation individually rounded
so the FP64 engine reproduces an IEEE CPU evaluation of the same expressions
in the same order; the FP32 engine is compiled with FMA contraction.
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


# (source, fmad) pairs
UNITS = [("api.cu", False), ("engine_f64.cu", False), ("engine_f32.cu", True), ("labc_train.cu", True),
         ("scene_compile.cpp", False), ("core_ingest.cpp", False), ("host_copy.cpp", False)]


def sources() -> list[Path]:
    return [CSRC / u for u, _ in UNITS]


def build(force: bool = False, verbose: bool = False) -> Path:
    deps = sources() + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "xfdtd_b200.h"]
    if LIB.exists() and not force:
        mt = LIB.stat().st_mtime
        if all(p.stat().st_mtime <= mt for p in deps):
            return LIB
    tmp = LIB.with_suffix(".so.tmp")
    objdir = ROOT / "_build" / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    objs = []
    procs = []
    for unit, fmad in UNITS:
        obj = objdir / (unit + ".o")
        cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", f"--fmad={'true' if fmad else 'false'}",
               "-Xcompiler", "-fPIC,-O3,-fopenmp", "-I", str(ROOT / "include"), "-c", "-o", str(obj), str(CSRC / unit)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        procs.append((unit, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    for unit, p in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out + err)
            raise RuntimeError(f"nvcc failed on {unit}")
        if verbose:
            sys.stderr.write(err)
    cmd = [nvcc(), "-shared", "-cudart", "static", *ARCH, "-o", str(tmp), *[str(o) for o in objs], "-lgomp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed linking libxfdtd_b200.so")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
