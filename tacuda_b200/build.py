"""Build the in-tree shared library libtacuda_b200.so for sm_100a.

    python -m tacuda_b200.build            # library
    python -m tacuda_b200.build --oracle   # library + CPU checkers (oracle/)

The library is compiled with nvcc directly (no torch extension machinery): the
product is a plain C-ABI shared object. FMA contraction is disabled
(--fmad=false) because the TA-Lib arithmetic is reproduced with explicit fma()
calls exactly where TA-Lib uses them.
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
OUT = PKG / "libtacuda_b200.so"
SOURCES = ["engine.cu", "adjoint.cu", "api.cu", "scheduler.cpp", "pool.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    return str(cand) if cand.exists() else (shutil.which("nvcc") or "nvcc")


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_library(verbose: bool = False) -> Path:
    srcs = [s for s in SOURCES if (CSRC / s).exists()]
    objdir = ROOT / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    for s in srcs:
        obj = objdir / (s + ".o")
        src = CSRC / s
        deps = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.inc")) + [ROOT / "include" / "tacuda.h", src]
        if not obj.exists() or any(d.stat().st_mtime > obj.stat().st_mtime for d in deps):
            cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                   f"-I{ROOT / 'include'}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
        objs.append(str(obj))
    _run([nvcc(), *ARCH, "-shared", "-o", str(OUT), *objs])
    return OUT


def build_oracle() -> None:
    _run(["make", "-s", "-C", str(ROOT / "oracle")])


if __name__ == "__main__":
    build_library(verbose="-v" in sys.argv)
    if "--oracle" in sys.argv:
        build_oracle()
