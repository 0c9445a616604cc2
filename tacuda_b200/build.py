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
# (source, object name, extra defines): engine.cu is compiled twice, the second
# time for the kernels of the precision variants only
SOURCES = [("engine.cu", "engine.cu.o", []), ("engine.cu", "engine_prec.cu.o", ["-DTB_PREC_TU"]),
           ("rows.cu", "rows.cu.o", []), ("adjoint.cu", "adjoint.cu.o", []), ("api.cu", "api.cu.o", []),
           ("scheduler.cpp", "scheduler.cpp.o", []), ("pool.cpp", "pool.cpp.o", [])]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    return str(cand) if cand.exists() else (shutil.which("nvcc") or "nvcc")


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _compile(cmd, obj: Path):
    """Compile, then date the object at the compile's start: a source edited
    while nvcc ran stays newer than the object and is rebuilt next time."""
    import time
    t0 = time.time()
    _run(cmd)
    os.utime(obj, (t0, t0))


def _includes(src: Path, seen: set) -> set:
    """Project headers a source includes, directly or through other headers."""
    import re
    for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', src.read_text(), re.M):
        for d in (src.parent, CSRC, ROOT / "include"):
            h = d / name
            if h.exists():
                if h not in seen:
                    seen.add(h)
                    _includes(h, seen)
                break
    return seen


def build_library(verbose: bool = False) -> Path:
    from concurrent.futures import ThreadPoolExecutor
    objdir = ROOT / "_build"
    objdir.mkdir(exist_ok=True)
    jobs, objs = [], []
    for src_name, obj_name, defines in SOURCES:
        src = CSRC / src_name
        if not src.exists():
            continue
        obj = objdir / obj_name
        objs.append(str(obj))
        deps = sorted(_includes(src, set()))
        if not obj.exists() or any(d.stat().st_mtime > obj.stat().st_mtime for d in deps + [src]):
            cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                   f"-I{ROOT / 'include'}", f"-I{CSRC}", *defines, "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append((cmd, obj))
    # translation units compile in parallel (the two engine halves dominate)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_compile, cmd, obj) for cmd, obj in jobs]:
            f.result()
    _run([nvcc(), *ARCH, "-shared", "-o", str(OUT), *objs])
    return OUT


# The reference tree the oracle's reference builds compile from, where it exists
# (only in the build container; the GPU box uses the prebuilt oracle/_ref files).
REFERENCE_TREE = Path(os.environ.get("TACUDA_REFERENCE_TREE", "/root/reference"))


def build_oracle() -> None:
    cmd = ["make", "-s", "-C", str(ROOT / "oracle")]
    if REFERENCE_TREE.is_dir():
        cmd.append(f"REF={REFERENCE_TREE}")
    _run(cmd)


if __name__ == "__main__":
    build_library(verbose="-v" in sys.argv)
    if "--oracle" in sys.argv:
        build_oracle()
