"""Build recipe of the native library ``gelios_2d_b200/_lib/libgelios_b200.so``.

nvcc compiles the CUDA kernels for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) and the host C++ (grid builders, C ABI)
into one shared library with a plain C ABI (include/gelios_b200.h).  The
library is built in-tree so that it travels with the repository to the GPU
machine; it cross-compiles without a GPU.
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
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libgelios_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# FMA contraction on: each fused multiply-add rounds once where the
# reference's x86-64 build rounds twice (<= 1 ulp per operation, inside the
# 1e-12-per-step parity bound the tests enforce).
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=true", "-Xcompiler", "-fPIC", "-Xptxas", "-O3"]
CUDA_SOURCES = ["step_kernels.cu", "capi.cu", "noalloc.cu", "mlp.cu"]
HOST_SOURCES = ["mesh.cpp", "common.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return [Path(__file__)] + [CSRC / s for s in CUDA_SOURCES + HOST_SOURCES] + sorted(CSRC.glob("*.cuh")) + [
        ROOT / "include" / "gelios_b200.h"]


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _sources())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for src in CUDA_SOURCES:
        o = obj_dir / (Path(src).stem + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(o)]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(o)
    for src in HOST_SOURCES:
        o = obj_dir / (Path(src).stem + ".o")
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-c", str(CSRC / src), "-o", str(o)]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(o)
    for cmd, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode != 0:
            sys.stderr.write(out.decode(errors="replace"))
        if p.returncode != 0:
            raise RuntimeError("build failed: " + " ".join(cmd))
    tmp = LIB.with_suffix(".so.tmp")
    link = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
