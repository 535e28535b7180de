"""Builds the sm_100a engine library in-tree: ragdoll_b200/libragdoll_cuda.so.

Plain nvcc (no torch extension machinery): the library is a C ABI over the CUDA runtime, so it
loads through ctypes and is the same file a Rust / C host would link.
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
LIB = PKG / "libragdoll_cuda.so"
BUILD = PKG / "_build"

SOURCES = ["engine_kernels.cu", "ssim_kernels.cu", "rg_api.cu", "ssim_noalloc.cu", "candidate_net.cu", "cavlc_writer.cpp",
           "cabac_writer.cpp", "containers.cpp", "host_encoder.cpp", "records.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "-Xcompiler", "-march=x86-64-v3", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + [ROOT / "include" / "ragdoll_cuda.h", Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    BUILD.mkdir(exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        extra = ["-Xptxas", "-v"] if ptxas_v else []
        if src in ("ssim_kernels.cu", "ssim_noalloc.cu"):
            extra += ["-fmad=false"]
        cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv)
    print(LIB)
