"""Builds libicflow_b200.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ behind an extern "C" ABI (include/icflow_b200.h);
it links only the CUDA runtime, so a C# host can load it through P/Invoke and a
Python host through ctypes.  Usage: ``python -m icflow_b200.build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libicflow_b200.so"
BUILD = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "--expt-relaxed-constexpr"]
# Files whose integer outputs depend on floating-point comparisons are built
# without fused multiply-add so that every operation rounds on its own.
NO_FMA = {"icf_contact.cu", "icf_broad.cu", "icf_contact_deriv.cu"}
SOURCES = ["icf_api.cu", "icf_assembly.cu", "icf_pattern.cu", "icf_contact.cu", "icf_contact_deriv.cu",
           "icf_noalloc.cu", "icf_gather.cu", "icf_tune.cu", "icf_solve.cu", "icf_broad.cu", "icf_mlp.cu",
           "icf_tile.cu"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build icflow_b200")
    return cand


def _needs(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "icflow_b200.h"]
    objs = []
    for src in SOURCES:
        s = CSRC / src
        if not s.exists():
            continue
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or _needs(o, [s, *headers]):
            cmd = [nvcc(), *ARCH, *COMMON, "-c", str(s), "-o", str(o)]
            if src in NO_FMA:
                cmd.insert(1, "-fmad=false")
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _needs(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
