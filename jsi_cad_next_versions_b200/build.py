"""Builds libjsi_b200.so (sm_100a) in-tree with nvcc.

    python -m jsi_cad_next_versions_b200.build

The library is the product: hand-written CUDA kernels plus the C++ host
orchestration behind the C ABI declared in include/jsi_b200.h.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libjsi_b200.so"
SHIM = PKG / "libjsi_v5_shim.so"
SOURCES = ["jsi_kernels.cu", "jsi_capi.cu", "jsi_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: products and sums round separately, in the written order, so
# the FP32 form reproduces the reference's x86 results bit for bit.  Explicit
# fma() calls are still honoured where a kernel asks for them.
FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "jsi_b200.h"]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build_shim(force: bool = False) -> Path:
    """libjsi_v5_shim.so: the reference's C++ query API over the C ABI."""
    src = CSRC / "jsi_v5_shim.cpp"
    if not force and SHIM.exists() and SHIM.stat().st_mtime >= max(src.stat().st_mtime, LIB.stat().st_mtime):
        return SHIM
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", f"-I{ROOT / 'include'}", str(src), f"-L{PKG}",
           "-ljsi_b200", "-Wl,-rpath,$ORIGIN", "-o", str(SHIM)]
    subprocess.run(cmd, check=True)
    return SHIM


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        build_shim()
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, *FLAGS, "-shared", f"-I{ROOT / 'include'}", f"-I{CSRC}", "-o", str(tmp)]
    cmd += [str(CSRC / s) for s in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_shim(force=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
