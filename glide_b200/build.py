"""Build the in-tree native library ``glide_b200/libglide_b200.so`` for sm_100a.

Usage: ``python -m glide_b200.build [--verbose]``.  The library is a plain
shared object with a C ABI (``include/glide_b200.h``); it is rebuilt when any
source is newer than it.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libglide_b200.so"
SOURCES = ["ssa_stencil.cu", "vanka.cu", "transfer.cu", "driver.cu", "tc_gemm.cu", "unet_ops.cu",
           "vanka_noalloc.cu", "losses.cu", "krylov.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale(lib: Path, deps) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "glide_b200.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = ROOT / "_build"
    objdir.mkdir(exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"),
                    "--expt-relaxed-constexpr"]
    if ptxas_info:
        flags += ["-Xptxas", "-v"]
    objs = []
    for s in SOURCES:
        obj = objdir / (Path(s).stem + ".o")
        cmd = [nvcc()] + flags + ["-c", str(CSRC / s), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + objs + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas_info))
    sys.exit(0)
