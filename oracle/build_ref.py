"""Build ``oracle/_ref/libglide_ref.so`` from the reference's CUDA sources.

Test infrastructure: compiles the reference kernels where they lie
(``<reference>/glide/cuda/*.cu``; ``<reference>`` is ``$GLIDE_REFERENCE``, else
the ``reference`` directory beside this repository) together with the host launchers in
``oracle/ref_ice_shim.cu`` / ``oracle/ref_util_shim.cu``.  The ice kernels get
``--use_fast_math`` like the reference's NVRTC build (glide/kernels.py:72);
the transfer kernels do not (glide/kernels.py:63).  Outputs go to
``oracle/_ref/`` only.  Skipped when the reference tree is absent.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIB = OUT / "libglide_ref.so"
# the reference checkout: GLIDE_REFERENCE, else a "reference" directory beside this repository
REF_ROOT = Path(os.environ.get("GLIDE_REFERENCE", HERE.parent.parent / "reference"))
REF_CUDA = REF_ROOT / "glide" / "cuda"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def build(force=False):
    if not REF_CUDA.exists():
        return None
    srcs = [HERE / "ref_ice_shim.cu", HERE / "ref_util_shim.cu"] + sorted(REF_CUDA.glob("*.cu"))
    if LIB.exists() and not force and all(s.stat().st_mtime <= LIB.stat().st_mtime for s in srcs):
        return LIB
    OUT.mkdir(exist_ok=True)
    nvcc = "/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else "nvcc"
    base = [nvcc] + ARCH + ["-O3", "-Xcompiler", "-fPIC", "-I", str(REF_CUDA), "-w"]
    o1, o2 = OUT / "ref_ice.o", OUT / "ref_util.o"
    subprocess.run(base + ["--use_fast_math", "-c", str(HERE / "ref_ice_shim.cu"), "-o", str(o1)], check=True)
    subprocess.run(base + ["-c", str(HERE / "ref_util_shim.cu"), "-o", str(o2)], check=True)
    subprocess.run([nvcc] + ARCH + ["-shared", "-o", str(LIB), str(o1), str(o2), "-lcudart"], check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
