"""Golden VTI file from the reference's own writer (glide/io.py:20-137).

Run where the reference tree is present (path in GLIDE_REFERENCE, else the
``reference`` directory beside this repository).  CuPy and h5py are absent there, so ``glide/io.py`` is
loaded with stand-in ``cupy`` (``asnumpy`` = ``numpy.asarray``; the writer
only moves arrays to the host with it) and ``h5py`` (empty; only the HDF5
writer, not exercised here, uses it) modules.  Writes
``tests/golden/reference_write_vti.vti`` from ``vti_fields()``.
"""
import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def vti_fields():
    rng = np.random.default_rng(21)
    ny, nx = 5, 7
    return {"H": rng.random((ny, nx)).astype(np.float32) * 100,
            "vel": [rng.standard_normal((ny, nx)).astype(np.float32), rng.standard_normal((ny, nx)).astype(np.float32)]}


def main():
    ref = Path(os.environ.get("GLIDE_REFERENCE", HERE.parents[2] / "reference")) / "glide" / "io.py"
    cp = types.ModuleType("cupy")
    cp.asnumpy = np.asarray
    sys.modules.setdefault("cupy", cp)
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    spec = importlib.util.spec_from_file_location("reference_glide_io", ref)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.write_vti(HERE / "reference_write_vti.vti", vti_fields(), 1500.0, time_value=3.5)
    print("wrote", HERE / "reference_write_vti.vti")


if __name__ == "__main__":
    main()
