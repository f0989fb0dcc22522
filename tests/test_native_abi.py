"""The C-ABI library loads and exports every symbol the header declares.

CPU-only: no compute call is made; argument validation paths that return
before any CUDA call are exercised.
"""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        for m in re.finditer(r"^\s*(?:int|const char\*|long long|size_t)\s+(glide_\w+)\s*\(", txt, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared()
    assert "glide_residual" in names and "glide_fascd_vcycle" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    from glide_b200 import _native as N
    if not N.lib_path().exists():
        pytest.skip("native library not built")
    lib = C.CDLL(str(N.lib_path()))
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(N.SYMBOLS) <= set(_declared())


def test_argument_validation_without_gpu():
    from glide_b200 import _native as N
    if not N.lib_path().exists():
        pytest.skip("native library not built")
    lib = N.load()
    assert lib.glide_version().decode().startswith("glide_b200")
    a = N.LevelArgs()
    a.ny, a.nx, a.nb, a.dtype = 8, 8, 1, 7
    assert lib.glide_residual(C.byref(a), None, None, None, None, None, None, None) == -1   # dtype
    a.dtype = N.F64
    assert lib.glide_residual(C.byref(a), None, None, None, None, None, None, None) == -3   # null state
    a.ny = 0
    assert lib.glide_residual(C.byref(a), None, None, None, None, None, None, None) == -2   # shape
    assert lib.glide_restrict(5, 0, 0, None, None, 4, 4, 1, None) == -1
    assert lib.glide_fascd_vcycle(None, 0, 0, 1, None, None) == -3
    # a problem whose fields reach 2^31 elements is refused before any launch
    a.ny, a.nx = 50_000, 50_000
    assert lib.glide_residual(C.byref(a), None, None, None, None, None, None, None) == -5   # too large
