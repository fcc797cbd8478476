"""The C-ABI library loads and exports every entry point of include/tmx.h.

No compute call is made (no GPU needed)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if not hdr.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", hdr)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(tmx_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from costuum_b200 import _lib
    path = _lib.LIB_PATH
    if not os.path.exists(path):
        from costuum_b200 import build
        build.build()
    return ctypes.CDLL(path)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "tmx_create" in names and "tmx_tmatrix_batch" in names
    assert len(names) >= 10


def test_library_exports_all(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from costuum_b200 import _lib
    missing = [n for n in declared_symbols() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_pure_functions(lib):
    # tmx_tmatrix_size needs no device: 4 nmax^2 + 4 sum_{m>=1} (nmax+1-m)^2
    lib.tmx_tmatrix_size.restype = ctypes.c_int64
    lib.tmx_tmatrix_size.argtypes = [ctypes.c_int32]
    assert lib.tmx_tmatrix_size(1) == 4 + 4
    assert lib.tmx_tmatrix_size(3) == 36 + 4 * (9 + 4 + 1)
    import oracle as O
    for n in (5, 17, 40):
        assert lib.tmx_tmatrix_size(n) == O.tmatrix_size(n)
