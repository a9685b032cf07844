"""The C-ABI library loads on a CPU-only machine and exports every function include/emfem.h declares."""
import ctypes
import os
import re

from emerge_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "emfem.h")).read()
    return sorted(set(re.findall(r"^int\s+(emfem_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared()) <= set(_lib.exported_symbols())


def test_host_only_calls():
    L = _lib.lib()
    assert L.emfem_version() >= 10000
    buf = ctypes.create_string_buffer(64)
    assert L.emfem_last_error(buf, 64) == 0
    sz = ctypes.c_size_t()
    assert L.emfem_krylov_workspace_size(1000, 20000, 3, 0, ctypes.byref(sz)) == 0 and sz.value > 0
    assert L.emfem_krylov_workspace_size(1000, 20000, 65, 0, ctypes.byref(sz)) == _lib.ERR_INVALID_ARG
