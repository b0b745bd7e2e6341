"""CPU-only checks of the C-ABI library: it loads without a GPU and exports
every symbol that include/simcraft_fluid_capi.h declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "simcraft_fluid_capi.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sc_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_declared_symbols():
    from simcraft_b200 import build

    build.build()
    lib = ctypes.CDLL(build.LIB)
    names = declared_symbols()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from simcraft_b200 import _capi

    names = set(declared_symbols())
    assert names <= set(_capi.SIGNATURES), sorted(names - set(_capi.SIGNATURES))


def test_status_strings_without_gpu():
    from simcraft_b200 import _capi

    L = _capi.lib()
    assert L.sc_status_string(0) == b"ok"
    assert L.sc_status_string(-6) == b"device wait timed out"
    assert L.sc_version() >= 10000
