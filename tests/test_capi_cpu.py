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
    assert L.sc_version() >= 10100


def test_python_structs_match_header_layout(tmp_path):
    """Every struct of the C ABI has the size and field offsets its ctypes mirror
    assumes (a probe compiled with the system C compiler against the header)."""
    import shutil
    import subprocess

    from simcraft_b200 import _capi

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest

        pytest.skip("no C compiler")
    structs = [getattr(_capi, n) for n in ("sc_pcg_options", "sc_pcg_stats", "sc_fluid_config", "sc_fluid_stats",
                                            "sc_diff_config")]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "simcraft_fluid_capi.h"', "int main(void) {"]
    for st in structs:
        lines.append(f'  printf("{st.__name__} size %zu\\n", sizeof({st.__name__}));')
        for f, _ in st._fields_:
            lines.append(f'  printf("{st.__name__} {f} %zu\\n", offsetof({st.__name__}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.check_call([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        name, field, val = line.split()
        got[(name, field)] = int(val)
    for st in structs:
        assert got[(st.__name__, "size")] == ctypes.sizeof(st), st.__name__
        for f, _ in st._fields_:
            assert got[(st.__name__, f)] == getattr(st, f).offset, (st.__name__, f)


def test_header_compiles_as_cxx_and_links(tmp_path):
    """A C++ caller includes the header (warnings as errors) and links the
    library; nothing is called, so no GPU is needed."""
    import shutil
    import subprocess

    from simcraft_b200 import build

    cxx = shutil.which("g++")
    if cxx is None:
        import pytest

        pytest.skip("no C++ compiler")
    build.build()
    src = tmp_path / "caller.cc"
    src.write_text('#include "simcraft_fluid_capi.h"\n'
                   "int main(int argc, char**) {\n"
                   "  sc_pcg_options o;\n"
                   "  if (argc > 5) sc_pcg_default_options(&o);\n"
                   "  return argc > 5 ? sc_version() : 0;\n"
                   "}\n")
    exe = tmp_path / "caller"
    libdir = os.path.dirname(build.LIB)
    subprocess.check_call([cxx, "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                           str(src), "-o", str(exe), "-L", libdir, "-lsimcraft_fluid", "-Wl,-rpath," + libdir])
    assert exe.exists()


def test_null_handles_are_rejected():
    """Host-side fault injection at the boundary: every exported function that
    takes a handle, given NULL for it (and ones, zeros or NULLs for the rest),
    returns SC_ERR_INVALID (a status), 0 (a count) or nothing, and touches
    neither the handle nor the device."""
    import ctypes

    from simcraft_b200 import _capi

    L = _capi.lib()
    probed = 0
    for name, (rt, at) in sorted(_capi.SIGNATURES.items()):
        if not at or at[0] is not ctypes.c_void_p:
            continue
        args = [1 if t in (ctypes.c_int, ctypes.c_int64, ctypes.c_uint32) else 1.0 if t is ctypes.c_double else None
                for t in at]
        r = getattr(L, name)(*args)
        if rt is None or rt is ctypes.c_void_p:  # nothing, or a NULL pointer
            assert r is None, name
        elif rt is ctypes.c_char_p:
            assert r == b"no context", name
        elif name in ("sc_fluid_num_particles", "sc_diff_last_pcg_iterations"):
            assert r == 0, name
        else:
            assert r == -1, (name, r)  # SC_ERR_INVALID
        probed += 1
    assert probed >= 50


def test_context_creation_fails_cleanly_without_a_device():
    import ctypes

    import torch

    from simcraft_b200 import _capi

    if torch.cuda.is_available():
        import pytest

        pytest.skip("a device is present")
    h = ctypes.c_void_p(1234)
    assert _capi.lib().sc_context_create(0, ctypes.byref(h)) == -2  # SC_ERR_CUDA
    assert h.value is None
    assert _capi.lib().sc_context_create(0, None) == -1
