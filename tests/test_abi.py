"""The C ABI library loads and exports every symbol include/pantometry_gpu.h declares (no GPU
needed: nothing here calls into the device)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pantometry_gpu.h")
LIB = os.path.join(ROOT, "pantometry_b200", "libpantometry_b200.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pm_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        import pantometry_b200.build as b

        b.build()
    return ctypes.CDLL(LIB)


def test_header_declares_the_domain_surface():
    names = declared_functions()
    for prefix in ("pm_heat_", "pm_hall_", "pm_room_", "pm_tube_", "pm_bar_", "pm_cavity_"):
        for verb in ("create", "step", "ledger", "checkpoint", "restore", "destroy", "set_tolerance"):
            assert prefix + verb in names, prefix + verb


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_declares_every_header_symbol():
    from pantometry_b200 import _native as N

    declared = set(declared_functions())
    bound = set(N.SIGNATURES) | set(N.OPTIONAL_SIGNATURES)
    assert declared <= bound, sorted(declared - bound)


def test_status_strings_without_a_device(lib):
    lib.pm_status_string.restype = ctypes.c_char_p
    assert lib.pm_status_string(3) == b"violation"
    lib.pm_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.pm_version()


def test_entry_build_in_a_fresh_interpreter():
    """build() as the driver calls it: a new process, nothing imported beforehand."""
    import subprocess
    import sys

    r = subprocess.run([sys.executable, "-c", "import __graft_entry__ as g; g.build()"], cwd=ROOT,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c", "-std=c11"), ("c++", "-std=c++11"), ("c++", "-std=c++17")])
def test_header_compiles_as_c_and_cpp(tmp_path, lang, std):
    """A Rust `bindgen`, a C host or a C++ host each include the header on its own: it must
    compile alone, warning-free, in C and in C++."""
    import shutil
    import subprocess

    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    src = tmp_path / ("use." + ("c" if lang == "c" else "cpp"))
    src.write_text('#include "pantometry_gpu.h"\n'
                   "int main(void) { pm_violation v; pm_ledger l; (void)v; (void)l;\n"
                   "  return (int)sizeof(pm_status_string(PM_OK)) - (int)sizeof(const char*); }\n")
    r = subprocess.run([cc, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
