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
