"""The C ABI library loads and exports every declared entry point (no GPU)."""
import os
import re

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "include", "hpsi.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hpsi_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "hpsi_apply_h" in names and "hpsi_taylor_step" in names
    assert len(names) >= 20


def test_library_exports_and_binds_every_symbol():
    from hpsi import lib
    L = lib.load()
    for name in declared_functions():
        assert hasattr(L, name), f"{name} not exported"
        assert name in lib.SIGNATURES, f"{name} has no ctypes binding"


def test_errors_are_status_codes_without_gpu():
    """Argument validation answers before any device work."""
    import ctypes as C
    from hpsi import lib
    L = lib.load()
    d = lib.MeshDesc()
    d.np = 0
    h = C.c_void_p()
    assert L.hpsi_mesh_create(C.byref(d), C.byref(h)) == 1
    assert b"bad descriptor" in L.hpsi_last_error_string()
    assert L.hpsi_version().startswith(b"hpsi")


def test_python_package_has_no_cpu_fallback():
    """The host mirror only wraps the shared library: no compute in Python."""
    import inspect
    from hpsi import lib
    src = inspect.getsource(lib)
    assert "oracle" not in src
