"""The C-ABI library loads and exports every entry point include/kcfd.h declares.

Host only: no device call is made."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "kcfd.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:int|void)\s+(kcfd_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "kcfd_solver_solve" in names and "kcfd_mesh_build" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    from kcfd import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"
    # the Python binding knows every declared function too
    assert set(declared_functions()) <= set(_lib.SIGNATURES), set(declared_functions()) - set(_lib.SIGNATURES)


def test_last_error_roundtrip():
    from kcfd import _lib
    L = _lib.lib()
    rc = L.kcfd_mesh_build(5, 0, None, 0, None, None, None, None, None, None, 0, None, None, None,
                           ctypes.byref(ctypes.c_void_p()))
    assert rc == _lib.BAD_INPUT
    assert "ndim" in _lib.last_error()


def test_graph_entry_points_reject_null_arguments():
    """The graph entry points check their arguments before any CUDA call."""
    from kcfd import _lib
    L = _lib.lib()
    assert L.kcfd_graph_capture_begin(None) == _lib.BAD_INPUT
    assert L.kcfd_graph_launch(None, None) == _lib.BAD_INPUT
    assert L.kcfd_graph_capture_end(None, None) == _lib.BAD_INPUT
    L.kcfd_graph_destroy(None)
    assert "kcfd_graph" in _lib.last_error()
