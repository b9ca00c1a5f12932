"""The ctypes mirror agrees with include/kcfd.h, checked on the host without a device:

- every declared entry point has the same number of parameters, of the same kinds
  (pointer, int32, int64, double, float), and the same return type in the Python table;
- every struct the header defines has the size and field offsets of its ctypes mirror,
  taken from a probe compiled with gcc against the header itself."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "kcfd.h")


def _header_source():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _c_kind(param):
    p = param.strip()
    if "*" in p:
        return "ptr"
    t = p.replace("const", "").split()[0]
    return {"int": "i32", "int32_t": "i32", "int64_t": "i64", "double": "f64", "float": "f32"}.get(t, "?" + t)


def _py_kind(a):
    if a in (C.c_void_p, C.c_char_p) or (isinstance(a, type) and issubclass(a, C._Pointer)):
        return "ptr"
    return {C.c_int32: "i32", C.c_int64: "i64", C.c_double: "f64", C.c_float: "f32"}.get(a, "?" + repr(a))


def test_entry_point_signatures_match_the_header():
    from kcfd import _lib
    protos = re.findall(r"^\s*(int|void)\s+(kcfd_\w+)\s*\(([^;]*?)\)\s*;", _header_source(), flags=re.M)
    assert len(protos) >= 50
    bad = []
    for ret, name, params in protos:
        restype, argtypes = _lib.SIGNATURES[name]
        ps = [] if params.strip() in ("", "void") else params.split(",")
        if [_c_kind(p) for p in ps] != [_py_kind(a) for a in argtypes]:
            bad.append((name, [_c_kind(p) for p in ps], [_py_kind(a) for a in argtypes]))
        if (ret == "int") != (restype in (C.c_int, C.c_int32)):
            bad.append((name, ret, restype))
    assert not bad, bad


def _mirrors():
    from kcfd import _lib
    from kcfd.batch import BatchOpts
    from kcfd.device_mesh import BCDesc, DMeshDesc
    return {"kcfd_mesh_export_t": _lib.MeshExport, "kcfd_csr_t": _lib.Csr, "kcfd_solver_opts_t": _lib.SolverOpts,
            "kcfd_batch_opts_t": BatchOpts, "kcfd_dmesh_t": DMeshDesc, "kcfd_bc_t": BCDesc,
            "kcfd_mom_params_t": _lib.MomParams, "kcfd_tf_params_t": _lib.TfParams,
            "kcfd_face_layout_t": _lib.FaceLayout, "kcfd_amg_opts_t": _lib.AmgOpts}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layouts_match_the_header(tmp_path):
    mirrors = _mirrors()
    declared = set(re.findall(r"^\}\s*(kcfd_\w+_t)\s*;", _header_source(), flags=re.M))
    assert declared == set(mirrors), declared ^ set(mirrors)
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "kcfd.h"', "int main(void) {"]
    for tname, cls in mirrors.items():
        lines.append(f'  printf("{tname} size %zu\\n", sizeof({tname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{tname} {fname} %zu\\n", offsetof({tname}, {fname}));')
    lines += ["  return 0;", "}"]
    probe = tmp_path / "layout.c"
    probe.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), str(probe), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        t, f, v = ln.split()
        got[(t, f)] = int(v)
    for tname, cls in mirrors.items():
        assert got[(tname, "size")] == C.sizeof(cls), tname
        for fname, _ in cls._fields_:
            assert got[(tname, fname)] == getattr(cls, fname).offset, (tname, fname)
