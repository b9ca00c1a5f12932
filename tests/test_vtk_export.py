"""VTU snapshot export (kcfd.vtk_exporter, the reference's mesh/vtk_exporter.py:17-115).

Host code only. The reference writes through meshio, which is not installed here, so
its own call returns without writing; these tests restate its layout rules and read
the written file back: points padded to 3D, cells grouped by type in order of first
appearance (mesh order inside a group), connectivity / offsets / VTK type codes,
and cell fields reordered into the same order (arrays of another length skipped)."""
import base64
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from conftest import load_golden, golden_inputs
from kcfd import mesh as km, meshgen
from kcfd.vtk_exporter import export_mesh_to_vtu

VTK_CODE = {(2, 3): 5, (2, 4): 9, (3, 8): 12, (3, 4): 10, (3, 6): 13, (3, 5): 14}
DT = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}


def _read(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    out = {}
    for da in piece.iter("DataArray"):
        dt = DT[da.get("type")]
        if da.get("format") == "ascii":
            a = np.array(da.text.split(), dtype=dt)
        else:
            raw = base64.b64decode(da.text)
            nb = int(np.frombuffer(raw[:8], dtype="<u8")[0])
            a = np.frombuffer(raw[8:8 + nb], dtype=np.dtype(dt).newbyteorder("<")).astype(dt)
        k = int(da.get("NumberOfComponents", "1"))
        out[da.get("Name")] = a.reshape(-1, k) if k > 1 else a
    return int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells")), out


def _expected_order(cells, ndim):
    kinds = [VTK_CODE.get((ndim, len(c)), 7) for c in cells]
    first = {}
    for k in kinds:
        first.setdefault(k, len(first))
    return sorted(range(len(cells)), key=lambda i: (first[kinds[i]], i)), kinds


def _meshes():
    d = load_golden("mesh_hybrid")
    nodes, cells, bdict, cfl = golden_inputs(d)
    yield "hybrid", km.build_mesh(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl), \
        [list(c) for c in cells], int(d["ndim"])
    d = load_golden("mesh_tri")
    nodes, cells, bdict, cfl = golden_inputs(d)
    yield "tri", km.build_mesh(nodes, cells, bdict, ndim=2), [list(c) for c in cells], 2
    nodes, cells, cf, bd = meshgen.hex_box_arrays(1.0, 1.0, 1.0, 3, 2, 2)
    yield "hex", km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf), [list(c) for c in cells], 3


@pytest.mark.parametrize("ascii", [False, True])
def test_vtu_layout_and_fields(tmp_path, ascii):
    for name, m, cells, ndim in _meshes():
        n = m.n_cells
        rng = np.random.default_rng(0)
        p = rng.standard_normal(n)
        U = rng.standard_normal((n, ndim))
        path = tmp_path / f"{name}.vtu"
        export_mesh_to_vtu(m, str(path), {"p": p, "U": U, "short": p[:-1]}, ascii=ascii)
        npts, ncells, arr = _read(path)
        assert (npts, ncells) == (len(m.nodes), n)
        pts = arr["Points"]
        np.testing.assert_array_equal(pts[:, :m.nodes.shape[1]], m.nodes)
        if m.nodes.shape[1] == 2:
            assert not pts[:, 2].any()
        order, kinds = _expected_order(cells, ndim)
        np.testing.assert_array_equal(arr["types"], [kinds[i] for i in order])
        np.testing.assert_array_equal(arr["connectivity"], np.concatenate([cells[i] for i in order]))
        np.testing.assert_array_equal(arr["offsets"], np.cumsum([len(cells[i]) for i in order]))
        np.testing.assert_array_equal(arr["p"], p[order])
        np.testing.assert_array_equal(arr["U"], U[order])
        assert "short" not in arr
        if name == "hybrid":
            assert len(set(kinds)) == 2


def test_vtu_rejects_3d_cells_without_a_type(tmp_path):
    nodes, cells, cf, bd = meshgen.hex_box_arrays(1.0, 1.0, 1.0, 1, 1, 1)
    m = km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
    m.cell_ptr = np.array([0, 7])
    with pytest.raises(ValueError):
        export_mesh_to_vtu(m, str(tmp_path / "bad.vtu"))


def test_vtu_from_a_reference_shaped_mesh_and_input_json(tmp_path):
    """An FVMesh-shaped object (nodes, cells[i].nodes) gives the same file; the
    parameter JSON turns numpy values into plain JSON."""
    import json
    from types import SimpleNamespace
    from kcfd.vtk_exporter import export_input_json
    d = load_golden("mesh_hybrid")
    nodes, cells, bdict, cfl = golden_inputs(d)
    m = km.build_mesh(nodes, cells, bdict, ndim=3, cell_face_node_list=cfl)
    fv = SimpleNamespace(nodes=np.asarray(nodes, dtype=np.float64), ndim=3,
                         cells=[SimpleNamespace(nodes=list(c)) for c in cells], n_cells=len(cells))
    p = np.arange(len(cells), dtype=np.float64)
    export_mesh_to_vtu(m, str(tmp_path / "a.vtu"), {"p": p})
    export_mesh_to_vtu(fv, str(tmp_path / "b.vtu"), {"p": p})
    assert (tmp_path / "a.vtu").read_text() == (tmp_path / "b.vtu").read_text()
    export_input_json({"n": np.int64(3), "x": np.float32(0.5), "v": np.arange(3), "t": (1, np.int32(2))},
                      str(tmp_path / "in.json"))
    assert json.loads((tmp_path / "in.json").read_text()) == {"n": 3, "x": 0.5, "v": [0, 1, 2], "t": [1, 2]}
