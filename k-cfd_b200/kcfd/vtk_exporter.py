"""Field snapshots as VTK XML unstructured grids (.vtu), for ParaView.

Public API as in the reference (mesh/vtk_exporter.py:17-115):
export_mesh_to_vtu(mesh, filepath, cell_data=None). The reference hands the mesh to
meshio; this writer produces the same grid without it:

- points: the mesh nodes, 2D meshes padded with z = 0 (vtk_exporter.py:38-47);
- cells grouped into blocks by type, the blocks in order of the type's first
  appearance and the cells of a block in mesh order (vtk_exporter.py:50-90): 2D by
  node count 4 quad, 3 triangle, else polygon; 3D 8 hexahedron, 4 tetra, 6 wedge,
  5 pyramid (a 3D cell of another node count has no fixed VTK type and is rejected);
- cell_data: every array whose first dimension is the cell count, as float64,
  reordered into the block order (vtk_exporter.py:92-112); other arrays are skipped,
  as in the reference. Device tensors are copied to the host.

Arrays are written inline as base64 binary (VTK's 'binary' format, UInt64 headers,
little endian) or, with ascii=True, as text. The mesh may be a kcfd Mesh or an
object shaped like the reference's FVMesh (nodes, cells[i].nodes, ndim).
export_input_json(params, filepath) saves a parameter dict as the reference's does
(vtk_exporter.py:118-146): numpy scalars and arrays as plain JSON, indent 2.
"""
from __future__ import annotations

import base64

import numpy as np

_TYPES_2D = {4: ("quad", 9), 3: ("triangle", 5)}
_TYPES_3D = {8: ("hexahedron", 12), 4: ("tetra", 10), 6: ("wedge", 13), 5: ("pyramid", 14)}
_POLYGON = ("polygon", 7)


def _host(a):
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    return np.asarray(a)


def _cell_type(k, ndim):
    if ndim == 2:
        return _TYPES_2D.get(k, _POLYGON)
    if k not in _TYPES_3D:
        raise ValueError(f"export_mesh_to_vtu: a 3D cell with {k} nodes has no fixed VTK cell type")
    return _TYPES_3D[k]


def _cell_lists(mesh):
    """(nodes, ptr, flat): node coordinates and the cell -> node lists as CSR."""
    nodes = getattr(mesh, "nodes", None)
    if getattr(mesh, "cell_ptr", None) is not None and nodes is not None:
        return np.asarray(nodes, dtype=np.float64), np.asarray(mesh.cell_ptr, np.int64), \
            np.asarray(mesh.cell_nodes, np.int64)
    cells = getattr(mesh, "cells", None)
    if cells is None or nodes is None:
        raise ValueError("export_mesh_to_vtu: the mesh carries no node coordinates / cell node lists")
    lists = [np.asarray(c.nodes, dtype=np.int64) for c in cells]
    ptr = np.zeros(len(lists) + 1, dtype=np.int64)
    np.cumsum([len(c) for c in lists], out=ptr[1:])
    flat = np.concatenate(lists) if lists else np.zeros(0, np.int64)
    return np.asarray(nodes, dtype=np.float64), ptr, flat


def vtu_blocks(mesh):
    """(order, types): cell indices in VTU order (blocks by first appearance of their
    type, mesh order inside a block) and the VTK type code of each written cell."""
    nodes, ptr, _ = _cell_lists(mesh)
    k = np.diff(ptr)
    nd = 2 if (getattr(mesh, "ndim", 2) == 2 or nodes.shape[1] == 2) else 3
    counts = np.unique(k)
    code_of = {int(c): _cell_type(int(c), nd)[1] for c in counts}
    codes = np.zeros(len(k), dtype=np.uint8)
    for c, code in code_of.items():
        codes[k == c] = code
    # blocks in order of each type's first appearance (node counts sharing a type,
    # such as 2D polygons, share a block)
    uniq, first_idx = np.unique(codes, return_index=True)
    rank_of = np.empty(256, dtype=np.int64)
    rank_of[uniq[np.argsort(first_idx)]] = np.arange(len(uniq))
    order = np.argsort(rank_of[codes], kind="stable")
    return order, codes[order]


def _encode(arr, ascii):
    arr = np.ascontiguousarray(arr)
    if ascii:
        if arr.dtype.kind == "f":
            return " ".join(repr(float(v)) for v in arr.reshape(-1))
        return " ".join(str(int(v)) for v in arr.reshape(-1))
    raw = arr.astype(arr.dtype.newbyteorder("<"), copy=False).tobytes()
    return base64.b64encode(np.uint64(len(raw)).tobytes() + raw).decode("ascii")


_VTK_DTYPES = {np.dtype(np.float64): "Float64", np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8"}


def _data_array(name, arr, ncomp, ascii):
    fmt = "ascii" if ascii else "binary"
    comp = f' NumberOfComponents="{ncomp}"' if ncomp > 1 else ""
    return (f'<DataArray type="{_VTK_DTYPES[arr.dtype]}" Name="{name}"{comp} format="{fmt}">'
            f"{_encode(arr, ascii)}</DataArray>")


def export_mesh_to_vtu(mesh, filepath: str, cell_data: dict = None, ascii: bool = False):
    """Write the mesh (and cell fields) to a .vtu file (mesh/vtk_exporter.py:17)."""
    nodes, ptr, cn = _cell_lists(mesh)
    pts = np.zeros((nodes.shape[0], 3))
    pts[:, : min(3, nodes.shape[1])] = nodes[:, :3]
    order, codes = vtu_blocks(mesh)
    lens = np.diff(ptr)[order]
    offsets = np.cumsum(lens).astype(np.int64)
    # gather each written cell's node run: entry e of the output sits at
    # ptr[order[c]] + (e - start of c in the output)
    starts_out = offsets - lens
    idx = np.repeat(ptr[:-1][order] - starts_out, lens) + np.arange(int(offsets[-1]) if len(offsets) else 0)
    conn = cn[idx]
    n = len(ptr) - 1
    out = ['<?xml version="1.0"?>',
           '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
           "<UnstructuredGrid>", f'<Piece NumberOfPoints="{pts.shape[0]}" NumberOfCells="{n}">',
           "<Points>", _data_array("Points", pts.reshape(-1), 3, ascii), "</Points>",
           "<Cells>", _data_array("connectivity", conn, 1, ascii), _data_array("offsets", offsets, 1, ascii),
           _data_array("types", codes, 1, ascii), "</Cells>"]
    fields = []
    for name, values in (cell_data or {}).items():
        arr = _host(values).astype(np.float64)
        if arr.shape[0] != n:
            continue
        fields.append((name, arr[order]))
    if fields:
        out.append("<CellData>")
        for name, arr in fields:
            ncomp = 1 if arr.ndim == 1 else int(np.prod(arr.shape[1:]))
            out.append(_data_array(name, arr.reshape(-1), ncomp, ascii))
        out.append("</CellData>")
    out += ["</Piece>", "</UnstructuredGrid>", "</VTKFile>"]
    with open(filepath, "w") as f:
        f.write("\n".join(out) + "\n")


def export_input_json(params: dict, filepath: str):
    """Save a parameter dict as JSON (mesh/vtk_exporter.py:118-146)."""
    import json

    def convert(obj):
        if isinstance(obj, np.integer):
            return int(obj)
        if isinstance(obj, np.floating):
            return float(obj)
        if isinstance(obj, np.ndarray):
            return obj.tolist()
        if isinstance(obj, dict):
            return {k: convert(v) for k, v in obj.items()}
        if isinstance(obj, (list, tuple)):
            return [convert(v) for v in obj]
        return obj

    with open(filepath, "w", encoding="utf-8") as f:
        json.dump(convert(params), f, indent=2, ensure_ascii=False)
