"""Unstructured FV mesh: native face discovery and the structure-of-arrays layout.

build_mesh() is the counterpart of build_fvmesh_from_arrays
(mesh/mesh_reader.py:141-242) and _build_fvmesh_3d (:245-323): it takes the same
inputs (node coordinates, cell node lists, per-cell face node lists in 3D, the
boundary dict) and returns the same connectivity and geometry, computed by the C++
builder in libkcfd (kcfd_mesh_build). from_fvmesh() reads a reference FVMesh object.
The result also carries what the device path needs: the canonical CSR pattern of the
FVM matrix, the face -> CSR slot map, a face colouring and a cell colouring.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class Mesh:
    """Host-side SoA mesh (numpy). Face arrays are in reference face order."""

    def __init__(self):
        self.ndim = 2
        self.n_cells = self.n_faces = self.n_internal_faces = self.n_boundary_faces = 0
        self.owner = self.neighbour = None
        self.area = self.normal = self.fcenter = None
        self.ccenter = self.volume = None
        self.face_nodes = self.cell_faces = None
        self.nodes = self.cell_ptr = self.cell_nodes = None
        self.boundary_patches = {}
        self.indptr = self.indices = self.slot_on = self.slot_no = self.diag_slot = None
        self.face_color = self.cell_color = self.level_natural = None
        self.n_int_colors = self.n_bnd_colors = self.n_cell_colors = self.n_levels = 0

    @property
    def nnz(self):
        return int(self.indptr[-1])


def _flat(lists):
    lens = np.fromiter((len(x) for x in lists), dtype=np.int64, count=len(lists))
    flat = np.concatenate([np.asarray(x, dtype=np.int64) for x in lists]) if len(lists) else np.zeros(0, np.int64)
    return lens, flat


def build_fvmesh_from_arrays(node_coords, cell_node_list, boundary_faces_dict, cell_zone_map=None, ndim=2,
                             cell_face_node_list=None):
    """The reference's builder signature (mesh/mesh_reader.py:141-242); the cell zone
    map is kept on the mesh (cell_zones) and not used by the solvers."""
    m = build_mesh(node_coords, cell_node_list, boundary_faces_dict, ndim=ndim, cell_face_node_list=cell_face_node_list)
    m.cell_zones = dict(cell_zone_map or {})
    return m


def build_mesh(node_coords, cell_node_list, boundary_faces_dict, ndim=2, cell_face_node_list=None):
    """Build a Mesh with the reference builder's face order, owner/neighbour and geometry."""
    L = _lib.lib()
    nodes = np.ascontiguousarray(node_coords, dtype=np.float64)
    D = 3 if (ndim == 3 and cell_face_node_list is not None) else 2
    nodes = np.ascontiguousarray(nodes[:, :D])
    if isinstance(cell_node_list, np.ndarray) and cell_node_list.ndim == 2:
        n = cell_node_list.shape[0]
        cell_ptr = np.arange(0, n * cell_node_list.shape[1] + 1, cell_node_list.shape[1], dtype=np.int64)
        cell_nodes = np.ascontiguousarray(cell_node_list.reshape(-1), dtype=np.int64)
    else:
        lens, cell_nodes = _flat(cell_node_list)
        n = len(lens)
        cell_ptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(lens, out=cell_ptr[1:])
    cface = [None] * 4
    if D == 3:
        cfl = cell_face_node_list
        if isinstance(cfl, np.ndarray) and cfl.ndim == 3:
            nc, kf, kn = cfl.shape
            cface_ptr = np.arange(0, nc * kf + 1, kf, dtype=np.int64)
            cface_len = np.full(nc * kf, kn, dtype=np.int64)
            cface_off = np.arange(0, nc * kf * kn, kn, dtype=np.int64)
            cface_nodes = np.ascontiguousarray(cfl.reshape(-1), dtype=np.int64)
        else:
            cnt = np.fromiter((len(fl) for fl in cfl), dtype=np.int64, count=len(cfl))
            cface_ptr = np.zeros(len(cfl) + 1, dtype=np.int64)
            np.cumsum(cnt, out=cface_ptr[1:])
            faces = [f for fl in cfl for f in fl]
            cface_len, cface_nodes = _flat(faces)
            cface_off = np.zeros(len(faces), dtype=np.int64)
            if len(faces) > 1:
                np.cumsum(cface_len[:-1], out=cface_off[1:])
        cface = [cface_ptr, cface_len, cface_off, cface_nodes]
    names = list(boundary_faces_dict.keys())
    blists, bpatch = [], []
    for pi, nm in enumerate(names):
        lst = boundary_faces_dict[nm]
        if isinstance(lst, np.ndarray) and lst.ndim == 2:
            blists.extend(list(lst))
            bpatch.extend([pi] * lst.shape[0])
        else:
            blists.extend(lst)
            bpatch.extend([pi] * len(lst))
    if blists and all(len(b) == len(blists[0]) for b in blists):
        arr = np.asarray(blists, dtype=np.int64)
        blen = np.full(len(blists), arr.shape[1], dtype=np.int64)
        bnodes = np.ascontiguousarray(arr.reshape(-1))
    else:
        blen, bnodes = _flat(blists)
    bpatch = np.asarray(bpatch, dtype=np.int32)
    h = C.c_void_p()
    _lib.check(L.kcfd_mesh_build(D, len(nodes), _lib.ptr(nodes), n, _lib.ptr(cell_ptr), _lib.ptr(cell_nodes),
                                 *[_lib.ptr(x) for x in cface], len(blen), _lib.ptr(blen), _lib.ptr(bnodes),
                                 _lib.ptr(bpatch), C.byref(h)), "kcfd_mesh_build")
    try:
        info = np.zeros(10, dtype=np.int64)
        _lib.check(L.kcfd_mesh_info(h, info.ctypes.data_as(_lib.P_i64)), "kcfd_mesh_info")
        F, Fi, nnz, kfn, kcf = (int(v) for v in info[:5])
        m = Mesh()
        m.ndim = D
        m.n_cells, m.n_faces, m.n_internal_faces, m.n_boundary_faces = n, F, Fi, F - Fi
        m.n_int_colors, m.n_bnd_colors, m.n_cell_colors, m.n_levels = (int(v) for v in info[5:9])
        m.nodes = nodes
        m.cell_ptr, m.cell_nodes = cell_ptr, cell_nodes   # cell -> node lists (CSR), for export
        m.owner = np.empty(F, np.int64); m.neighbour = np.empty(F, np.int64)
        m.face_nodes = np.empty((F, kfn), np.int64); m.cell_faces = np.empty((n, kcf), np.int64)
        m.area = np.empty(F); m.normal = np.empty((F, D)); m.fcenter = np.empty((F, D))
        m.ccenter = np.empty((n, D)); m.volume = np.empty(n)
        face_patch = np.empty(F, np.int32)
        m.indptr = np.empty(n + 1, np.int32); m.indices = np.empty(nnz, np.int32)
        m.slot_on = np.empty(F, np.int32); m.slot_no = np.empty(F, np.int32); m.diag_slot = np.empty(n, np.int32)
        m.face_color = np.empty(F, np.int32); m.cell_color = np.empty(n, np.int32)
        m.level_natural = np.empty(n, np.int32)
        ex = _lib.MeshExport()
        for fld, arr in (("owner", m.owner), ("neighbour", m.neighbour), ("face_nodes", m.face_nodes),
                         ("cell_faces", m.cell_faces), ("area", m.area), ("normal", m.normal),
                         ("fcenter", m.fcenter), ("ccenter", m.ccenter), ("volume", m.volume),
                         ("face_patch", face_patch), ("indptr", m.indptr), ("indices", m.indices),
                         ("slot_on", m.slot_on), ("slot_no", m.slot_no), ("diag_slot", m.diag_slot),
                         ("face_color", m.face_color), ("cell_color", m.cell_color),
                         ("level_natural", m.level_natural)):
            setattr(ex, fld, arr.ctypes.data)
        _lib.check(L.kcfd_mesh_export(h, C.byref(ex)), "kcfd_mesh_export")
    finally:
        L.kcfd_mesh_free(h)
    # patches in order of first appearance among boundary faces (face-id order)
    bf = np.nonzero(m.neighbour < 0)[0]
    fp = face_patch[bf]
    labels = [names[p] if p >= 0 else "default" for p in fp.tolist()]
    patches = {}
    for fid, nm in zip(bf.tolist(), labels):
        patches.setdefault(nm, []).append(fid)
    m.boundary_patches = {k: np.asarray(v, dtype=np.int64) for k, v in patches.items()}
    m.face_patch_input = face_patch
    return m


def from_fvmesh(fv):
    """Read a reference FVMesh (AoS Face/Cell objects) into a Mesh with the CSR
    pattern and colourings, via the same native builder on the mesh's own faces."""
    ndim = getattr(fv, "ndim", 2)
    nodes = np.asarray(fv.nodes, dtype=np.float64)
    cells = [np.asarray(c.nodes) for c in fv.cells]
    bdict = {nm: [np.asarray(fv.faces[f].nodes) for f in fids] for nm, fids in fv.boundary_patches.items()}
    cfl = None
    if ndim == 3:
        cfl = [[np.asarray(fv.faces[f].nodes) for f in c.faces] for c in fv.cells]
    return build_mesh(nodes, cells, bdict, ndim=ndim, cell_face_node_list=cfl)
