"""Device-resident mesh (kcfd_dmesh_t) and boundary conditions (kcfd_bc_t).

Faces are reordered colour by colour: internal faces first (by colour, then by
reference face id), then boundary faces (by colour, then id). No two faces of one
colour share a cell, so each colour's owner/neighbour scatter is conflict-free.
face_ref maps device faces back to reference face ids (mass flux output order).

Per-face geometry used by the kernels is computed once here with the reference's
formulas: gc = dN/(dO+dN) (models/single_phase.py:380-388), |d_PN| and
d_orth = max(|d_PN . n|, 0.1 |d_PN|) (:166-175), |x_f - x_P| on boundary faces (:197).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

BC_TYPES = {"zero_gradient": 0, "dirichlet": 1, "neumann": 2}


class DMeshDesc(C.Structure):
    _fields_ = [("ndim", C.c_int32), ("n_cells", C.c_int32), ("n_faces", C.c_int32), ("n_internal", C.c_int32)] + \
               [(n, C.c_void_p) for n in ("owner", "neigh", "area", "normal", "fcenter", "ccenter", "volume", "gc",
                                          "dlen", "dorth", "slot_on", "slot_no", "diag_slot", "indptr", "face_ref",
                                          "color_ptr")] + \
               [("n_colors_int", C.c_int32), ("n_colors_bnd", C.c_int32), ("cf_ptr", C.c_void_p),
                ("cf_face", C.c_void_p)]


class BCDesc(C.Structure):
    _fields_ = [("u_type", C.c_void_p), ("u_val", C.c_void_p), ("p_type", C.c_void_p), ("p_val", C.c_void_p),
                ("has_p_dirichlet", C.c_int32), ("pad", C.c_int32)]


def device_layout(mesh):
    """Host arrays of the device face layout (kcfd_mesh_device_layout, no device call):
    faces colour by colour, internal colours first, by reference face id inside a
    colour; owner / neighbour / geometry gathered in that order; gc, dlen, dorth; the
    faces of each cell in ascending reference id as device face indices."""
    L = _lib.lib()
    D, n, F, Fi = mesh.ndim, mesh.n_cells, mesh.n_faces, mesh.n_internal_faces
    nc = mesh.n_int_colors + mesh.n_bnd_colors
    kcf = mesh.cell_faces.shape[1]
    out = {"order": np.empty(F, np.int64), "color_ptr": np.empty(nc + 1, np.int32), "owner": np.empty(F, np.int32),
           "neigh": np.empty(Fi, np.int32), "area": np.empty(F), "normal": np.empty((F, D)),
           "fcenter": np.empty((F, D)), "gc": np.empty(Fi), "dlen": np.empty(F), "dorth": np.empty(Fi),
           "slot_on": np.empty(Fi, np.int32), "slot_no": np.empty(Fi, np.int32), "cf_ptr": np.empty(n + 1, np.int32),
           "cf_face": np.empty(max(n * kcf, 1), np.int32)}
    lay = _lib.FaceLayout(**{k: v.ctypes.data for k, v in out.items()})

    def arg(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    keep = []
    _lib.check(L.kcfd_mesh_device_layout(
        D, n, F, Fi, nc, kcf, arg(mesh.owner, np.int64), arg(mesh.neighbour, np.int64),
        arg(mesh.face_color, np.int32), arg(mesh.ccenter, np.float64), arg(mesh.fcenter, np.float64),
        arg(mesh.normal, np.float64), arg(mesh.area, np.float64), arg(mesh.slot_on, np.int32),
        arg(mesh.slot_no, np.int32), arg(mesh.cell_faces, np.int64), C.byref(lay)), "kcfd_mesh_device_layout")
    out["cf_face"] = out["cf_face"][:int(out["cf_ptr"][n])]
    return out


class DeviceMesh:
    def __init__(self, mesh, device="cuda"):
        torch = _lib.require_cuda()
        self.host = mesh
        self.ndim = D = mesh.ndim
        self.n_cells = n = mesh.n_cells
        F, Fi = mesh.n_faces, mesh.n_internal_faces
        self.n_faces, self.n_internal, self.n_boundary = F, Fi, F - Fi
        lay = device_layout(mesh)
        order, color_ptr = lay["order"], lay["color_ptr"]
        nci, ncb = mesh.n_int_colors, mesh.n_bnd_colors
        assert color_ptr[nci] == Fi and color_ptr[-1] == F
        self.face_ref = order
        self.color_ptr = color_ptr
        # boundary face bookkeeping: device boundary slot of each (patch, local index)
        bref = order[Fi:]
        pos_of_ref = np.full(F, -1, dtype=np.int64)
        pos_of_ref[bref] = np.arange(F - Fi)
        self.patch_slots = {nm: pos_of_ref[fids] for nm, fids in mesh.boundary_patches.items()}

        def dev(a, dt):
            return torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(device)

        i32, f64 = np.int32, np.float64
        self.t = {
            "owner": dev(lay["owner"], i32), "neigh": dev(lay["neigh"], i32), "area": dev(lay["area"], f64),
            "normal": dev(lay["normal"], f64), "fcenter": dev(lay["fcenter"], f64), "ccenter": dev(mesh.ccenter, f64),
            "volume": dev(mesh.volume, f64), "gc": dev(lay["gc"], f64), "dlen": dev(lay["dlen"], f64),
            "dorth": dev(lay["dorth"], f64), "slot_on": dev(lay["slot_on"], i32), "slot_no": dev(lay["slot_no"], i32),
            "diag_slot": dev(mesh.diag_slot, i32), "indptr": dev(mesh.indptr, i32),
            "indices": dev(mesh.indices, i32), "face_ref": dev(order, i32),
            # faces of each cell, ascending reference face id, as device face indices
            "cf_ptr": dev(lay["cf_ptr"], i32), "cf_face": dev(lay["cf_face"], i32),
        }
        self._color_ptr_np = np.ascontiguousarray(color_ptr, dtype=np.int32)
        d = DMeshDesc()
        d.ndim, d.n_cells, d.n_faces, d.n_internal = D, n, F, Fi
        for k in ("owner", "neigh", "area", "normal", "fcenter", "ccenter", "volume", "gc", "dlen", "dorth",
                  "slot_on", "slot_no", "diag_slot", "indptr", "face_ref"):
            setattr(d, k, self.t[k].data_ptr())
        d.color_ptr = self._color_ptr_np.ctypes.data
        d.n_colors_int, d.n_colors_bnd = nci, ncb
        d.cf_ptr, d.cf_face = self.t["cf_ptr"].data_ptr(), self.t["cf_face"].data_ptr()
        self.desc = d
        self.nnz = mesh.nnz
        self.cell_color = mesh.cell_color
        self.level_natural = mesh.level_natural

    def to_reference_faces(self, face_values):
        """Device-order face array -> reference face order (host numpy)."""
        v = face_values.detach().cpu().numpy() if hasattr(face_values, "detach") else np.asarray(face_values)
        out = np.empty_like(v)
        out[self.face_ref] = v
        return out


class BoundaryConditions:
    """Per-boundary-face BC types and values on the device (kcfd_bc_t)."""

    def __init__(self, dmesh, device="cuda"):
        torch = _lib.require_cuda()
        Fb, D = dmesh.n_boundary, dmesh.ndim
        self.dmesh = dmesh
        self.u_type = np.zeros(Fb, np.int8)
        self.u_val = np.zeros((Fb, D))
        self.p_type = np.zeros(Fb, np.int8)
        self.p_val = np.zeros(Fb)
        self.bc_u, self.bc_p = {}, {}
        self._dev = None
        self.device = device
        self.dirty = True

    def set_velocity(self, patch, bc_type, value=None):
        slots = self.dmesh.patch_slots.get(patch)
        if slots is None:
            return
        if value is not None:
            v = np.asarray(value, dtype=np.float64)
            self.u_val[slots] = v
        self.u_type[slots] = BC_TYPES[bc_type]
        self.bc_u[patch] = {"type": bc_type}
        self.dirty = True

    def set_pressure(self, patch, bc_type, value=None):
        slots = self.dmesh.patch_slots.get(patch)
        if slots is None:
            return
        if value is not None:
            self.p_val[slots] = value
        self.p_type[slots] = BC_TYPES[bc_type]
        self.bc_p[patch] = {"type": bc_type}
        self.dirty = True

    def has_p_dirichlet(self):
        return any(v.get("type") == "dirichlet" for v in self.bc_p.values())

    def upload(self):
        torch = _lib.require_cuda()
        if not self.dirty and self._dev is not None:
            return self.desc
        t = {"u_type": torch.from_numpy(self.u_type.copy()).to(self.device),
             "u_val": torch.from_numpy(np.ascontiguousarray(self.u_val)).to(self.device),
             "p_type": torch.from_numpy(self.p_type.copy()).to(self.device),
             "p_val": torch.from_numpy(self.p_val.copy()).to(self.device)}
        # p' boundary treatment for its Green-Gauss gradient: 0 on dirichlet-p faces,
        # the owner value elsewhere (models/single_phase.py:357-366)
        pp_type = (self.p_type == 1).astype(np.int8)
        t["pp_type"] = torch.from_numpy(pp_type).to(self.device)
        t["pp_val"] = torch.zeros(len(pp_type), dtype=torch.float64, device=self.device)
        self._dev = t
        d = BCDesc()
        d.u_type, d.u_val = t["u_type"].data_ptr(), t["u_val"].data_ptr()
        d.p_type, d.p_val = t["p_type"].data_ptr(), t["p_val"].data_ptr()
        d.has_p_dirichlet = 1 if self.has_p_dirichlet() else 0
        self.desc = d
        self.dirty = False
        return d

    def tensor(self, name):
        self.upload()
        return self._dev[name]
