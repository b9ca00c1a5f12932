"""Cell-centre field containers with the reference's API (core/fields.py:12-152).

ScalarField and VectorField hold host arrays: values [n] or [n, ndim], per-patch
boundary_values (arrays in patch order), old_values; copy, store_old, set_uniform,
set_boundary, get_face_value, min / max / mean, x / y / z and magnitude. They are what
the drop-in functions (kcfd.fvm_operators, kcfd.gradient, kcfd.interpolation) accept
as fields; the device solvers keep their own device copies.
"""
from __future__ import annotations

import numpy as np


class ScalarField:
    def __init__(self, mesh, name="scalar", default=0.0):
        self.mesh = mesh
        self.name = name
        self.values = np.full(mesh.n_cells, default, dtype=np.float64)
        self.boundary_values = {b: np.full(len(f), default, dtype=np.float64) for b, f in mesh.boundary_patches.items()}
        self.old_values = None

    def copy(self):
        sf = ScalarField(self.mesh, self.name)
        sf.values = self.values.copy()
        sf.boundary_values = {b: v.copy() for b, v in self.boundary_values.items()}
        sf.old_values = None if self.old_values is None else self.old_values.copy()
        return sf

    def store_old(self):
        self.old_values = self.values.copy()

    def set_uniform(self, value):
        self.values[:] = value
        for v in self.boundary_values.values():
            v[:] = value

    def set_boundary(self, patch_name, value):
        if patch_name not in self.boundary_values:
            return
        if np.isscalar(value):
            self.boundary_values[patch_name][:] = value
        else:
            self.boundary_values[patch_name] = np.array(value, dtype=np.float64)

    def get_face_value(self, face_idx):
        """The owner's value on an internal face; on a boundary face the patch's value
        (the owner's if the face is in no patch)."""
        nb, own = _face_cells(self.mesh, face_idx)
        if nb < 0:
            for b, fids in self.mesh.boundary_patches.items():
                hit = np.flatnonzero(np.asarray(fids) == face_idx)
                if len(hit):
                    return self.boundary_values[b][hit[0]]
        return self.values[own]

    def max(self):
        return float(np.max(self.values))

    def min(self):
        return float(np.min(self.values))

    def mean(self):
        return float(np.mean(self.values))


class VectorField:
    def __init__(self, mesh, name="vector", default=None):
        self.mesh = mesh
        self.name = name
        ndim = getattr(mesh, "ndim", 2)
        d = np.zeros(ndim) if default is None else np.array(default, dtype=np.float64)
        if len(d) < ndim:
            d = np.pad(d, (0, ndim - len(d)))
        self.values = np.tile(d, (mesh.n_cells, 1)).astype(np.float64)
        self.boundary_values = {b: np.tile(d, (len(f), 1)).astype(np.float64) for b, f in mesh.boundary_patches.items()}
        self.old_values = None

    @property
    def x(self):
        return self.values[:, 0]

    @x.setter
    def x(self, v):
        self.values[:, 0] = v

    @property
    def y(self):
        return self.values[:, 1]

    @y.setter
    def y(self, v):
        self.values[:, 1] = v

    @property
    def z(self):
        return self.values[:, 2] if self.values.shape[1] >= 3 else np.zeros(self.values.shape[0])

    @z.setter
    def z(self, v):
        if self.values.shape[1] >= 3:
            self.values[:, 2] = v

    def copy(self):
        vf = VectorField(self.mesh, self.name)
        vf.values = self.values.copy()
        vf.boundary_values = {b: v.copy() for b, v in self.boundary_values.items()}
        vf.old_values = None if self.old_values is None else self.old_values.copy()
        return vf

    def store_old(self):
        self.old_values = self.values.copy()

    def set_uniform(self, value):
        value = np.array(value, dtype=np.float64)
        self.values[:] = value
        for v in self.boundary_values.values():
            v[:] = value

    def set_boundary(self, patch_name, value):
        if patch_name not in self.boundary_values:
            return
        value = np.array(value, dtype=np.float64)
        if value.ndim == 1:
            self.boundary_values[patch_name][:] = value
        else:
            self.boundary_values[patch_name] = value

    def magnitude(self):
        return np.sqrt(np.sum(self.values ** 2, axis=1))


def _face_cells(mesh, f):
    """(neighbour, owner) of face f for a kcfd Mesh or an FVMesh-shaped object."""
    nbr = getattr(mesh, "neighbour", None)
    if nbr is not None and not callable(nbr):
        return int(nbr[f]), int(mesh.owner[f])
    face = mesh.faces[f]
    return int(face.neighbour), int(face.owner)
