"""FVMSystem mirror of core/fvm_operators.py:13-56 (host container).

The reference's FVMSystem collects COO triplets on the host; this class keeps the
same API (add_diagonal, add_off_diagonal, add_source, to_sparse, reset, diag, rhs)
so reference-style assembly code can hand its system to the device solvers in
kcfd.linear_solver. Device-side assembly lives in kcfd.assembly (DeviceSystem).
"""
from __future__ import annotations

import numpy as np
from scipy import sparse


class FVMSystem:
    def __init__(self, n: int):
        self.n = n
        self.rows, self.cols, self.vals = [], [], []
        self.rhs = np.zeros(n, dtype=np.float64)
        self.diag = np.zeros(n, dtype=np.float64)
        self._csr = None

    @classmethod
    def from_csr(cls, A, rhs):
        s = cls(A.shape[0])
        s._csr = sparse.csr_matrix(A)
        s.rhs = np.asarray(rhs, dtype=np.float64).copy()
        s.diag = s._csr.diagonal().copy()
        return s

    def add_diagonal(self, i, val):
        self.rows.append(i); self.cols.append(i); self.vals.append(val)
        self.diag[i] += val
        self._csr = None

    def add_off_diagonal(self, i, j, val):
        self.rows.append(i); self.cols.append(j); self.vals.append(val)
        self._csr = None

    def add_source(self, i, val):
        self.rhs[i] += val

    def to_sparse(self):
        if self._csr is not None and not self.rows:
            return self._csr
        return sparse.coo_matrix((self.vals, (self.rows, self.cols)), shape=(self.n, self.n)).tocsr()

    def reset(self):
        self.rows.clear(); self.cols.clear(); self.vals.clear()
        self.rhs[:] = 0.0
        self.diag[:] = 0.0
        self._csr = None


# ---------------------------------------------------------------- operators --
# The reference's module-level operators (core/fvm_operators.py:59-240) with its
# signatures: op(mesh, ..., system). mesh is a reference FVMesh or a kcfd Mesh; cell
# fields are ScalarField-like (.values), ndarrays or device tensors; mass fluxes are in
# reference face order; phi.boundary_values holds per-patch arrays in patch order.
# The work runs on the device (the generic operator kernels of kcfd.assembly). With a
# kcfd.assembly.DeviceSystem the system stays on the device; with this module's host
# FVMSystem the device result (CSR values, tracked diagonal, rhs) is added to it as
# triplets, so to_sparse() sums to the reference's matrix.

_MESHES = {}


def _dmesh(mesh):
    from .device_mesh import DeviceMesh
    from .mesh import Mesh, from_fvmesh
    key = id(mesh)
    hit = _MESHES.get(key)
    if hit is not None and hit[0] is mesh:
        return hit[1]
    m = mesh if isinstance(mesh, Mesh) else from_fvmesh(mesh)
    dm = DeviceMesh(m)
    _MESHES[key] = (mesh, dm)
    return dm


def _cells(x, dm):
    from . import _lib
    torch = _lib.require_cuda()
    v = getattr(x, "values", x)
    if isinstance(v, torch.Tensor):
        return v.to(device=dm.t["owner"].device, dtype=torch.float64)
    return torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).to(dm.t["owner"].device)


def _faces(mf, dm):
    from . import _lib
    torch = _lib.require_cuda()
    dev = dm.t["owner"].device
    if isinstance(mf, torch.Tensor):
        return mf.to(device=dev, dtype=torch.float64)[dm.t["face_ref"].long()]
    return torch.from_numpy(np.ascontiguousarray(np.asarray(mf, dtype=np.float64)[dm.face_ref])).to(dev)


def _apply(mesh, system, fn):
    from .assembly import DeviceSystem
    if isinstance(system, DeviceSystem):
        fn(system, system.dm)
        return
    dm = _dmesh(mesh)
    ds = DeviceSystem(dm)
    fn(ds, dm)
    system.add_device(ds)


def _add_device(self, ds):
    """Add a DeviceSystem's CSR values, tracked diagonal and rhs to this host system."""
    if self._csr is not None and not self.rows:
        A = self._csr.tocoo()
        self.rows.extend(A.row.tolist()); self.cols.extend(A.col.tolist()); self.vals.extend(A.data.tolist())
    A = ds.to_sparse().tocoo()
    self.rows.extend(A.row.tolist()); self.cols.extend(A.col.tolist()); self.vals.extend(A.data.tolist())
    self.diag += ds.diag.cpu().numpy()
    self.rhs += ds.rhs.cpu().numpy()
    self._csr = None


FVMSystem.add_device = _add_device


def diffusion_operator(mesh, gamma, system):
    """core/fvm_operators.py:59-100."""
    _apply(mesh, system, lambda ds, dm: ds.diffusion_operator(_cells(gamma, dm)))


def convection_operator_upwind(mesh, mass_flux, system):
    """core/fvm_operators.py:103-129."""
    _apply(mesh, system, lambda ds, dm: ds.convection_operator_upwind(_faces(mass_flux, dm)))


def temporal_operator(mesh, rho, dt, phi_old, system):
    """core/fvm_operators.py:132-148."""
    _apply(mesh, system, lambda ds, dm: ds.temporal_operator(rho, dt, _cells(phi_old, dm)))


def source_term(mesh, source_values, system):
    """core/fvm_operators.py:151-161."""
    _apply(mesh, system, lambda ds, dm: ds.source_term(_cells(source_values, dm)))


def linearized_source(mesh, Sp, Su, system):
    """core/fvm_operators.py:164-175."""
    _apply(mesh, system, lambda ds, dm: ds.linearized_source(_cells(Sp, dm), _cells(Su, dm)))


def apply_boundary_conditions(mesh, phi, gamma, mass_flux, system, bc_types):
    """core/fvm_operators.py:178-225 (dirichlet values from phi.boundary_values)."""
    from .assembly import boundary_arrays

    def fn(ds, dm):
        bt, bv, bg = boundary_arrays(dm, bc_types, getattr(phi, "boundary_values", {}) or {},
                                     device=dm.t["owner"].device)
        ds.apply_boundary_conditions(bt, bv, bg, _cells(gamma, dm), _faces(mass_flux, dm))

    _apply(mesh, system, fn)


def under_relax(system, phi, alpha):
    """core/fvm_operators.py:228-240: a_P (1 - alpha) / alpha on the diagonal and times
    phi on the rhs, a_P the system's tracked diagonal."""
    from .assembly import DeviceSystem
    if alpha >= 1.0:
        return
    if isinstance(system, DeviceSystem):
        system.under_relax(_cells(phi, system.dm), alpha)
        return
    ap = system.diag.copy()
    add = ap * (1.0 - alpha) / alpha
    idx = np.arange(system.n)
    if system._csr is not None and not system.rows:
        A = system._csr.tocoo()
        system.rows.extend(A.row.tolist()); system.cols.extend(A.col.tolist()); system.vals.extend(A.data.tolist())
    system.rows.extend(idx.tolist()); system.cols.extend(idx.tolist()); system.vals.extend(add.tolist())
    system.diag += add
    system.rhs += add * np.asarray(getattr(phi, "values", phi), dtype=np.float64)
    system._csr = None
