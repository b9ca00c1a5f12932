"""Device linear systems assembled with the generic FVM operators.

DeviceSystem mirrors the reference's FVMSystem (core/fvm_operators.py:13-56) on the
device: CSR values on the mesh's canonical pattern, the tracked diagonal and the rhs.
Its methods are the reference's operators (core/fvm_operators.py:59-240,
core/interpolation.py:227-303) with the same argument meaning; fields are device
tensors (cells [n], faces in device face order, boundary values per boundary face in
device boundary order, see DeviceMesh.patch_slots). The system plugs into
kcfd.linear_solver.solve_linear_system(backend='b200') without leaving the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
from scipy import sparse

from . import _lib
from .device_mesh import BC_TYPES
from .solver import DeviceCSR


class DeviceSystem:
    def __init__(self, dmesh):
        torch = _lib.require_cuda()
        self.dm = dmesh
        self.n = dmesh.n_cells
        dev = dmesh.t["owner"].device
        self.vals = torch.zeros(dmesh.nnz, dtype=torch.float64, device=dev)
        self.diag = torch.zeros(self.n, dtype=torch.float64, device=dev)
        self.rhs = torch.zeros(self.n, dtype=torch.float64, device=dev)
        self.ilu_levels = dmesh.cell_color

    def reset(self):
        self.vals.zero_(); self.diag.zero_(); self.rhs.zero_()

    def _call(self, name, *args):
        _lib.check(getattr(_lib.lib(), name)(C.byref(self.dm.desc), *args, _lib.stream_handle()), name)

    # ---- operators (reference argument meaning) ----
    def diffusion_operator(self, gamma):
        self._call("kcfd_op_diffusion", _lib.ptr(gamma), _lib.ptr(self.vals), _lib.ptr(self.diag))

    def convection_operator_upwind(self, mass_flux):
        self._call("kcfd_op_convection_upwind", _lib.ptr(mass_flux), _lib.ptr(self.vals), _lib.ptr(self.diag))

    def temporal_operator(self, rho, dt, phi_old):
        self._call("kcfd_op_cells", 0, float(rho), float(dt), _lib.ptr(phi_old), None, _lib.ptr(self.vals),
                   _lib.ptr(self.diag), _lib.ptr(self.rhs))

    def source_term(self, S):
        self._call("kcfd_op_cells", 1, 0.0, 0.0, _lib.ptr(S), None, _lib.ptr(self.vals), _lib.ptr(self.diag),
                   _lib.ptr(self.rhs))

    def linearized_source(self, Sp, Su):
        self._call("kcfd_op_cells", 2, 0.0, 0.0, _lib.ptr(Sp), _lib.ptr(Su), _lib.ptr(self.vals),
                   _lib.ptr(self.diag), _lib.ptr(self.rhs))

    def apply_boundary_conditions(self, btype, bval, bgrad, gamma, mass_flux):
        self._call("kcfd_op_boundary", _lib.ptr(btype), _lib.ptr(bval), _lib.ptr(bgrad), _lib.ptr(gamma),
                   _lib.ptr(mass_flux), _lib.ptr(self.vals), _lib.ptr(self.diag), _lib.ptr(self.rhs))

    def under_relax(self, phi, alpha):
        if alpha >= 1.0:
            return
        self._call("kcfd_op_cells", 3, float(alpha), 0.0, _lib.ptr(phi), None, _lib.ptr(self.vals),
                   _lib.ptr(self.diag), _lib.ptr(self.rhs))

    # ---- solver hand-off ----
    def device_csr(self):
        return DeviceCSR(self.dm.t["indptr"], self.dm.t["indices"], self.vals)

    def device_rhs(self):
        return self.rhs

    def to_sparse(self):
        m = self.dm.host
        return sparse.csr_matrix((self.vals.cpu().numpy(), m.indices.copy(), m.indptr.copy()),
                                 shape=(self.n, self.n))


def boundary_arrays(dmesh, bc_types, phi_b_by_patch, device="cuda"):
    """Per-boundary-face (btype, bval, bgrad) device tensors from the reference's
    bc_types dict ({patch: {'type': ..., 'value': ...}}) and per-patch phi_b arrays."""
    torch = _lib.require_cuda()
    Fb = dmesh.n_boundary
    bt = np.zeros(Fb, np.int8)
    bv = np.zeros(Fb)
    bg = np.zeros(Fb)
    for nm, slots in dmesh.patch_slots.items():
        bc = bc_types.get(nm, {"type": "zero_gradient"})
        t = BC_TYPES.get(bc["type"], -1)
        bt[slots] = t
        if nm in phi_b_by_patch:
            bv[slots] = np.asarray(phi_b_by_patch[nm], dtype=np.float64)
        if t == 2:
            bg[slots] = float(bc.get("value", 0.0))
    return (torch.from_numpy(bt).to(device), torch.from_numpy(bv).to(device), torch.from_numpy(bg).to(device))


def muscl_deferred_correction(dmesh, phi, mass_flux, grad, limiter_name="van_leer"):
    """Device counterpart of core/interpolation.py:227-303 (returns corr [n])."""
    torch = _lib.require_cuda()
    if limiter_name not in ("minmod", "superbee", "van_albada", "van_leer"):
        raise ValueError(f"Unknown limiter: {limiter_name}")
    corr = torch.empty(dmesh.n_cells, dtype=torch.float64, device=phi.device)
    _lib.check(_lib.lib().kcfd_muscl_correction(C.byref(dmesh.desc), _lib.LIMITERS[limiter_name], _lib.ptr(phi),
                                                _lib.ptr(mass_flux), _lib.ptr(grad), _lib.ptr(corr),
                                                _lib.stream_handle()), "kcfd_muscl_correction")
    return corr
