"""Device drop-ins for the reference's gradient and face-flux functions.

  green_gauss_gradient(phi)      core/gradient.py:12-48
  least_squares_gradient(phi)    core/gradient.py:51-99
  compute_mass_flux(U, rho, mesh) core/interpolation.py:163-182

They take the reference's field objects (anything with .mesh, .values and a
.boundary_values dict of per-patch arrays, as core/fields.py) and return host
ndarrays in the reference's cell / face order; the work runs in libkcfd's kernels
(kcfd_gg_gradient, kcfd_lsq_gradient, kcfd_tf_mass_flux). On the boundary the
reference uses the patch value of every boundary face, and so do these.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

_CACHE: list = []  # [(reference mesh object, DeviceMesh)], a few recent meshes


def _device_mesh(mesh):
    from .device_mesh import DeviceMesh
    from .mesh import Mesh, from_fvmesh
    for src, dm in _CACHE:
        if src is mesh:
            return dm
    m = mesh if isinstance(mesh, Mesh) else from_fvmesh(mesh)
    dm = DeviceMesh(m)
    _CACHE.append((mesh, dm))
    del _CACHE[:-4]
    return dm


def _boundary_values(dm, bvals, ncomp):
    torch = _lib.require_cuda()
    out = np.zeros((dm.n_boundary, ncomp) if ncomp > 1 else dm.n_boundary)
    for nm, slots in dm.patch_slots.items():
        if nm in bvals:
            out[slots] = np.asarray(bvals[nm], dtype=np.float64).reshape(out[slots].shape)
    return torch.from_numpy(out).cuda()


def _dev(a):
    torch = _lib.require_cuda()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def green_gauss_gradient(phi):
    torch = _lib.require_cuda()
    dm = _device_mesh(phi.mesh)
    n, nd = dm.n_cells, dm.ndim
    pv = _dev(phi.values)
    pb = _boundary_values(dm, phi.boundary_values, 1)
    bt = torch.ones(dm.n_boundary, dtype=torch.int8, device="cuda")
    g = torch.empty(n, nd, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().kcfd_gg_gradient(C.byref(dm.desc), 1, _lib.ptr(pv), _lib.ptr(bt), _lib.ptr(pb),
                                           _lib.ptr(g), _lib.stream_handle()), "kcfd_gg_gradient")
    return g.cpu().numpy()


def least_squares_gradient(phi):
    torch = _lib.require_cuda()
    dm = _device_mesh(phi.mesh)
    n, nd = dm.n_cells, dm.ndim
    pv = _dev(phi.values)
    pb = _boundary_values(dm, phi.boundary_values, 1)
    g = torch.empty(n, nd, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().kcfd_lsq_gradient(C.byref(dm.desc), _lib.ptr(pv), _lib.ptr(pb), _lib.ptr(g),
                                            _lib.stream_handle()), "kcfd_lsq_gradient")
    return g.cpu().numpy()


def compute_mass_flux(U, rho, mesh):
    torch = _lib.require_cuda()
    dm = _device_mesh(mesh)
    uv = _dev(np.asarray(U.values).reshape(dm.n_cells, dm.ndim))
    ub = _boundary_values(dm, U.boundary_values, dm.ndim)
    mf = torch.empty(dm.n_faces, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().kcfd_tf_mass_flux(C.byref(dm.desc), float(rho), _lib.ptr(uv), _lib.ptr(ub), _lib.ptr(mf),
                                            _lib.stream_handle()), "kcfd_tf_mass_flux")
    return dm.to_reference_faces(mf)
