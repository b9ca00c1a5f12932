"""Drop-ins for core/interpolation.py of the K-CFD reference.

- The TVD limiters (interpolation.py:17-44), LIMITER_REGISTRY and get_limiter
  (:47-52): the same formulas, elementwise on numpy arrays or device tensors (the
  device kernels of the MUSCL correction evaluate the same expressions per face).
- muscl_deferred_correction(mesh, phi, mass_flux, grad_phi, limiter_name) with the
  reference's signature (:227-303): mass flux in reference face order, phi a
  ScalarField-like field or an array, grad_phi [n, ndim]; computed by the device
  kernel (kcfd_muscl_correction), returned as an ndarray like the reference's.
- compute_mass_flux(U, rho, mesh) (:163-182), from kcfd.gradient.
"""
from __future__ import annotations

import numpy as np

from .gradient import compute_mass_flux  # noqa: F401  (re-export, core/interpolation.py:163)


def _xp(r):
    mod = type(r).__module__
    if mod.startswith("torch"):
        import torch
        return torch
    return np


def _where(xp, cond, a, b):
    if xp is np:
        return np.where(cond, a, b)
    return xp.where(cond, a, xp.zeros_like(a) + b)


def limiter_minmod(r):
    xp = _xp(r)
    return xp.maximum(xp.zeros_like(r) if xp is not np else 0.0, xp.minimum(xp.ones_like(r) if xp is not np else 1.0, r))


def limiter_superbee(r):
    xp = _xp(r)
    if xp is np:
        return np.maximum(0.0, np.maximum(np.minimum(2.0 * r, 1.0), np.minimum(r, 2.0)))
    one, two, zero = xp.ones_like(r), 2.0 * xp.ones_like(r), xp.zeros_like(r)
    return xp.maximum(zero, xp.maximum(xp.minimum(2.0 * r, one), xp.minimum(r, two)))


def limiter_van_albada(r):
    xp = _xp(r)
    return _where(xp, r > 0, (r * r + r) / (r * r + 1.0), 0.0)


def limiter_van_leer(r):
    xp = _xp(r)
    if xp is np:
        with np.errstate(divide="ignore", invalid="ignore"):  # r = -1 lies in the discarded branch
            return np.where(r > 0, 2.0 * r / (1.0 + r), 0.0)
    return _where(xp, r > 0, 2.0 * r / (1.0 + r), 0.0)


LIMITER_REGISTRY = {
    "minmod": limiter_minmod,
    "superbee": limiter_superbee,
    "van_albada": limiter_van_albada,
    "van_leer": limiter_van_leer,
}


def get_limiter(name: str):
    if name not in LIMITER_REGISTRY:
        raise ValueError(f"Unknown limiter: {name}. Available: {list(LIMITER_REGISTRY.keys())}")
    return LIMITER_REGISTRY[name]


def muscl_deferred_correction(mesh, phi, mass_flux, grad_phi, limiter_name="van_leer"):
    """core/interpolation.py:227-303 on the device; returns the per-cell rhs
    correction as an ndarray."""
    from .assembly import muscl_deferred_correction as _device_muscl
    from .fvm_operators import _cells, _dmesh, _faces
    get_limiter(limiter_name)
    dm = _dmesh(mesh)
    grad = _cells(np.asarray(grad_phi, dtype=np.float64).reshape(dm.n_cells, dm.ndim), dm)
    corr = _device_muscl(dm, _cells(phi, dm), _faces(mass_flux, dm), grad, limiter_name)
    return corr.cpu().numpy()
