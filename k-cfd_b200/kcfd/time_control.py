"""CFL-based adaptive time step, as the reference's core/time_control.py:10-164.

AdaptiveTimeControl keeps the reference's API and arithmetic: the cell size is
dx = V^(1/ndim) (floored at 1e-30), the CFL number |u| dt / dx with |u| the row norm
of the cell velocity, the Fourier number alpha dt / dx^2; compute_dt takes the CFL
limit cfl_target dx / |u| (|u| floored at 1e-30) times the safety factor, the Fourier
limit likewise when a diffusivity is given, caps growth at growth_factor x the last
dt, shrinks by shrink_factor when the step did not converge, clips to [dt_min,
dt_max] and records the CFL and Fourier numbers at the new dt. The per-cell loops
of the reference are numpy array operations here (the same operations per cell).
The velocity comes to the host once per step (the two-fluid solver hands over its
liquid velocity, as the reference does).
"""
from __future__ import annotations

import numpy as np


def _cell_size(mesh):
    ndim = getattr(mesh, "ndim", 2)
    vol = getattr(mesh, "volume", None)
    if vol is None or callable(vol):
        vol = np.array([c.volume for c in mesh.cells], dtype=np.float64)
    vol = np.asarray(vol, dtype=np.float64)
    return np.maximum(vol ** (1.0 / ndim), 1e-30)


def _speed(velocity):
    velocity = np.asarray(velocity)
    return np.abs(velocity) if velocity.ndim == 1 else np.linalg.norm(velocity, axis=1)


class AdaptiveTimeControl:
    def __init__(self, dt_init, dt_min=1e-8, dt_max=1.0, cfl_target=0.5, cfl_max=1.0, fourier_max=0.5,
                 growth_factor=1.2, shrink_factor=0.5, safety_factor=0.9):
        self.dt = dt_init
        self.dt_min, self.dt_max = dt_min, dt_max
        self.cfl_target, self.cfl_max, self.fourier_max = cfl_target, cfl_max, fourier_max
        self.growth_factor, self.shrink_factor, self.safety_factor = growth_factor, shrink_factor, safety_factor
        self.dt_history, self.cfl_history, self.fourier_history = [], [], []

    def compute_cfl(self, mesh, velocity, dt):
        cfl = _speed(velocity) * dt / _cell_size(mesh)
        return float(np.max(cfl)), cfl

    def compute_fourier(self, mesh, alpha_diff, dt):
        fo = alpha_diff * dt / (_cell_size(mesh) ** 2)
        return float(np.max(fo)), fo

    def compute_dt(self, mesh, velocity, alpha_diff=None, converged=True):
        dx = _cell_size(mesh)
        u = _speed(velocity)
        dt_new = float(np.min(self.cfl_target * dx / np.maximum(u, 1e-30))) * self.safety_factor
        limited_by = "cfl"
        if alpha_diff is not None:
            dt_fo = float(np.min(self.fourier_max * dx ** 2 / np.maximum(alpha_diff, 1e-30))) * self.safety_factor
            if dt_fo < dt_new:
                dt_new, limited_by = dt_fo, "fourier"
        dt_new = min(dt_new, self.growth_factor * self.dt)
        if not converged:
            dt_new, limited_by = self.shrink_factor * self.dt, "divergence"
        dt_new = float(np.clip(dt_new, self.dt_min, self.dt_max))
        cfl_max, _ = self.compute_cfl(mesh, velocity, dt_new)
        fo_max = self.compute_fourier(mesh, alpha_diff, dt_new)[0] if alpha_diff is not None else 0.0
        self.dt = dt_new
        self.dt_history.append(dt_new)
        self.cfl_history.append(cfl_max)
        self.fourier_history.append(fo_max)
        return dt_new, {"cfl_max": cfl_max, "fourier_max": fo_max, "dt_limited_by": limited_by, "dt": dt_new}

    def get_info(self):
        return {"dt": self.dt, "dt_history": self.dt_history.copy(), "cfl_history": self.cfl_history.copy(),
                "fourier_history": self.fourier_history.copy()}
