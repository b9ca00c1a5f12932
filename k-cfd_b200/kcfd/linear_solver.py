"""Drop-in for core/linear_solver.py and core/preconditioner.py of the K-CFD reference.

solve_linear_system(system, x0, method, tol, maxiter, backend, preconditioner, **kw)
keeps the reference signature (core/linear_solver.py:14-19). backend='b200' (or
'auto') runs on libkcfd and is chosen before anything that could hide an error: a
device failure raises instead of falling back to the CPU. Semantics kept:
  * method='bicgstab': scipy's BiCGSTAB loop as the reference calls it
    (core/linear_solver.py:59): atol=tol and scipy's default rtol=1e-5 unless the
    caller passes rtol=..., so the stop is ||r|| < max(tol, rtol ||b||); x0=None
    starts from zero; non-convergence prints and returns x (:60-61).
  * preconditioner: 'none' | 'jacobi' (1/d where |d| > 1e-30, :43-47) | 'ilu0'
    (structural, level-scheduled ILU(0); the reference's 'ilu0' is SuperLU spilu,
    so agreement with it is at the solution level) | 'iluk' (structural ILU(k),
    fill_level=k, default 1, on a distance-(k+1) colouring; the reference's 'iluk'
    is SuperLU's threshold ILU with fill_factor=3 (:56-61), so agreement is again at
    the solution level and fill_factor is not used) | 'amg' (device smoothed-aggregation
    multigrid, kcfd.amg; the reference's is pyamg's (:63-74), absent here, so
    agreement is at the solution level; max_levels and max_coarse are honoured, the
    coarsest level being at most 256 rows).
  * method='direct': the device has no sparse LU; BiCGSTAB + ILU(0) to a relative
    residual of 1e-12 stands in for spsolve (documented difference).
system may be the reference's FVMSystem (anything with .to_sparse() and .rhs), a
kcfd FVMSystem, or a device-assembled kcfd DeviceSystem.
"""
from __future__ import annotations

import time

import numpy as np

from . import _lib
from .solver import DeviceCSR, Solver

DIRECT_RTOL = 1e-12
SCIPY_DEFAULT_RTOL = 1e-5


def create_preconditioner(A_csr, method="none", **kwargs):
    """(M, info) as core/preconditioner.py:18-76: M is None for 'none', else a
    scipy.sparse.linalg.LinearOperator whose matvec applies the device preconditioner
    (host vector in, host vector out; kcfd_solver_apply_precond), so M can be handed to
    scipy's Krylov solvers as the reference's is. info carries 'method' and
    'setup_time' like the reference's, ('levels', 'complexity' for 'amg'), and under
    'device' the handle and device matrix for callers that stay on the device."""
    from scipy.sparse.linalg import LinearOperator
    torch = _lib.require_cuda()
    t0 = time.time()
    if method == "none":
        return None, {"method": "none", "setup_time": 0.0}
    fill = 0
    name = method
    prec = method
    if method == "iluk":
        fill = int(kwargs.get("fill_level", 1))
        prec, name = "ilu0", f"iluk(level={fill})"
    if prec not in _lib.PREC:
        raise ValueError(f"Unknown preconditioner: {method}")
    d = DeviceCSR.from_scipy(A_csr) if not isinstance(A_csr, DeviceCSR) else A_csr
    s = Solver(d, precond=prec, levels=None if fill else kwargs.get("levels"), fill_level=fill,
               amg_max_levels=int(kwargs.get("max_levels", 0)) if prec == "amg" else 0,
               amg_coarse_max=min(int(kwargs.get("max_coarse", 0)), 256) if prec == "amg" else 0)
    s.setup(d)
    n = d.n
    r_dev = torch.empty(n, dtype=torch.float64, device=d.vals64.device)
    z_dev = torch.empty_like(r_dev)

    def matvec(v):
        r_dev.copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(v, dtype=np.float64).ravel())))
        s.apply_precond(d, r_dev, z_dev)
        return z_dev.cpu().numpy()

    M = LinearOperator((n, n), matvec=matvec, dtype=np.float64)
    torch.cuda.synchronize()
    info = {"method": name, "setup_time": time.time() - t0, "device": {"solver": s, "csr": d}}
    if prec == "amg":
        ai = s.amg_info()
        info["levels"] = ai["levels"]
        info["complexity"] = float(sum(ai["nnz"]) / max(ai["nnz"][0], 1))
    return M, info


def _as_device(system):
    """(DeviceCSR, b device tensor, levels or None) from any supported system."""
    torch = _lib.require_cuda()
    if hasattr(system, "device_csr"):
        return system.device_csr(), system.device_rhs(), getattr(system, "ilu_levels", None)
    A = system.to_sparse()
    b = torch.from_numpy(np.ascontiguousarray(system.rhs, dtype=np.float64)).cuda()
    return DeviceCSR.from_scipy(A), b, None


def solve_linear_system(system, x0=None, method="direct", tol=1e-8, maxiter=1000, backend="auto",
                        preconditioner="none", **precond_kwargs):
    if backend not in ("auto", "b200", "gpu"):
        raise ValueError(f"kcfd runs on the device only (backend '{backend}' is the reference's CPU path)")
    torch = _lib.require_cuda()
    rtol = precond_kwargs.pop("rtol", SCIPY_DEFAULT_RTOL)
    d, b, levels = _as_device(system)
    levels = precond_kwargs.pop("levels", levels)
    fill = 0
    n = d.n
    if method == "direct":
        prec, atol, rtol_eff, its = "ilu0", 0.0, DIRECT_RTOL, max(maxiter, 20 * n)
    elif method == "bicgstab":
        prec, atol, rtol_eff, its = preconditioner, float(tol), float(rtol), maxiter
        if prec == "iluk":
            prec, fill, levels = "ilu0", int(precond_kwargs.pop("fill_level", 1)), None
            precond_kwargs.pop("fill_factor", None)
    elif method == "gmres":
        raise NotImplementedError("gmres is not on the kcfd device path (use 'bicgstab')")
    else:
        raise ValueError(f"Unknown solver method: {method}")
    x = torch.zeros(n, dtype=torch.float64, device=b.device) if x0 is None else \
        torch.from_numpy(np.array(x0, dtype=np.float64)).to(b.device)
    amg_kw = {}
    if prec == "amg":
        amg_kw = {"amg_max_levels": int(precond_kwargs.pop("max_levels", 0)),
                  "amg_coarse_max": min(int(precond_kwargs.pop("max_coarse", 0)), 256)}
    s = Solver(d, precond=prec, stop=_lib.STOP_SCIPY, maxiter=its, rtol=rtol_eff, atol=atol, levels=levels,
               fill_level=fill, **amg_kw)
    s.setup(d)
    it, rr, st = s.solve(d, b, x)
    status = int(st[0])
    if status == _lib.MAXITER and method == "bicgstab":
        print(f"[bicgstab] 수렴 실패: {int(it[0])} 반복 후 중단")
    elif status not in (_lib.OK, _lib.MAXITER, _lib.BREAKDOWN):
        raise _lib.KcfdError(status, "device solve failed")
    err = s.barrier_error()
    if err:
        raise _lib.KcfdError(err, "device barrier wait expired")
    return x.cpu().numpy()


def solve_pressure_correction(system, method="direct", tol=1e-6, maxiter=2000, preconditioner="none",
                              **precond_kwargs):
    """core/linear_solver.py:73-93: 'direct' as solve_linear_system; any other method runs
    scipy's conjugate gradients from x0 = 0 with atol=tol (and scipy's default rtol) and
    the given preconditioner, on the device (the graph engine's CG)."""
    if method == "direct":
        return solve_linear_system(system, None, "direct", tol, maxiter, "b200", preconditioner, **precond_kwargs)
    torch = _lib.require_cuda()
    rtol = precond_kwargs.pop("rtol", SCIPY_DEFAULT_RTOL)
    d, b, levels = _as_device(system)
    levels = precond_kwargs.pop("levels", levels)
    prec, fill = preconditioner, 0
    if prec == "iluk":
        prec, fill, levels = "ilu0", int(precond_kwargs.pop("fill_level", 1)), None
        precond_kwargs.pop("fill_factor", None)
    amg_kw = {}
    if prec == "amg":
        amg_kw = {"amg_max_levels": int(precond_kwargs.pop("max_levels", 0)),
                  "amg_coarse_max": min(int(precond_kwargs.pop("max_coarse", 0)), 256)}
    x = torch.zeros(d.n, dtype=torch.float64, device=b.device)
    s = Solver(d, precond=prec, stop=_lib.STOP_SCIPY, maxiter=maxiter, rtol=float(rtol), atol=float(tol),
               levels=levels, fill_level=fill, method="cg", **amg_kw)
    s.setup(d)
    it, rr, st = s.solve(d, b, x)
    status = int(st[0])
    if status not in (_lib.OK, _lib.MAXITER, _lib.BREAKDOWN):
        raise _lib.KcfdError(status, "device solve failed")
    return x.cpu().numpy()
