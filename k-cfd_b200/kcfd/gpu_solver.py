"""Drop-in for core/gpu_solver.py of the K-CFD reference, on libkcfd.

Same signatures as the reference (scipy CSR and ndarray in, ndarray out):
  detect_gpu_backend()                       core/gpu_solver.py:26-52
  gpu_spmv(A_csr, x)                         core/gpu_solver.py:55-79
  gpu_bicgstab(A_csr, b, x0, tol, max_iter)  core/gpu_solver.py:82-108 / :111-155
  benchmark_solvers(A_csr, b, n_runs)        core/gpu_solver.py:202-251
The reference's CuPy path copies the system to the device on every call and then
synchronises with the host five times per iteration; here the whole BiCGSTAB runs in
one persistent kernel (one copy in, one copy out). Its stopping rule is kept:
||s||/||b|| < tol (after x += alpha p) or ||r||/||b|| < tol, with the 1e-30 guards.
Unlike the reference this module never falls back to the CPU: without the native
library or a CUDA device it raises.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .solver import DeviceCSR, Solver


def detect_gpu_backend() -> str:
    """'b200' when libkcfd loads and a CUDA device of compute capability 10.x is
    present; raises otherwise (no silent CPU answer)."""
    import ctypes as C
    _lib.require_cuda()
    sm, ma, mi = C.c_int32(), C.c_int32(), C.c_int32()
    _lib.check(_lib.lib().kcfd_device_info(C.byref(sm), C.byref(ma), C.byref(mi)), "kcfd_device_info")
    if ma.value != 10:
        raise _lib.KcfdError(_lib.CUDA_ERROR, f"libkcfd is built for sm_100a; device is sm_{ma.value}{mi.value}")
    return "b200"


def gpu_spmv(A_csr, x):
    """y = A x on the device (FP64)."""
    torch = _lib.require_cuda()
    d = DeviceCSR.from_scipy(A_csr)
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()
    y = d.spmv(xd)
    return y.cpu().numpy()


def gpu_bicgstab(A_csr, b, x0=None, tol=1e-6, max_iter=1000, return_info=False):
    """Unpreconditioned BiCGSTAB with the reference GPU path's stopping rule."""
    torch = _lib.require_cuda()
    d = DeviceCSR.from_scipy(A_csr)
    bd = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).cuda()
    if x0 is None:
        xd = torch.zeros_like(bd)
    else:
        xd = torch.from_numpy(np.array(x0, dtype=np.float64)).cuda()
    s = Solver(d, precond="none", stop=_lib.STOP_GPU, maxiter=max_iter, rtol=tol)
    it, rr, st = s.solve(d, bd, xd)
    x = xd.cpu().numpy()
    if return_info:
        return x, {"iterations": int(it[0]), "relres": float(rr[0]), "status": _lib.STATUS_NAMES[int(st[0])]}
    return x


def benchmark_solvers(A_csr, b, n_runs=3):
    """core/gpu_solver.py:202-251: median wall-clock seconds of scipy's spsolve
    ('cpu_direct', with its solution as 'x_direct'), scipy's bicgstab at tol 1e-6
    ('cpu_bicgstab'; the reference times its own CPU restatement of the GPU loop) and
    this module's gpu_bicgstab at tol 1e-6, host arrays in and out, after one warm-up
    call ('gpu_bicgstab'); 'backend' is detect_gpu_backend()."""
    import time
    import scipy.sparse.linalg as spla
    results = {"backend": detect_gpu_backend()}

    def median_time(fn):
        ts = []
        out = None
        for _ in range(n_runs):
            t0 = time.time()
            out = fn()
            ts.append(time.time() - t0)
        return float(np.median(ts)), out

    results["cpu_direct"], results["x_direct"] = median_time(lambda: spla.spsolve(A_csr, b))
    results["cpu_bicgstab"], _ = median_time(lambda: spla.bicgstab(A_csr, b, rtol=1e-6, atol=0.0, maxiter=1000))
    gpu_bicgstab(A_csr, b, None, 1e-6, 1000)
    results["gpu_bicgstab"], _ = median_time(lambda: gpu_bicgstab(A_csr, b, None, 1e-6, 1000))
    return results
