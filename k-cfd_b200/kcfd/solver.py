"""Device CSR matrices and the BiCGSTAB solver handle (libkcfd kcfd_solver_*).

Torch tensors serve only as device buffers; every computation runs in libkcfd's
sm_100a kernels. A Solver binds one sparsity pattern and keeps its Krylov scratch
and preconditioner resident, so repeated solves (SIMPLE outer iterations) allocate
nothing and never synchronise with the host unless results are read.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class DeviceCSR:
    """CSR on the device: int32 indptr/indices, FP64 values and optional FP32 copy."""

    def __init__(self, indptr, indices, vals64, vals32=None):
        self.indptr, self.indices, self.vals64, self.vals32 = indptr, indices, vals64, vals32
        self.n = int(indptr.numel() - 1)
        self.nnz = int(indices.numel())

    @classmethod
    def from_scipy(cls, A, fp32=False, device="cuda"):
        torch = _lib.require_cuda()
        A = A.tocsr()
        if not A.has_sorted_indices:
            A = A.sorted_indices()
        ip = torch.from_numpy(np.ascontiguousarray(A.indptr, dtype=np.int32)).to(device)
        ix = torch.from_numpy(np.ascontiguousarray(A.indices, dtype=np.int32)).to(device)
        v = torch.from_numpy(np.ascontiguousarray(A.data, dtype=np.float64)).to(device)
        out = cls(ip, ix, v)
        if fp32:
            out.refresh_fp32()
        return out

    @classmethod
    def from_pattern(cls, indptr, indices, device="cuda", fp32=False):
        torch = _lib.require_cuda()
        ip = torch.from_numpy(np.ascontiguousarray(indptr, dtype=np.int32)).to(device)
        ix = torch.from_numpy(np.ascontiguousarray(indices, dtype=np.int32)).to(device)
        v = torch.zeros(len(indices), dtype=torch.float64, device=device)
        out = cls(ip, ix, v)
        if fp32:
            out.vals32 = torch.zeros(len(indices), dtype=torch.float32, device=device)
        return out

    def refresh_fp32(self, stream=None):
        """FP32 copy of the FP64 values (kcfd_cast_f64_f32)."""
        torch = _lib.require_cuda()
        if self.vals32 is None:
            self.vals32 = torch.empty(self.nnz, dtype=torch.float32, device=self.vals64.device)
        _lib.check(_lib.lib().kcfd_cast_f64_f32(self.nnz, _lib.ptr(self.vals64), _lib.ptr(self.vals32),
                                                _lib.stream_handle(stream)), "kcfd_cast_f64_f32")

    def desc(self):
        d = _lib.Csr()
        d.n, d.nnz = self.n, self.nnz
        d.indptr, d.indices = _lib.ptr(self.indptr), _lib.ptr(self.indices)
        d.vals64 = _lib.ptr(self.vals64)
        d.vals32 = _lib.ptr(self.vals32) if self.vals32 is not None else None
        return d

    def spmv(self, x, y=None, nrhs=1, fp32=False, stream=None):
        torch = _lib.require_cuda()
        if y is None:
            y = torch.empty_like(x)
        d = self.desc()
        fn = _lib.lib().kcfd_spmv_f32 if fp32 else _lib.lib().kcfd_spmv_f64
        _lib.check(fn(C.byref(d), _lib.ptr(x), _lib.ptr(y), nrhs, _lib.stream_handle(stream)), "kcfd_spmv")
        return y


class Solver:
    """BiCGSTAB handle for one pattern.

    method: 'bicgstab' or 'cg' (scipy's conjugate gradients: one right-hand side, FP64, the
    scipy stop rule, on the graph engine).
    precond: 'none' | 'jacobi' | 'ilu0' | 'amg' (smoothed-aggregation multigrid, one right-hand
    side, graph engine; mode MIXED keeps the Krylov iteration FP64 and stores the multigrid
    hierarchy in FP32); stop: _lib.STOP_SCIPY | _lib.STOP_GPU;
    mode: _lib.MODE_FP64 | _lib.MODE_MIXED; nrhs: 1 or 3; team: 0 auto, 1 one CTA,
    2 whole grid (persistent cooperative kernel), 3 graph engine (phase kernels in a
    CUDA graph with a device-side WHILE loop; FP64 only); levels: ILU(0) level of each row (e.g. mesh.cell_color), None for
    natural-order levels. fill_level k > 0 with precond 'ilu0' gives ILU(k): rows ordered by a distance-(k+1)
    colouring of the matrix graph (levels is then not used), the factor on A's pattern plus the fill of level <= k.
    """

    def __init__(self, csr, precond="jacobi", stop=_lib.STOP_SCIPY, mode=_lib.MODE_FP64, nrhs=1, maxiter=1000,
                 rtol=1e-8, atol=0.0, team=0, lanes=0, block=0, inner_rtol=1e-3, max_refine=60, levels=None,
                 inner_maxiter=400, fill_level=0, amg_max_levels=0, amg_coarse_max=0, method="bicgstab"):
        torch = _lib.require_cuda()
        if precond not in _lib.PREC:
            raise ValueError(f"Unknown preconditioner: {precond}")
        o = _lib.SolverOpts()
        o.precond, o.stop, o.mode, o.nrhs, o.maxiter = _lib.PREC[precond], stop, mode, nrhs, int(maxiter)
        o.team, o.lanes, o.block = team, lanes, block
        o.rtol, o.atol, o.inner_rtol, o.max_refine = float(rtol), float(atol), float(inner_rtol), int(max_refine)
        o.inner_maxiter = int(inner_maxiter)
        o.fill_level = int(fill_level)
        o.amg_max_levels, o.amg_coarse_max = int(amg_max_levels), int(amg_coarse_max)
        if method not in ("bicgstab", "cg"):
            raise ValueError(f"Unknown Krylov method: {method}")
        o.method = _lib.METHOD_CG if method == "cg" else _lib.METHOD_BICGSTAB
        self.method = method
        self.opts = o
        self.n, self.nrhs, self.mode = csr.n, nrhs, mode
        self.precond = precond
        lev = None
        if levels is not None:
            lev = np.ascontiguousarray(levels, dtype=np.int32)
        h = C.c_void_p()
        d = csr.desc()
        _lib.check(_lib.lib().kcfd_solver_create(C.byref(d), C.byref(o), _lib.ptr(lev), C.byref(h)),
                   "kcfd_solver_create")
        self._h = h
        dev = csr.vals64.device
        self.iters = torch.zeros(nrhs, dtype=torch.int32, device=dev)
        self.relres = torch.zeros(nrhs, dtype=torch.float64, device=dev)
        self.status = torch.zeros(nrhs, dtype=torch.int32, device=dev)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.release("kcfd_solver_destroy", h)
            except Exception:   # interpreter shutdown: the module may be gone already
                pass
            self._h = None

    def set_tolerances(self, rtol=None, atol=None, maxiter=None):
        """Tolerances live in the handle; a change re-creates nothing."""
        raise NotImplementedError("create a new Solver to change tolerances")

    def setup(self, csr, stream=None):
        d = csr.desc()
        _lib.check(_lib.lib().kcfd_solver_setup(self._h, C.byref(d), _lib.stream_handle(stream)), "kcfd_solver_setup")

    def solve(self, csr, b, x, stream=None):
        """x (FP64, [n] or [n, nrhs]) holds x0 on entry and the solution on return.
        Launches one kernel; returns the device arrays (iters, relres, status)."""
        if self.mode == _lib.MODE_MIXED and csr.vals32 is None:
            csr.refresh_fp32(stream)
        d = csr.desc()
        _lib.check(_lib.lib().kcfd_solver_solve(self._h, C.byref(d), _lib.ptr(b), _lib.ptr(x), _lib.ptr(self.iters),
                                                _lib.ptr(self.relres), _lib.ptr(self.status),
                                                _lib.stream_handle(stream)), "kcfd_solver_solve")
        return self.iters, self.relres, self.status

    def apply_precond(self, csr, r, z=None, stream=None):
        """z = M^-1 r with the set-up preconditioner (one right-hand side, FP64 tensors)."""
        torch = _lib.require_cuda()
        if z is None:
            z = torch.empty_like(r)
        d = csr.desc()
        _lib.check(_lib.lib().kcfd_solver_apply_precond(self._h, C.byref(d), _lib.ptr(r), _lib.ptr(z),
                                                        _lib.stream_handle(stream)), "kcfd_solver_apply_precond")
        return z

    def _amg_handle(self):
        h = C.c_void_p()
        _lib.check(_lib.lib().kcfd_solver_amg(self._h, C.byref(h)), "kcfd_solver_amg")
        if not h.value:
            raise ValueError("not an AMG handle")
        return h

    def amg_levels(self):
        """Rows, entries and prolongator entries of every multigrid level (precond 'amg')."""
        from .amg import levels_of
        return levels_of(self._amg_handle())

    def amg_info(self):
        """Levels, rows and entries per level and device bytes of the multigrid hierarchy
        (precond 'amg')."""
        from .amg import info_of
        return info_of(self._amg_handle())

    def info(self):
        """Resolved launch shape: dict(team, lanes, block, levels); levels is the ILU
        level count, or the multigrid level count with precond 'amg'."""
        v = np.zeros(4, dtype=np.int32)
        _lib.check(_lib.lib().kcfd_solver_info(self._h, v.ctypes.data_as(_lib.P_i32)), "kcfd_solver_info")
        return {"team": int(v[0]), "lanes": int(v[1]), "block": int(v[2]), "levels": int(v[3])}

    @property
    def graph_engine(self):
        """True when solves run as the handle's own CUDA graph (team 3). Such a solve
        is not nested into an enclosing stream capture (there it runs on the
        persistent grid kernel), so callers keep it outside their captures."""
        return self.info()["team"] == 3

    def barrier_error(self, stream=None):
        e = C.c_int32(0)
        _lib.check(_lib.lib().kcfd_solver_error(self._h, C.byref(e), _lib.stream_handle(stream)), "kcfd_solver_error")
        return e.value


class DeviceGraph:
    """The device work of the kcfd calls issued on `stream` inside the with-block,
    captured as a CUDA graph (kcfd_graph_*); launch() replays it. Allocate (handles,
    tensors) before the block; issue the calls on `stream` (pass it, or make it
    torch's current stream)."""

    def __init__(self, stream):
        self.stream = stream
        self._h = C.c_void_p()

    def __enter__(self):
        _lib.check(_lib.lib().kcfd_graph_capture_begin(_lib.stream_handle(self.stream)), "kcfd_graph_capture_begin")
        return self

    def __exit__(self, et, ev, tb):
        h = C.c_void_p()
        st = _lib.lib().kcfd_graph_capture_end(_lib.stream_handle(self.stream), C.byref(h))
        if et is None:
            _lib.check(st, "kcfd_graph_capture_end")
        self._h = h
        return False

    def launch(self, stream=None):
        _lib.check(_lib.lib().kcfd_graph_launch(self._h, _lib.stream_handle(stream or self.stream)),
                   "kcfd_graph_launch")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.release("kcfd_graph_destroy", h)
            except Exception:   # interpreter shutdown: the module may be gone already
                pass
            self._h = None
