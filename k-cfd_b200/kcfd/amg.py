"""Smoothed-aggregation algebraic multigrid on the device (libkcfd kcfd_amg_*).

The device counterpart of create_preconditioner(A, 'amg') (core/preconditioner.py:63-74,
pyamg's smoothed_aggregation_solver(A).aspreconditioner() in the reference). The
hierarchy's patterns are built once per sparsity pattern (AMG(csr)); setup(csr)
refreshes every level's values from the matrix's current values on the device, and
apply(b, x) runs one V(1,1) cycle, x = M^-1 b. As the preconditioner of a Solver
(precond='amg') the cycle runs inside the graph engine's loop instead.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def info_of(h):
    nl = C.c_int32(0)
    rn = np.zeros(32, dtype=np.int64)
    by = C.c_int64(0)
    _lib.check(_lib.lib().kcfd_amg_info(h, C.byref(nl), rn.ctypes.data_as(_lib.P_i64), C.byref(by)), "kcfd_amg_info")
    L = nl.value
    return {"levels": L, "rows": rn[0:2 * L:2].tolist(), "nnz": rn[1:2 * L:2].tolist(), "device_bytes": by.value}


def levels_of(h):
    """Per level: rows, entries and (above the coarsest) prolongator entries."""
    inf = info_of(h)
    out = []
    for l in range(inf["levels"]):
        d = {"rows": inf["rows"][l], "nnz": inf["nnz"][l], "p_nnz": 0}
        if l < inf["levels"] - 1:
            pip = np.zeros(inf["rows"][l] + 1, dtype=np.int32)
            _lib.check(_lib.lib().kcfd_amg_export(h, l, _lib.AMG_ITEMS["p_indptr"], pip.ctypes.data), "kcfd_amg_export")
            d["p_nnz"] = int(pip[-1])
        out.append(d)
    return out


class AMG:
    def __init__(self, csr, mode=_lib.MODE_FP64, coarse_max=0, max_levels=0, power_iters=0):
        _lib.require_cuda()
        o = _lib.AmgOpts()
        o.mode, o.coarse_max, o.max_levels, o.power_iters = int(mode), int(coarse_max), int(max_levels), int(power_iters)
        h = C.c_void_p()
        d = csr.desc()
        _lib.check(_lib.lib().kcfd_amg_create(C.byref(d), C.byref(o), C.byref(h)), "kcfd_amg_create")
        self._h = h
        self.n = csr.n
        self.mode = mode

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.release("kcfd_amg_destroy", h)
            except Exception:   # interpreter shutdown: the module may be gone already
                pass
            self._h = None

    def setup(self, csr, stream=None):
        d = csr.desc()
        _lib.check(_lib.lib().kcfd_amg_setup(self._h, C.byref(d), _lib.stream_handle(stream)), "kcfd_amg_setup")

    def apply(self, b, x=None, stream=None):
        """x = M^-1 b on the device (FP64 tensors of n entries)."""
        torch = _lib.require_cuda()
        if x is None:
            x = torch.empty_like(b)
        _lib.check(_lib.lib().kcfd_amg_apply(self._h, _lib.ptr(b), _lib.ptr(x), _lib.stream_handle(stream)),
                   "kcfd_amg_apply")
        return x

    def info(self):
        return info_of(self._h)

    def export(self, level, item):
        """One item of a level as a host array (synchronises the device): 'aggregates',
        'indptr', 'indices', 'values', 'p_indptr', 'p_indices', 'p_values', 'omega',
        'coarse_inverse'."""
        inf = self.info()
        n, nnz = inf["rows"][level], inf["nnz"][level]
        if item in ("p_indices", "p_values"):
            pip = self.export(level, "p_indptr")
            size = int(pip[-1])
        else:
            size = {"aggregates": n, "indptr": n + 1, "indices": nnz, "values": nnz, "p_indptr": n + 1, "omega": 1,
                    "coarse_inverse": n * n}[item]
        dt = np.float64 if item in ("values", "p_values", "omega", "coarse_inverse") else np.int32
        out = np.zeros(max(size, 1), dtype=dt)
        _lib.check(_lib.lib().kcfd_amg_export(self._h, int(level), _lib.AMG_ITEMS[item], out.ctypes.data),
                   "kcfd_amg_export")
        return out[:size]

    def level_matrix(self, level, A0=None):
        """Level `level`'s operator as a scipy CSR (level 0: A0's values)."""
        from scipy import sparse
        inf = self.info()
        n = inf["rows"][level]
        ip, ix = self.export(level, "indptr"), self.export(level, "indices")
        v = self.export(level, "values") if level > 0 else np.asarray(A0.data, dtype=np.float64)
        return sparse.csr_matrix((v, ix, ip), shape=(n, n))

    def prolongator(self, level):
        from scipy import sparse
        inf = self.info()
        pip, pix, pv = self.export(level, "p_indptr"), self.export(level, "p_indices"), self.export(level, "p_values")
        return sparse.csr_matrix((pv, pix, pip), shape=(inf["rows"][level], inf["rows"][level + 1]))
