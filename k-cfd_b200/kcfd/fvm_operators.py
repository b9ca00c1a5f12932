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
