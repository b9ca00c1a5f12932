"""Oracle: smoothed-aggregation algebraic multigrid — test infrastructure.

The reference's 'amg' preconditioner is pyamg's smoothed_aggregation_solver(A)
.aspreconditioner() (core/preconditioner.py:63-74); pyamg is an optional dependency
that is not installed here (without it the reference falls back to no
preconditioner), so parity with it is at the solution level. This module restates
the published method the device hierarchy follows -- smoothed aggregation (Vanek,
Mandel and Brezina, "Algebraic multigrid by smoothed aggregation for second and
fourth order elliptic problems", Computing 56, 1996) -- with the exact aggregation
rule and formulas of the device set-up, so that the aggregates are compared bit for
bit and the operators to rounding:

* strength: every stored off-diagonal entry of row i links i to its column
  (structural strength: the aggregates depend on the pattern only, so the device
  builds them once per pattern and refreshes only the values);
* aggregation, three greedy passes in row order:
  1. a row whose strong neighbours are all free starts an aggregate with them
     (a row with no strong neighbour is left for pass 3);
  2. a free row joins the pass-1 aggregate that holds the most of its neighbours
     (on a tie, the one met first in row order);
  3. a row still free starts an aggregate with its free strong neighbours;
* tentative prolongator T_iJ = 1 when row i is in aggregate J;
* smoothed prolongator P = (I - omega D^-1 A) T with omega = (4/3) / rho; rho is the
  Gershgorin bound max_i sum_j |a_ij| |dinv_i| on level 0 and a power-iteration
  estimate of rho(D^-1 A) (8 steps from a fixed hashed start vector) below, where the
  bound overestimates (about 2 against a measured 1.2 on the p' hierarchies);
* Galerkin coarse operator A_c = P^T A P, formed as P^T (A P);
* levels are added until a level has at most `coarse_max` rows, coarsening stalls
  (more than 0.8 of the rows kept) or `max_levels` is reached; the coarsest level is
  solved exactly (dense Gauss-Jordan inverse with partial pivoting);
* V(1,1) cycle with damped Jacobi (weight omega of the level) from a zero guess:
  x = omega D^-1 b; r = b - A x; x += P V(P^T r); x += omega D^-1 (b - A x).
"""
from __future__ import annotations

import numpy as np
from scipy import sparse


def strength(A):
    """Boolean mask over A's stored entries (CSR order): the off-diagonal links."""
    A = A.tocsr()
    n = A.shape[0]
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    return rows != A.indices


def aggregate(A):
    """Aggregate id of every row (the three passes above) and the aggregate count."""
    A = A.tocsr()
    n = A.shape[0]
    ip, ix = A.indptr, A.indices
    strong = strength(A)
    agg = -np.ones(n, dtype=np.int64)
    na = 0
    # pass 1
    for i in range(n):
        if agg[i] >= 0:
            continue
        s = ix[ip[i]:ip[i + 1]][strong[ip[i]:ip[i + 1]]]
        if len(s) == 0 or np.any(agg[s] >= 0):
            continue
        agg[i] = na
        agg[s] = na
        na += 1
    p1 = agg.copy()
    # pass 2: join the pass-1 aggregate holding most of the row's neighbours
    for i in range(n):
        if agg[i] >= 0:
            continue
        cand, cnt = [], []
        for k in range(ip[i], ip[i + 1]):
            a = p1[ix[k]]
            if strong[k] and a >= 0:
                if a in cand:
                    cnt[cand.index(a)] += 1
                else:
                    cand.append(a)
                    cnt.append(1)
        if cand:
            agg[i] = cand[int(np.argmax(cnt))]
    # pass 3
    for i in range(n):
        if agg[i] >= 0:
            continue
        s = ix[ip[i]:ip[i + 1]][strong[ip[i]:ip[i + 1]]]
        agg[i] = na
        free = s[agg[s] < 0]
        agg[free] = na
        na += 1
    return agg, na


def _dinv(A):
    """1/a_ii where |a_ii| > 1e-30, else 0 (the Jacobi rule of core/preconditioner.py:43-47)."""
    d = A.diagonal()
    return np.where(np.abs(d) > 1e-30, 1.0 / np.where(d == 0, 1.0, d), 0.0)


def gershgorin_omega(A):
    """omega = (4/3) / max_i sum_j |a_ij| |dinv_i| (level 0)."""
    A = A.tocsr()
    rs = np.asarray(abs(A).sum(axis=1)).ravel()
    r = float(np.max(rs * np.abs(_dinv(A))))
    return (4.0 / 3.0) / r if r > 1e-300 else 4.0 / 3.0


def power_omega(A, iters=8):
    """omega = (4/3) / lambda, lambda from `iters` power iterations on D^-1 A started at
    v_i = 0.5 + ((i * 2654435761) mod 2^32 >> 22) / 1024 (levels below 0)."""
    A = A.tocsr()
    n = A.shape[0]
    h = (np.arange(n, dtype=np.uint64) * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)
    v = 0.5 + (h >> np.uint64(22)).astype(np.float64) / 1024.0
    nv2 = float(v @ v)
    dinv = _dinv(A)
    for _ in range(iters):
        w = dinv * ((A @ v) * (1.0 / np.sqrt(nv2)))
        nv2 = float(w @ w)
        v = w
    lam = np.sqrt(nv2)
    return (4.0 / 3.0) / lam if lam > 1e-300 else 4.0 / 3.0


def prolongator(A, agg, na, omega):
    """P = (I - omega D^-1 A) T as CSR with sorted columns."""
    A = A.tocsr()
    n = A.shape[0]
    T = sparse.csr_matrix((np.ones(n), (np.arange(n), agg)), shape=(n, na))
    AT = A @ T
    P = T - sparse.diags(omega * _dinv(A)) @ AT
    P = P.tocsr()
    P.sort_indices()
    return P


def dense_inverse(M):
    """Gauss-Jordan inverse with partial pivoting (largest |entry| of the column, the
    first row on ties). A pivot not above 1e-13 of the largest |entry| of its column in
    the matrix before elimination drops its unknown: that row and column of the inverse
    are set to zero (per column, so that a row pinned by a huge diagonal does not drop
    the others)."""
    M = np.array(M, dtype=np.float64)
    n = M.shape[0]
    inv = np.eye(n)
    tol = 1e-13 * (np.abs(M).max(axis=0) if n else np.zeros(0))
    drop = np.zeros(n, dtype=bool)
    for k in range(n):
        col = np.abs(M[k:, k])
        p = k + int(np.argmax(col))
        if col[p - k] <= tol[k]:
            drop[k] = True
            continue
        if p != k:
            M[[k, p]] = M[[p, k]]
            inv[[k, p]] = inv[[p, k]]
        ip = 1.0 / M[k, k]
        M[k] *= ip
        inv[k] *= ip
        f = M[:, k].copy()
        f[k] = 0.0
        M -= np.outer(f, M[k])
        inv -= np.outer(f, inv[k])
    inv[drop, :] = 0.0
    inv[:, drop] = 0.0
    return inv


class Level:
    def __init__(self, A):
        self.A = A.tocsr()
        self.dinv = _dinv(self.A)
        self.omega = None
        self.P = None
        self.R = None
        self.agg = None


class Hierarchy:
    """The device hierarchy's rules: stop at <= coarse_max rows, at max_levels, or when
    an aggregation keeps more than 0.8 of the rows; the coarsest level must have at
    most dense_max rows."""

    def __init__(self, A, coarse_max=128, max_levels=12, power_iters=8, dense_max=256):
        self.levels = [Level(A)]
        while True:
            L = self.levels[-1]
            n = L.A.shape[0]
            if n <= coarse_max or len(self.levels) >= max_levels:
                break
            agg, na = aggregate(L.A)
            if na > 0.8 * n:
                break
            L.omega = gershgorin_omega(L.A) if len(self.levels) == 1 else power_omega(L.A, power_iters)
            L.agg = agg
            L.P = prolongator(L.A, agg, na, L.omega)
            L.R = L.P.T.tocsr()
            Ac = (L.R @ (L.A @ L.P)).tocsr()
            Ac.sort_indices()
            self.levels.append(Level(Ac))
        if self.levels[-1].A.shape[0] > dense_max:
            raise ValueError("AMG coarsening stopped at %d rows" % self.levels[-1].A.shape[0])
        self.coarse_inv = dense_inverse(self.levels[-1].A.toarray())

    def vcycle(self, b, l=0):
        L = self.levels[l]
        if l == len(self.levels) - 1:
            return self.coarse_inv @ b
        w = L.omega
        x = w * L.dinv * b
        r = b - L.A @ x
        xc = self.vcycle(L.R @ r, l + 1)
        x = x + L.P @ xc
        x = x + w * L.dinv * (b - L.A @ x)
        return x

    def operator(self):
        from scipy.sparse.linalg import LinearOperator
        n = self.levels[0].A.shape[0]
        return LinearOperator((n, n), matvec=lambda v: self.vcycle(np.asarray(v, dtype=np.float64).ravel()))

    def sizes(self):
        return [(L.A.shape[0], L.A.nnz) for L in self.levels]
