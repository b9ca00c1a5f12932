"""Oracle: linear solvers of the reference hot path, restated in numpy (test infrastructure).

* bicgstab_gpu_semantics -- core/gpu_solver.py:158-199 (_cpu_bicgstab, the CPU twin of
  the CuPy path :111-155): unpreconditioned; stops when ||s||/||b|| < tol (after
  x += alpha p) or ||r||/||b|| < tol; guards at 1e-30 zero the scalar instead of
  stopping, except rho which stops.
* bicgstab_scipy -- the loop of scipy.sparse.linalg.bicgstab (scipy 1.18.1, the
  reference's dependency, called from core/linear_solver.py:59 with atol=tol and the
  default rtol=1e-5): stop when ||r|| < max(atol, rtol ||b||) at the top of an
  iteration or ||s|| below it mid-iteration; rho/omega breakdown at eps^2.
* jacobi -- core/preconditioner.py:43-47 (1/d where |d| > 1e-30, else 0).
* ilu0 -- structural ILU(0) (no fill outside the pattern), Saad's IKJ variant, in an
  optional symmetric row/column ordering. The reference's 'ilu0' is SuperLU spilu
  (core/preconditioner.py:49-54), which is not a structural ILU(0); parity with it is
  at the solution level only.
* distance_colouring / iluk_pattern / iluk_factor -- the structural ILU(k) of the
  kcfd device path (not the reference's 'iluk', which is SuperLU's threshold ILU with
  fill_factor=3, core/preconditioner.py:56-61): rows ordered by a greedy distance-
  (k+1) colouring of A's symmetrised graph, the level-of-fill pattern of that order
  (Saad, Iterative Methods for Sparse Linear Systems, 10.3.3: lev(i,j) =
  min(lev(i,j), lev(i,k) + lev(k,j) + 1), kept when <= k), and the IKJ factorisation
  restricted to that pattern. ilu0_apply applies it.
"""
from __future__ import annotations

import numpy as np
from scipy import sparse


def bicgstab_gpu_semantics(A, b, x0=None, tol=1e-6, max_iter=1000):
    x = x0.copy() if x0 is not None else np.zeros_like(b)
    r = b - A @ x
    r_hat = r.copy()
    rho = alpha = omega = 1.0
    v = np.zeros_like(b)
    p = np.zeros_like(b)
    b_norm = np.linalg.norm(b)
    iters = 0
    if b_norm < 1e-30:
        return x, iters
    for it in range(max_iter):
        iters = it + 1
        rho_new = np.dot(r_hat, r)
        if abs(rho_new) < 1e-30:
            break
        beta = (rho_new / rho) * (alpha / omega) if abs(rho * omega) > 1e-30 else 0.0
        p = r + beta * (p - omega * v)
        v = A @ p
        denom = np.dot(r_hat, v)
        alpha = rho_new / denom if abs(denom) > 1e-30 else 0.0
        s = r - alpha * v
        if np.linalg.norm(s) / b_norm < tol:
            x += alpha * p
            break
        t = A @ s
        t_dot_t = np.dot(t, t)
        omega = np.dot(t, s) / t_dot_t if t_dot_t > 1e-30 else 0.0
        x += alpha * p + omega * s
        r = s - omega * t
        rho = rho_new
        if np.linalg.norm(r) / b_norm < tol:
            break
    return x, iters


def bicgstab_scipy(A, b, x0=None, rtol=1e-5, atol=0.0, maxiter=None, M=None):
    """Returns (x, info, iterations started)."""
    n = len(b)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    bnrm2 = np.linalg.norm(b)
    atol = max(float(atol), float(rtol) * float(bnrm2))
    if bnrm2 == 0:
        return b.copy(), 0, 0
    if maxiter is None:
        maxiter = n * 10
    psolve = (lambda z: z) if M is None else M
    rhotol = np.finfo(np.float64).eps ** 2
    omegatol = rhotol
    r = b - A @ x if x.any() else b.copy()
    rtilde = r.copy()
    rho_prev = omega = alpha = p = v = None
    for iteration in range(maxiter):
        if np.linalg.norm(r) < atol:
            return x, 0, iteration
        rho = np.dot(rtilde, r)
        if np.abs(rho) < rhotol:
            return x, -10, iteration
        if iteration > 0:
            if np.abs(omega) < omegatol:
                return x, -11, iteration
            beta = (rho / rho_prev) * (alpha / omega)
            p -= omega * v
            p *= beta
            p += r
        else:
            s = np.empty_like(r)
            p = r.copy()
        phat = psolve(p)
        v = A @ phat
        rv = np.dot(rtilde, v)
        if rv == 0:
            return x, -11, iteration + 1
        alpha = rho / rv
        r -= alpha * v
        s[:] = r[:]
        if np.linalg.norm(s) < atol:
            x += alpha * phat
            return x, 0, iteration + 1
        shat = psolve(s)
        t = A @ shat
        omega = np.dot(t, s) / np.dot(t, t)
        x += alpha * phat
        x += omega * shat
        r -= omega * t
        rho_prev = rho
    return x, maxiter, maxiter


def jacobi(A):
    d = A.diagonal()
    safe = np.where(np.abs(d) > 1e-30, d, 1.0)
    dinv = np.where(np.abs(d) > 1e-30, 1.0 / safe, 0.0)
    return lambda z: dinv * z


def ilu0_factor(A, perm=None):
    """Structural ILU(0) of P A P^T (P from perm: new row k = old row perm[k]).

    Returns (B, perm) where B holds L (strict lower, unit diagonal implied) and U
    (upper incl. diagonal) in the pattern of P A P^T, canonical CSR.
    """
    A = sparse.csr_matrix(A)
    n = A.shape[0]
    if perm is None:
        perm = np.arange(n)
    B = A[perm][:, perm].tocsr()
    B.sort_indices()
    ip, ix, val = B.indptr, B.indices, B.data.astype(np.float64).copy()
    diagpos = np.empty(n, dtype=np.int64)
    for i in range(n):
        lo, hi = ip[i], ip[i + 1]
        k = lo + np.searchsorted(ix[lo:hi], i)
        diagpos[i] = k
    for i in range(n):
        lo, hi = ip[i], ip[i + 1]
        cols = ix[lo:hi]
        pos = {int(c): lo + j for j, c in enumerate(cols)}
        for kk in range(lo, diagpos[i]):
            k = int(ix[kk])
            val[kk] = val[kk] / val[diagpos[k]]
            lik = val[kk]
            for jj in range(diagpos[k] + 1, ip[k + 1]):
                j = int(ix[jj])
                q = pos.get(j)
                if q is not None:
                    val[q] -= lik * val[jj]
    B = sparse.csr_matrix((val, ix.copy(), ip.copy()), shape=(n, n))
    return B, np.asarray(perm)


def distance_colouring(A, d):
    """Greedy colouring in row order: each row takes the smallest colour not used by a
    row within d edges of it in the symmetrised graph of A."""
    A = sparse.csr_matrix(A)
    n = A.shape[0]
    P = sparse.csr_matrix((np.ones(len(A.indices)), A.indices, A.indptr), shape=A.shape)
    G = (P + P.T).tocsr()
    colour = -np.ones(n, dtype=np.int64)
    for v in range(n):
        seen = {v}
        front = [v]
        near = set()
        for _ in range(d):
            nxt = []
            for u in front:
                for w in G.indices[G.indptr[u]:G.indptr[u + 1]]:
                    w = int(w)
                    if w in seen:
                        continue
                    seen.add(w)
                    nxt.append(w)
                    if colour[w] >= 0:
                        near.add(int(colour[w]))
            front = nxt
        c = 0
        while c in near:
            c += 1
        colour[v] = c
    return colour


def iluk_pattern(B, k):
    """Level-of-fill pattern (rows of sorted columns, their levels) of the already
    ordered matrix B: A's entries at level 0, fill of level <= k."""
    B = sparse.csr_matrix(B)
    B.sort_indices()
    n = B.shape[0]
    rows, levs = [], []
    for i in range(n):
        lev = {int(c): 0 for c in B.indices[B.indptr[i]:B.indptr[i + 1]]}
        done = set()
        while True:
            pending = sorted(c for c in lev if c < i and c not in done)
            if not pending:
                break
            kk = pending[0]
            done.add(kk)
            for j, lj in zip(rows[kk], levs[kk]):
                if j <= kk:
                    continue
                nl = lev[kk] + lj + 1
                if nl <= k and nl < lev.get(j, k + 1):
                    lev[j] = nl
        cols = sorted(lev)
        rows.append(cols)
        levs.append([lev[c] for c in cols])
    return rows, levs


def iluk_factor(A, k):
    """ILU(k) of P A P^T in the colouring order. Returns (F, perm, colour) with F the
    factor (L strict lower with unit diagonal implied, U upper) on the fill pattern."""
    A = sparse.csr_matrix(A)
    n = A.shape[0]
    colour = distance_colouring(A, k + 1)
    perm = np.argsort(colour, kind="stable")
    B = A[perm][:, perm].tocsr()
    B.sort_indices()
    rows, _ = iluk_pattern(B, k)
    ip = np.zeros(n + 1, dtype=np.int64)
    ip[1:] = np.cumsum([len(r) for r in rows])
    ix = np.concatenate([np.asarray(r, dtype=np.int64) for r in rows])
    val = np.zeros(len(ix))
    for i in range(n):
        pos = {int(c): ip[i] + q for q, c in enumerate(rows[i])}
        for kk in range(B.indptr[i], B.indptr[i + 1]):
            val[pos[int(B.indices[kk])]] = B.data[kk]
    diagpos = np.array([ip[i] + rows[i].index(i) for i in range(n)])
    for i in range(n):
        lo = ip[i]
        pos = {int(c): lo + q for q, c in enumerate(rows[i])}
        for kk in range(lo, diagpos[i]):
            kr = int(ix[kk])
            val[kk] = val[kk] / val[diagpos[kr]]
            lik = val[kk]
            for jj in range(diagpos[kr] + 1, ip[kr + 1]):
                q = pos.get(int(ix[jj]))
                if q is not None:
                    val[q] -= lik * val[jj]
    F = sparse.csr_matrix((val, ix, ip), shape=(n, n))
    return F, perm, colour


def ilu0_apply(B, perm, r):
    """z = (LU)^{-1} applied in the permuted ordering: z[perm] = U^{-1} L^{-1} r[perm]."""
    n = B.shape[0]
    ip, ix, val = B.indptr, B.indices, B.data
    y = np.array(r[perm], dtype=np.float64)
    for i in range(n):
        s = y[i]
        for kk in range(ip[i], ip[i + 1]):
            j = ix[kk]
            if j < i:
                s -= val[kk] * y[j]
        y[i] = s
    zp = np.zeros(n)
    for i in range(n - 1, -1, -1):
        s = y[i]
        d = 1.0
        for kk in range(ip[i], ip[i + 1]):
            j = ix[kk]
            if j > i:
                s -= val[kk] * zp[j]
            elif j == i:
                d = val[kk]
        zp[i] = s / d
    z = np.empty(n)
    z[perm] = zp
    return z


def spilu_reference(A):
    """The reference's 'ilu0' preconditioner (core/preconditioner.py:49-54)."""
    from scipy.sparse.linalg import spilu
    ilu = spilu(sparse.csr_matrix(A).tocsc(), fill_factor=1, drop_tol=0)
    return ilu.solve


def greedy_colouring(A):
    """Greedy colouring of A's rows in row order: each row takes the smallest colour not
    used by an already coloured neighbour (off-diagonal entries of its row). The same
    rule as the device mesh builder's cell colouring (one colour per level of the
    device ILU(0)); on hexahedral meshes it gives the red-black parity colouring."""
    A = sparse.csr_matrix(A)
    n = A.shape[0]
    ip, ix = A.indptr.tolist(), A.indices.tolist()
    col = [-1] * n
    for i in range(n):
        used = {col[j] for j in ix[ip[i]:ip[i + 1]] if j != i and col[j] >= 0}
        c = 0
        while c in used:
            c += 1
        col[i] = c
    return np.asarray(col, dtype=np.int64)


def ilu0_two_colour(A, colour):
    """Structural ILU(0) of A in a two-colour ordering (colour 0 rows first, row order
    kept inside a colour), vectorised: with no coupling inside a colour the factor is
    L = I + A_10 D_0^-1, U = [D_0, A_01; 0, D_1'] with D_1' = D_1 - diag(A_10 D_0^-1 A_01)
    -- the IKJ ILU(0) (ilu0_factor) of the permuted matrix, entry for entry. Returns
    M^-1 as a function of a vector in A's own ordering."""
    A = sparse.csr_matrix(A)
    colour = np.asarray(colour)
    if colour.max() > 1:
        raise ValueError("ilu0_two_colour needs a two-colour ordering")
    r = np.flatnonzero(colour == 0)
    k = np.flatnonzero(colour == 1)
    A00, A01 = A[r][:, r], A[r][:, k]
    A10, A11 = A[k][:, r], A[k][:, k]
    if (A00 - sparse.diags(A00.diagonal())).count_nonzero() or (A11 - sparse.diags(A11.diagonal())).count_nonzero():
        raise ValueError("rows of one colour are coupled")
    d0 = A00.diagonal()
    L10 = (A10 @ sparse.diags(1.0 / d0)).tocsr()
    d1 = A11.diagonal() - np.asarray(L10.multiply(A01.T.tocsr()).sum(axis=1)).ravel()
    A01 = A01.tocsr()

    def apply(q):
        q = np.asarray(q, dtype=np.float64)
        y0 = q[r]
        z1 = (q[k] - L10 @ y0) / d1
        z = np.empty_like(q)
        z[k] = z1
        z[r] = (y0 - A01 @ z1) / d0
        return z

    return apply
