"""Oracle: vectorised FP64 restatement of the reference FVM operators (test infrastructure).

Each function keeps the reference's per-element operation order and the order in
which contributions are accumulated (face-id order, owner before neighbour), so
that on the golden fixtures it reproduces the reference to the last bit or within
one rounding of a BLAS dot product.

Reference: core/fvm_operators.py, core/gradient.py, core/interpolation.py.
"""
from __future__ import annotations

import numpy as np
from scipy import sparse

LIMITERS = ("minmod", "superbee", "van_albada", "van_leer")


class System:
    """COO triplets + rhs + tracked diagonal (core/fvm_operators.py:13-56).

    Entries are kept in the reference's append order so that scipy's coo->csr
    duplicate summation sees the same sequence.
    """

    def __init__(self, n):
        self.n = n
        self.rows, self.cols, self.vals = [], [], []
        self.rhs = np.zeros(n)
        self.diag = np.zeros(n)

    def add_entries(self, r, c, v, diag_mask=None):
        r = np.asarray(r, dtype=np.int64); c = np.asarray(c, dtype=np.int64); v = np.asarray(v, dtype=np.float64)
        self.rows.append(r); self.cols.append(c); self.vals.append(v)
        dm = (r == c) if diag_mask is None else diag_mask
        if np.any(dm):
            np.add.at(self.diag, r[dm], v[dm])

    def add_source(self, idx, val):
        np.add.at(self.rhs, np.asarray(idx, dtype=np.int64), np.asarray(val, dtype=np.float64))

    def to_sparse(self):
        """core/fvm_operators.py:43-48: coo_matrix((vals,(rows,cols))).tocsr()."""
        if self.rows:
            r = np.concatenate(self.rows); c = np.concatenate(self.cols); v = np.concatenate(self.vals)
        else:
            r = c = np.zeros(0, np.int64); v = np.zeros(0)
        return sparse.coo_matrix((v, (r, c)), shape=(self.n, self.n)).tocsr()


def _norm_rows(v):
    return np.sqrt((v * v).sum(axis=1))


def _interleave(*cols):
    """Stack per-face columns so that flattening gives face-major, column-minor order."""
    return np.stack(cols, axis=1).reshape(-1)


def interp_weight(mesh):
    """gc for internal faces (core/gradient.py:102-114, core/interpolation.py:185-196,
    models/single_phase.py:380-388): dN/(dO+dN), 0.5 when degenerate."""
    gc = np.full(mesh.n_faces, 0.5)
    it = mesh.neighbour >= 0
    fc = mesh.fcenter[it]
    dO = _norm_rows(fc - mesh.ccenter[mesh.owner[it]])
    dN = _norm_rows(fc - mesh.ccenter[mesh.neighbour[it]])
    tot = dO + dN
    g = np.where(tot < 1e-30, 0.5, dN / np.where(tot < 1e-30, 1.0, tot))
    gc[it] = g
    return gc


def face_patch_values(mesh, bvals_by_patch, owner_values):
    """Per-face boundary value: the patch value of the face, else the owner value
    (core/gradient.py:117-127)."""
    out = owner_values[mesh.owner].copy()
    for name, fids in mesh.boundary_patches.items():
        if name in bvals_by_patch:
            out[fids] = bvals_by_patch[name]
    return out


def diffusion_operator(mesh, gamma, system):
    """core/fvm_operators.py:59-100 (harmonic-mean Gamma, |d_PN|, internal faces only)."""
    it = np.nonzero(mesh.neighbour >= 0)[0]
    o, nb = mesh.owner[it], mesh.neighbour[it]
    d = _norm_rows(mesh.ccenter[nb] - mesh.ccenter[o])
    keep = ~(d < 1e-30)
    it, o, nb, d = it[keep], o[keep], nb[keep], d[keep]
    gO, gN = gamma[o], gamma[nb]
    s = gO + gN
    gf = np.where(s > 1e-30, 2.0 * gO * gN / np.where(s > 1e-30, s, 1.0), 0.0)
    coeff = gf * mesh.area[it] / d
    r = _interleave(o, nb, o, nb)
    c = _interleave(o, nb, nb, o)
    v = _interleave(coeff, coeff, -coeff, -coeff)
    system.add_entries(r, c, v)


def convection_operator_upwind(mesh, mf, system):
    """core/fvm_operators.py:103-129 (first-order upwind; outflow boundary on the diagonal)."""
    F = mf
    internal = mesh.neighbour >= 0
    o = mesh.owner
    nb = np.where(internal, mesh.neighbour, o)
    zero = np.zeros_like(F)
    # four slots per face; boundary faces use slot 0 only and only for F >= 0
    r = _interleave(o, o, nb, nb)
    c = _interleave(o, nb, nb, o)
    v = _interleave(np.where(internal, np.maximum(F, 0.0), F), np.minimum(F, 0.0),
                    np.maximum(-F, 0.0), np.minimum(-F, 0.0))
    m = _interleave(internal | (F >= 0), internal, internal, internal)
    del zero
    system.add_entries(r[m], c[m], v[m])


def temporal_operator(mesh, rho, dt, phi_old, system):
    """core/fvm_operators.py:132-148 (backward Euler)."""
    coeff = rho * mesh.volume / dt
    idx = np.arange(mesh.n_cells)
    system.add_entries(idx, idx, coeff)
    system.add_source(idx, coeff * phi_old)


def source_term(mesh, S, system):
    """core/fvm_operators.py:151-161."""
    system.add_source(np.arange(mesh.n_cells), S * mesh.volume)


def linearized_source(mesh, Sp, Su, system):
    """core/fvm_operators.py:164-175: diagonal -Sp V, rhs Su V."""
    idx = np.arange(mesh.n_cells)
    system.add_entries(idx, idx, -Sp * mesh.volume)
    system.add_source(idx, Su * mesh.volume)


def apply_boundary_conditions(mesh, phi_b_by_patch, gamma, mf, system, bc_types):
    """core/fvm_operators.py:178-225 (dirichlet / neumann / zero_gradient), patches in
    mesh order, faces in patch order."""
    for bname, fids in mesh.boundary_patches.items():
        bc = bc_types.get(bname, {"type": "zero_gradient"})
        t = bc["type"]
        o = mesh.owner[fids]
        dPf = _norm_rows(mesh.fcenter[fids] - mesh.ccenter[o])
        ok = ~(dPf < 1e-30)
        li = np.nonzero(ok)[0]
        f, o, dPf = fids[ok], o[ok], dPf[ok]
        if t == "dirichlet":
            phib = np.asarray(phi_b_by_patch[bname])[li]
            coeff = gamma[o] * mesh.area[f] / dPf
            F = mf[f]
            system.add_entries(o, o, coeff)
            # rhs order per face: coeff*phi_b, then -F*phi_b for inflow
            inflow = F < 0
            src_i = _interleave(o, o)
            src_v = _interleave(coeff * phib, np.where(inflow, -F * phib, 0.0))
            src_m = _interleave(np.ones(len(o), bool), inflow)
            system.add_source(src_i[src_m], src_v[src_m])
        elif t == "neumann":
            flux = bc.get("value", 0.0) * mesh.area[f]
            system.add_source(o, flux)
        elif t == "zero_gradient":
            F = mf[f]
            m = F < 0
            system.add_entries(o[m], o[m], -F[m])


def under_relax(system, phi, alpha):
    """core/fvm_operators.py:228-240 (uses the tracked diagonal)."""
    if alpha >= 1.0:
        return
    ap = system.diag.copy()
    add = ap * (1.0 - alpha) / alpha
    idx = np.arange(system.n)
    system.add_entries(idx, idx, add)
    system.rhs += add * phi


def green_gauss_gradient(mesh, phi, phi_face_b):
    """core/gradient.py:12-48. phi_face_b: per-face boundary value (ignored on internal
    faces)."""
    ndim = mesh.ndim
    n = mesh.n_cells
    internal = mesh.neighbour >= 0
    gc = interp_weight(mesh)
    nb = np.where(internal, mesh.neighbour, mesh.owner)
    phif = np.where(internal, gc * phi[mesh.owner] + (1.0 - gc) * phi[nb], phi_face_b)
    flux = phif[:, None] * mesh.normal[:, :ndim] * mesh.area[:, None]
    grad = np.zeros((n, ndim))
    idx = _interleave(mesh.owner, nb)
    val = np.stack([flux, np.where(internal[:, None], -flux, 0.0)], axis=1).reshape(-1, ndim)
    m = _interleave(np.ones(mesh.n_faces, bool), internal)
    np.add.at(grad, idx[m], val[m])
    vol = mesh.volume
    ok = vol > 1e-30
    grad[ok] = grad[ok] / vol[ok][:, None]
    return grad


def compute_mass_flux(mesh, U, U_face_b, rho):
    """core/interpolation.py:163-182: F = rho (u_f . n) A, u_f by gc on internal faces,
    the patch value on boundary faces."""
    internal = mesh.neighbour >= 0
    gc = interp_weight(mesh)
    nb = np.where(internal, mesh.neighbour, mesh.owner)
    uf = np.where(internal[:, None], gc[:, None] * U[mesh.owner] + (1.0 - gc)[:, None] * U[nb], U_face_b)
    dot = np.zeros(mesh.n_faces)
    for k in range(mesh.ndim):
        dot = dot + uf[:, k] * mesh.normal[:, k]
    return rho * dot * mesh.area


def limiter(name, r):
    """core/interpolation.py:17-44."""
    if name == "minmod":
        return np.maximum(0.0, np.minimum(1.0, r))
    if name == "superbee":
        return np.maximum(0.0, np.maximum(np.minimum(2.0 * r, 1.0), np.minimum(r, 2.0)))
    if name == "van_albada":
        return np.where(r > 0, (r * r + r) / (r * r + 1.0), 0.0)
    if name == "van_leer":
        with np.errstate(divide="ignore", invalid="ignore"):  # r = -1 lies in the discarded branch
            return np.where(r > 0, 2.0 * r / (1.0 + r), 0.0)
    raise ValueError(f"Unknown limiter: {name}")


def muscl_deferred_correction(mesh, phi, mf, grad, limiter_name="van_leer"):
    """core/interpolation.py:227-303: corr = |F| * 0.5 psi(r) (phi_D - phi_U), removed from
    the upwind cell and added to the downwind cell; faces with |phi_D-phi_U| < 1e-15 skip."""
    it = np.nonzero(mesh.neighbour >= 0)[0]
    o, nb = mesh.owner[it], mesh.neighbour[it]
    F = mf[it]
    pos = F >= 0
    up = np.where(pos, o, nb)
    dn = np.where(pos, nb, o)
    phiU, phiD = phi[up], phi[dn]
    dx = mesh.fcenter[it] - mesh.ccenter[up]
    dot = np.zeros(len(it))
    for k in range(mesh.ndim):
        dot = dot + grad[up, k] * dx[:, k]
    lin = phiU + dot
    dface = lin - phiU
    dcd = phiD - phiU
    keep = ~(np.abs(dcd) < 1e-15)
    safe = np.where(keep, dcd, 1.0)
    r = 2.0 * dface / safe - 1.0
    psi = limiter(limiter_name, r)
    muscl = phiU + 0.5 * psi * dcd
    fcorr = np.abs(F) * (muscl - phiU)
    corr = np.zeros(mesh.n_cells)
    idx = _interleave(up, dn)
    val = _interleave(-fcorr, fcorr)
    m = _interleave(keep, keep)
    np.add.at(corr, idx[m], val[m])
    return corr


def least_squares_gradient(mesh, phi, phi_face_b):
    """core/gradient.py:51-99: per cell, over its faces in the cell's own face order,
    dx = x_N - x_P (internal; N the other cell) or x_f - x_P (boundary, with the
    patch value), dphi likewise; grad = solve(A^T A, A^T dphi); zero for cells with
    fewer than ndim faces or a singular A^T A. phi_face_b: per-face boundary value."""
    nd = mesh.ndim
    n = mesh.n_cells
    cf = mesh.cell_faces
    grad = np.zeros((n, nd))
    for ci in range(n):
        fids = cf[ci][cf[ci] >= 0]
        if len(fids) < nd:
            continue
        xP = mesh.ccenter[ci, :nd]
        rows, rhs = [], []
        for f in fids:
            if mesh.neighbour[f] >= 0:
                nb = mesh.neighbour[f] if mesh.owner[f] == ci else mesh.owner[f]
                rows.append(mesh.ccenter[nb, :nd] - xP)
                rhs.append(phi[nb] - phi[ci])
            else:
                rows.append(mesh.fcenter[f, :nd] - xP)
                rhs.append(phi_face_b[f] - phi[ci])
        A = np.array(rows)
        b = np.array(rhs)
        try:
            grad[ci] = np.linalg.solve(A.T @ A, A.T @ b)
        except np.linalg.LinAlgError:
            pass
    return grad
