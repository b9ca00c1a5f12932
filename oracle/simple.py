"""Oracle: vectorised restatement of SIMPLESolver (models/single_phase.py) — test infrastructure.

Follows models/single_phase.py:
  solve_steady :70-101, _face_mass_flux :124-144, _momentum_eq :147-271,
  _pressure_correction :274-377, _gc :380-388.
Contributions are accumulated in face-id order with the reference's owner-then-
neighbour sequence, so on small meshes this reproduces the reference to rounding.

Extensions with no counterpart in the reference (parity unpinned, restated from the
published methods):
  * nonorth=True: over-relaxed non-orthogonal correction (Jasak 1996, sec. 3.3.1.3):
    S_f = Delta_f + k_f with Delta_f = (A_f / d_orth) d_PN, whose implicit part is the
    reference's own A_f/d_orth coefficient; the explicit part Gamma_f k_f . grad(phi)_f
    (gradient interpolated with g_c) goes to the owner rhs and, negated, to the
    neighbour rhs.
  * muscl=<limiter>: the reference's MUSCL deferred correction
    (core/interpolation.py:227-303) added to each momentum component's rhs, gradients
    by Green-Gauss with Dirichlet face values on velocity patches.
Linear solves: 'direct' (scipy spsolve, the reference as written) or iterative
BiCGSTAB (scipy's loop) with Jacobi / ILU preconditioning at a relative tolerance.
"""
from __future__ import annotations

import numpy as np
from scipy import sparse
from scipy.sparse.linalg import spsolve

from . import fvm
from . import linsolve


def _norm_rows(v):
    return np.sqrt((v * v).sum(axis=1))


class Simple:
    def __init__(self, mesh, rho=1.0, mu=1e-3):
        self.mesh = mesh
        self.rho = rho
        self.mu = mu
        n, ndim = mesh.n_cells, mesh.ndim
        self.U = np.zeros((n, ndim))
        self.p = np.zeros(n)
        self.U_b = {k: np.zeros((len(v), ndim)) for k, v in mesh.boundary_patches.items()}
        self.p_b = {k: np.zeros(len(v)) for k, v in mesh.boundary_patches.items()}
        self.bc_u, self.bc_p = {}, {}
        self.alpha_u, self.alpha_p = 0.7, 0.3
        self.max_outer_iter, self.tol = 500, 1e-6
        self.residuals = []
        self._aP = {c: np.ones(n) for c in range(ndim)}
        # solver options
        self.solver = "direct"      # or "bicgstab"
        self.rtol = 1e-8
        self.precond_u = "jacobi"
        self.precond_p = "jacobi"   # 'jacobi' | 'ilu0' (structural, two-colour) | 'spilu' (reference)
        self.maxiter = 5000
        self.muscl = None
        self.nonorth = False
        self.iters_log = []
        self._geom()

    # ---- set-up ----
    def set_velocity_bc(self, patch, bc_type, value=None):
        if patch not in self.mesh.boundary_patches:
            return
        if value is not None:
            self.U_b[patch][:] = np.asarray(value, dtype=float)
        self.bc_u[patch] = {"type": bc_type}

    def set_pressure_bc(self, patch, bc_type, value=None):
        if patch not in self.mesh.boundary_patches:
            return
        if value is not None:
            self.p_b[patch][:] = value
        self.bc_p[patch] = {"type": bc_type}

    def _geom(self):
        m = self.mesh
        it = m.neighbour >= 0
        self.it = it
        o = m.owner
        nb = np.where(it, m.neighbour, o)
        self.nb = nb
        fc, cc = m.fcenter, m.ccenter
        dvec = cc[nb] - cc[o]
        d_int = _norm_rows(dvec)
        d_bnd = _norm_rows(fc - cc[o])
        self.d = np.where(it, d_int, d_bnd)
        self.dvec = dvec
        dn = np.zeros(m.n_faces)
        for k in range(m.ndim):
            dn = dn + dvec[:, k] * m.normal[:, k]
        d_orth = np.abs(dn)
        self.d_orth = np.maximum(d_orth, 0.1 * d_int)
        dO = _norm_rows(fc - cc[o])
        dN = _norm_rows(fc - cc[nb])
        t = dO + dN
        self.gc = np.where(t > 1e-30, dN / np.where(t > 1e-30, t, 1.0), 0.5)
        # face -> (patch index, local index) for boundary faces
        self.face_patch = -np.ones(m.n_faces, dtype=np.int64)
        self.face_local = -np.ones(m.n_faces, dtype=np.int64)
        self.patch_names = list(m.boundary_patches.keys())
        for pi, (nm, fids) in enumerate(m.boundary_patches.items()):
            self.face_patch[fids] = pi
            self.face_local[fids] = np.arange(len(fids))

    def _face_bvals(self, store, bc):
        """Per-face boundary value arrays and a dirichlet mask."""
        m = self.mesh
        shape = (m.n_faces,) + store[self.patch_names[0]].shape[1:] if self.patch_names else (m.n_faces,)
        vals = np.zeros(shape)
        dirm = np.zeros(m.n_faces, dtype=bool)
        for nm, fids in m.boundary_patches.items():
            vals[fids] = store[nm]
            dirm[fids] = bc.get(nm, {"type": "zero_gradient"})["type"] == "dirichlet"
        return vals, dirm

    # ---- _face_mass_flux :124-144 ----
    def face_mass_flux(self):
        m = self.mesh
        ub, dirm = self._face_bvals(self.U_b, self.bc_u)
        o, nb, gc = m.owner, self.nb, self.gc
        uf_int = gc[:, None] * self.U[o] + (1 - gc)[:, None] * self.U[nb]
        uf_b = np.where(dirm[:, None], ub, self.U[o])
        uf = np.where(self.it[:, None], uf_int, uf_b)
        dot = np.zeros(m.n_faces)
        for k in range(m.ndim):
            dot = dot + uf[:, k] * m.normal[:, k]
        return self.rho * dot * m.area

    # ---- gradients of velocity components (extensions) ----
    def _grad_U(self, comp):
        m = self.mesh
        ub, dirm = self._face_bvals(self.U_b, self.bc_u)
        phi = self.U[:, comp]
        fb = np.where(dirm, ub[:, comp], phi[m.owner])
        return fvm.green_gauss_gradient(m, phi, fb)

    # ---- _momentum_eq :147-271 ----
    def momentum_system(self, comp, mf):
        """Returns (A_relaxed csr, b_relaxed, aP_relaxed)."""
        m = self.mesh
        n, F = m.n_cells, m.n_faces
        o, nb, it = m.owner, self.nb, self.it
        mu = self.mu
        Fm = mf
        ub, dirm = self._face_bvals(self.U_b, self.bc_u)
        valid = ~(self.d < 1e-30)
        # internal faces
        safe_do = np.where(it, self.d_orth, 1.0)
        Df_i = 2 * mu * mu / max(mu + mu, 1e-30) * m.area / safe_do
        Df_b = mu * m.area / np.where(valid, self.d, 1.0)
        # aP contributions per face, up to two slots each (owner, then neighbour or a
        # second owner term), in face order
        z = np.zeros(F)
        c_o1 = np.where(it, Df_i + np.maximum(Fm, 0), np.where(dirm, Df_b, np.where(Fm >= 0, Fm, -Fm)))
        c_2 = np.where(it, Df_i + np.maximum(-Fm, 0), np.where(dirm & (Fm >= 0), Fm, z))
        i_2 = np.where(it, nb, o)
        m_1 = valid & (it | (self.face_patch >= 0))
        m_2 = valid & (it | (dirm & (Fm >= 0)))
        aP = np.zeros(n)
        idx = np.stack([o, i_2], 1).reshape(-1)
        val = np.stack([c_o1, c_2], 1).reshape(-1)
        msk = np.stack([m_1, m_2], 1).reshape(-1)
        np.add.at(aP, idx[msk], val[msk])
        # rhs from dirichlet boundary faces: Df*phi_b then (-F)*phi_b for inflow
        b = np.zeros(n)
        phib = ub[:, comp] if ub.ndim == 2 else ub
        bd = ~it & dirm & valid
        bi = np.stack([o, o], 1).reshape(-1)
        bv = np.stack([Df_b * phib, (-Fm) * phib], 1).reshape(-1)
        bm = np.stack([bd, bd & (Fm < 0)], 1).reshape(-1)
        np.add.at(b, bi[bm], bv[bm])
        # off-diagonals (o,nb) then (nb,o) per internal face
        vi = it & valid
        aN_r = np.stack([o[vi], nb[vi]], 1).reshape(-1)
        aN_c = np.stack([nb[vi], o[vi]], 1).reshape(-1)
        aN_v = np.stack([-(Df_i[vi] + np.maximum(-Fm[vi], 0)), -(Df_i[vi] + np.maximum(Fm[vi], 0))], 1).reshape(-1)
        # pressure-gradient source :231-249
        pb, pdir = self._face_bvals(self.p_b, self.bc_p)
        pf_i = 0.5 * (self.p[o] + self.p[nb])
        pf_b = np.where(pdir, pb, self.p[o])
        src = np.where(it, pf_i, pf_b) * m.normal[:, comp] * m.area
        si = np.stack([o, nb], 1).reshape(-1)
        sv = np.stack([-src, src], 1).reshape(-1)
        sm = np.stack([np.ones(F, bool), it], 1).reshape(-1)
        np.add.at(b, si[sm], sv[sm])
        # extensions (no reference counterpart)
        if self.muscl is not None or self.nonorth:
            g = self._grad_U(comp)
            if self.muscl is not None:
                b = b + fvm.muscl_deferred_correction(m, self.U[:, comp], mf, g, self.muscl)
            if self.nonorth:
                b = b + self._nonorth_correction(g)
        # under-relaxation :251-258
        alpha = self.alpha_u
        phi_old = self.U[:, comp].copy()
        b = b + (1 - alpha) / alpha * aP * phi_old
        aP = aP / alpha
        rows = np.concatenate([aN_r, np.arange(n)])
        cols = np.concatenate([aN_c, np.arange(n)])
        vals = np.concatenate([aN_v, aP])
        A = sparse.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
        return A, b, aP

    def _nonorth_correction(self, g):
        """Explicit over-relaxed correction mu_f k_f . grad_f on internal faces."""
        m = self.mesh
        it = np.nonzero(self.it)[0]
        o, nb = m.owner[it], m.neighbour[it]
        gc = self.gc[it]
        S = m.normal[it] * m.area[it][:, None]
        k = S - (m.area[it] / self.d_orth[it])[:, None] * self.dvec[it]
        gf = gc[:, None] * g[o] + (1.0 - gc)[:, None] * g[nb]
        mu_f = 2 * self.mu * self.mu / max(self.mu + self.mu, 1e-30)
        kd = np.zeros(len(it))
        for c in range(m.ndim):
            kd = kd + k[:, c] * gf[:, c]
        flux = mu_f * kd
        corr = np.zeros(m.n_cells)
        np.add.at(corr, np.stack([o, nb], 1).reshape(-1), np.stack([flux, -flux], 1).reshape(-1))
        return corr

    def _solve(self, A, b, x0, precond):
        if self.solver == "direct":
            return spsolve(A, b), 0
        if precond == "jacobi":
            M = linsolve.jacobi(A)
        elif precond == "spilu":
            M = linsolve.spilu_reference(A)
        elif precond == "ilu0":
            # structural ILU(0) in the greedy (red-black on hexes) cell colouring, the
            # device's ILU(0) ordering; the colouring depends on the pattern only
            if getattr(self, "_colour", None) is None or len(self._colour) != A.shape[0]:
                self._colour = linsolve.greedy_colouring(A)
            M = linsolve.ilu0_two_colour(A, self._colour)
        elif precond == "none":
            M = None
        else:
            raise ValueError(precond)
        x, info, its = linsolve.bicgstab_scipy(A, b, x0=x0, rtol=self.rtol, atol=0.0, maxiter=self.maxiter, M=M)
        return x, its

    def momentum_eq(self, comp, mf):
        A, b, aP = self.momentum_system(comp, mf)
        self._aP[comp] = aP * self.alpha_u
        phi_old = self.U[:, comp].copy()
        x0 = phi_old if self.solver != "direct" else None
        phi, its = self._solve(A, b, x0, self.precond_u)
        self.iters_log.append(("u%d" % comp, its))
        if np.any(np.isnan(phi)):
            phi = phi_old
        self.U[:, comp] = phi
        r = np.linalg.norm(A @ phi - b)
        return r / max(np.linalg.norm(b), 1e-15)

    # ---- _pressure_correction :274-377 ----
    def pressure_system(self, mf):
        m = self.mesh
        n, F = m.n_cells, m.n_faces
        ndim = m.ndim
        o, nb, it = m.owner, self.nb, self.it
        aP_sum = sum(self._aP[c] for c in range(ndim))
        aP_mom = np.maximum(aP_sum / ndim, 1e-30)
        dP = m.volume / aP_mom
        valid_i = it & ~(self.d < 1e-30)
        df = self.rho * 0.5 * (dP[o] + dP[nb]) * m.area / np.where(it, self.d_orth, 1.0)
        pb, pdir = self._face_bvals(self.p_b, self.bc_p)
        bdir = ~it & pdir & (self.d > 1e-30) & (self.face_patch >= 0)
        df_b = self.rho * dP[o] * m.area / np.where(self.d > 1e-30, self.d, 1.0)
        aPp = np.zeros(n)
        idx = np.stack([o, nb], 1).reshape(-1)
        val = np.stack([np.where(it, df, df_b), df], 1).reshape(-1)
        msk = np.stack([valid_i | bdir, valid_i], 1).reshape(-1)
        np.add.at(aPp, idx[msk], val[msk])
        b = np.zeros(n)
        bi = np.stack([o, nb], 1).reshape(-1)
        bv = np.stack([-mf, mf], 1).reshape(-1)
        # mass imbalance counts on every face the loop does not skip
        bm = np.stack([valid_i | ~it, valid_i], 1).reshape(-1)
        np.add.at(b, bi[bm], bv[bm])
        r_ = np.concatenate([np.stack([o[valid_i], nb[valid_i]], 1).reshape(-1), np.arange(n)])
        c_ = np.concatenate([np.stack([nb[valid_i], o[valid_i]], 1).reshape(-1), np.arange(n)])
        v_ = np.concatenate([np.stack([-df[valid_i], -df[valid_i]], 1).reshape(-1), aPp])
        has_p_dir = any(v.get("type") == "dirichlet" for v in self.bc_p.values())
        if not has_p_dir:
            v_ = np.where(r_ == 0, 0.0, v_)
            r_ = np.concatenate([r_, [0]]); c_ = np.concatenate([c_, [0]]); v_ = np.concatenate([v_, [1.0]])
            b[0] = 0.0
        A = sparse.coo_matrix((v_, (r_, c_)), shape=(n, n)).tocsr()
        return A, b, dP

    def pp_face_values(self, pp):
        m = self.mesh
        fb = pp[m.owner].copy()
        for nm, fids in m.boundary_patches.items():
            if self.bc_p.get(nm, {"type": "zero_gradient"})["type"] == "dirichlet":
                fb[fids] = 0.0
        return fb

    def pressure_correction(self, mf):
        m = self.mesh
        A, b, dP = self.pressure_system(mf)
        x0 = np.zeros(m.n_cells) if self.solver != "direct" else None
        pp, its = self._solve(A, b, x0, self.precond_p)
        self.iters_log.append(("p", its))
        if np.any(np.isnan(pp)):
            pp = np.zeros(m.n_cells)
        g = fvm.green_gauss_gradient(m, pp, self.pp_face_values(pp))
        self.U -= dP[:, None] * g
        self.p += self.alpha_p * pp
        self.last_pp = pp
        return float(np.linalg.norm(pp) / max(np.linalg.norm(self.p) + 1e-10, 1e-10))

    # ---- solve_steady :70-101 ----
    def iterate(self):
        ndim = self.mesh.ndim
        mf = self.face_mass_flux()
        res_mom = [self.momentum_eq(c, mf) for c in range(ndim)]
        mf = self.face_mass_flux()
        res_p = self.pressure_correction(mf)
        return max(max(res_mom), res_p)

    def solve_steady(self):
        self.residuals = []
        res0 = None
        n, ndim = self.mesh.n_cells, self.mesh.ndim
        self._aP = {c: np.ones(n) for c in range(ndim)}
        for it in range(self.max_outer_iter):
            res = self.iterate()
            if res0 is None and res > 1e-30:
                res0 = res
            rn = res / res0 if res0 and res0 > 1e-30 else res
            self.residuals.append(rn)
            if rn < self.tol:
                return {"converged": True, "iterations": it + 1, "residuals": self.residuals}
        return {"converged": False, "iterations": self.max_outer_iter, "residuals": self.residuals}


def cavity_setup(sim, lid_speed=1.0):
    """Lid-driven cavity boundary conditions: 'lid' moves along x, other patches are
    no-slip walls; pressure zero-gradient everywhere (reference pin on row 0)."""
    ndim = sim.mesh.ndim
    for nm in sim.mesh.boundary_patches:
        v = [lid_speed] + [0.0] * (ndim - 1) if nm == "lid" else [0.0] * ndim
        sim.set_velocity_bc(nm, "dirichlet", v)
        sim.set_pressure_bc(nm, "zero_gradient")
