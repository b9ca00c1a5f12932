"""Oracle: vectorised FP64 restatement of the reference two-fluid model (test infrastructure).

Restates models/two_fluid.py (TwoFluidSolver: _simple_iteration :277-332,
_compute_phase_change_rate :334-360, _solve_coupled_energy :362-393,
_compute_interfacial_ht_coefficients :395-410, _solve_phase_energy :412-518,
_solve_phase_momentum :520-639, _solve_pressure_correction_two_phase :641-725,
_solve_volume_fraction :727-783, _update_zero_gradient_boundaries :224-250) and the
closures of models/closure.py (Schiller-Naumann drag :13-92, Ranz-Marshall :95-115,
Sato bubble-induced viscosity :146-164). Contributions are accumulated in the
reference's order (operator by operator, faces in face-id order, owner before
neighbour) and every linear system is solved with scipy's spsolve like the
reference's method='direct', so on the golden fixtures it reproduces the reference
to rounding. It is the checker for the device two-fluid path, never a product path.
"""
from __future__ import annotations

import numpy as np
from scipy.sparse.linalg import spsolve

from . import fvm


def drag_coefficient_implicit(alpha_g, rho_l, u_g, u_l, d_b, mu_l):
    """models/closure.py:72-92 with schiller_naumann_drag :13-34."""
    u_rel = u_g - u_l
    u_rel_mag = np.sqrt(np.sum(u_rel ** 2, axis=1))
    u_rel_mag = np.maximum(u_rel_mag, 1e-15)
    Re_p = rho_l * u_rel_mag * d_b / mu_l
    Re_p = np.maximum(Re_p, 1e-10)
    C_D = np.where(Re_p < 1000, 24.0 / Re_p * (1.0 + 0.15 * Re_p ** 0.687), 0.44)
    return 0.75 * C_D * alpha_g * rho_l * u_rel_mag / d_b


def sato_bubble_induced_turbulence(alpha_g, rho_l, u_g, u_l, d_b):
    """models/closure.py:146-164 (no floor on |u_rel|)."""
    u_rel = u_g - u_l
    u_rel_mag = np.sqrt(np.sum(u_rel ** 2, axis=1))
    return 0.6 * rho_l * alpha_g * d_b * u_rel_mag


class TwoFluid:
    """Fields and settings as the reference's TwoFluidSolver (models/two_fluid.py:35-95).

    Boundary values are kept per patch like the reference's fields
    (bv[name][patch] arrays, vectors [faces, ndim])."""

    FIELDS = ("alpha_g", "alpha_l", "U_l", "U_g", "p", "T_l", "T_g")

    def __init__(self, mesh):
        self.mesh = m = mesh
        n, nd = m.n_cells, m.ndim
        self.rho_l, self.rho_g = 998.2, 1.225
        self.mu_l, self.mu_g = 1.003e-3, 1.789e-5
        self.cp_l, self.cp_g = 4182.0, 1006.0
        self.k_l, self.k_g = 0.6, 0.0257
        self.d_b = 0.005
        self.g = np.zeros(nd)
        self.g[-1] = -9.81
        self.h_i_coeff, self.a_i_coeff = 1.0, 1.0
        self.T_sat, self.h_fg, self.r_phase_change = 373.15, 2.257e6, 0.1
        self.alpha_T = 0.7
        self.alpha_u, self.alpha_p, self.alpha_alpha = 0.5, 0.3, 0.5
        self.max_outer_iter, self.tol, self.dt = 200, 1e-4, 0.001
        self.solve_energy, self.solve_momentum = False, True
        self.wall_heat_flux = {}
        self.bc = {k: {} for k in ("alpha", "u_l", "u_g", "p", "T_l", "T_g")}
        self.v = {"alpha_g": np.zeros(n), "alpha_l": np.zeros(n), "U_l": np.zeros((n, nd)),
                  "U_g": np.zeros((n, nd)), "p": np.zeros(n), "T_l": np.zeros(n), "T_g": np.zeros(n)}
        self.bv = {}
        for f in self.FIELDS:
            shape = (lambda k: (k, nd)) if f.startswith("U") else (lambda k: (k,))
            self.bv[f] = {nm: np.zeros(shape(len(fids))) for nm, fids in m.boundary_patches.items()}
        self.old = {}
        self._aP = {}
        self._set_uniform("alpha_l", 0.95)
        self._set_uniform("alpha_g", 0.05)
        self._set_uniform("T_l", 300.0)
        self._set_uniform("T_g", 300.0)

    # ---- field helpers (core/fields.py set_uniform / set_boundary) ----
    def _set_uniform(self, f, val):
        self.v[f][:] = val
        for nm in self.bv[f]:
            self.bv[f][nm][:] = val

    def _set_boundary(self, f, patch, val):
        if patch not in self.bv[f]:
            return
        a = np.asarray(val, dtype=np.float64)
        self.bv[f][patch][:] = a

    # ---- set-up (models/two_fluid.py:97-165) ----
    def initialize(self, alpha_g_init=0.05):
        self._set_uniform("alpha_g", alpha_g_init)
        self._set_uniform("alpha_l", 1.0 - alpha_g_init)

    def set_inlet_bc(self, patch, alpha_g, U_l, U_g, T_l=None, T_g=None):
        self._set_boundary("alpha_g", patch, alpha_g)
        self._set_boundary("alpha_l", patch, 1.0 - alpha_g)
        self._set_boundary("U_l", patch, U_l)
        self._set_boundary("U_g", patch, U_g)
        for k in ("alpha", "u_l", "u_g"):
            self.bc[k][patch] = {"type": "dirichlet"}
        self.bc["p"][patch] = {"type": "zero_gradient"}
        if T_l is not None:
            self._set_boundary("T_l", patch, T_l)
            self.bc["T_l"][patch] = {"type": "dirichlet"}
        if T_g is not None:
            self._set_boundary("T_g", patch, T_g)
            self.bc["T_g"][patch] = {"type": "dirichlet"}

    def set_outlet_bc(self, patch, p_val=0.0):
        self._set_boundary("p", patch, p_val)
        self.bc["p"][patch] = {"type": "dirichlet"}
        for k in ("u_l", "u_g", "alpha", "T_l", "T_g"):
            self.bc[k][patch] = {"type": "zero_gradient"}

    def set_wall_bc(self, patch, q_wall=None, T_wall=None):
        self._set_boundary("U_l", patch, np.zeros(self.mesh.ndim))
        self.bc["u_l"][patch] = {"type": "dirichlet"}
        self.bc["u_g"][patch] = {"type": "zero_gradient"}
        self.bc["p"][patch] = {"type": "zero_gradient"}
        self.bc["alpha"][patch] = {"type": "zero_gradient"}
        if q_wall is not None:
            self.wall_heat_flux[patch] = q_wall
            self.bc["T_l"][patch] = {"type": "zero_gradient"}
            self.bc["T_g"][patch] = {"type": "zero_gradient"}
        elif T_wall is not None:
            self._set_boundary("T_l", patch, T_wall)
            self._set_boundary("T_g", patch, T_wall)
            self.bc["T_l"][patch] = {"type": "dirichlet"}
            self.bc["T_g"][patch] = {"type": "dirichlet"}
        else:
            self.bc["T_l"][patch] = {"type": "zero_gradient"}
            self.bc["T_g"][patch] = {"type": "zero_gradient"}

    # ---- time loop (models/two_fluid.py:167-222) ----
    def step(self, dt=None):
        if dt is not None:
            self.dt = dt
        for f in ("alpha_g", "alpha_l", "U_l", "U_g") + (("T_l", "T_g") if self.solve_energy else ()):
            self.old[f] = self.v[f].copy()
        return self._simple_iteration()

    def _update_zero_gradient_boundaries(self):
        m = self.mesh
        pairs = [("u_l", "U_l"), ("u_g", "U_g")]
        if self.solve_energy:
            pairs += [("T_l", "T_l"), ("T_g", "T_g")]
        for bk, f in pairs:
            for nm, bc in self.bc[bk].items():
                if bc["type"] == "zero_gradient" and nm in m.boundary_patches:
                    self.bv[f][nm] = self.v[f][m.owner[m.boundary_patches[nm]]].copy()
        for nm, bc in self.bc["alpha"].items():
            if bc["type"] == "zero_gradient" and nm in m.boundary_patches:
                o = m.owner[m.boundary_patches[nm]]
                self.bv["alpha_g"][nm] = self.v["alpha_g"][o].copy()
                self.bv["alpha_l"][nm] = self.v["alpha_l"][o].copy()

    def _face_b(self, f):
        """Per-face boundary values of field f in face-id layout (internal rows unused)."""
        m = self.mesh
        v = self.v[f]
        out = v[m.owner].copy()
        for nm, fids in m.boundary_patches.items():
            out[fids] = self.bv[f][nm]
        return out

    def _simple_iteration(self):
        m = self.mesh
        max_res = 0.0
        for _ in range(min(self.max_outer_iter, 30)):
            self._update_zero_gradient_boundaries()
            mf_l = fvm.compute_mass_flux(m, self.v["U_l"], self._face_b("U_l"), self.rho_l)
            mf_g = fvm.compute_mass_flux(m, self.v["U_g"], self._face_b("U_g"), self.rho_g)
            res_mom, res_p, res_alpha = [], 0.0, 0.0
            if self.solve_momentum:
                K = drag_coefficient_implicit(self.v["alpha_g"], self.rho_l, self.v["U_g"], self.v["U_l"], self.d_b,
                                              self.mu_l)
                for comp in range(m.ndim):
                    res_mom.append(self._momentum("liquid", comp, mf_l, K))
                for comp in range(m.ndim):
                    res_mom.append(self._momentum("gas", comp, mf_g, K))
                res_p = self._pressure(mf_l, mf_g)
                dot_m = self._phase_change() if self.solve_energy else np.zeros(m.n_cells)
                res_alpha = self._volume_fraction(mf_g, dot_m)
            else:
                dot_m = self._phase_change() if self.solve_energy else np.zeros(m.n_cells)
                if self.solve_energy:
                    res_alpha = self._volume_fraction(mf_g, dot_m)
            res_energy = self._energy(mf_l, mf_g, dot_m) if self.solve_energy else 0.0
            all_res = res_mom + [res_p, res_alpha, res_energy]
            max_res = max(r if np.isfinite(r) else 1e10 for r in all_res)
            if max_res < self.tol:
                break
        return max_res if np.isfinite(max_res) else 1e10

    @staticmethod
    def _residual(s, x):
        A = s.to_sparse()
        return np.linalg.norm(A @ x - s.rhs) / max(np.linalg.norm(s.rhs), 1e-15)

    @staticmethod
    def _floor(s):
        s.diag[s.diag < 1e-20] = 1e-10

    def _bc_dict(self, key, bvals):
        return {nm: bvals[nm] for nm in self.mesh.boundary_patches}, self.bc[key]

    # ---- momentum (models/two_fluid.py:520-639) ----
    def _momentum(self, phase, comp, mf, K):
        m = self.mesh
        n = m.n_cells
        liquid = phase == "liquid"
        U = self.v["U_l" if liquid else "U_g"]
        a = self.v["alpha_l" if liquid else "alpha_g"]
        rho, mu = (self.rho_l, self.mu_l) if liquid else (self.rho_g, self.mu_g)
        U_other = self.v["U_g" if liquid else "U_l"]
        bckey = "u_l" if liquid else "u_g"
        fname = "U_l" if liquid else "U_g"
        s = fvm.System(n)
        phi = U[:, comp].copy()
        gamma = a * mu
        mu_bit = sato_bubble_induced_turbulence(self.v["alpha_g"], self.rho_l, self.v["U_g"], self.v["U_l"], self.d_b)
        if liquid:
            gamma = gamma + a * mu_bit
        fvm.diffusion_operator(m, gamma, s)
        alpha_mf = mf * a[m.owner]
        fvm.convection_operator_upwind(m, alpha_mf, s)
        idx = np.arange(n)
        if fname in self.old:
            coeff = a * rho * m.volume / self.dt
            s.add_entries(idx, idx, coeff)
            s.add_source(idx, coeff * self.old[fname][:, comp])
        # pressure force, faces in id order, owner then neighbour
        internal = m.neighbour >= 0
        o = m.owner
        nb = np.where(internal, m.neighbour, o)
        p = self.v["p"]
        p_f = np.where(internal, 0.5 * (p[o] + p[nb]), p[o])
        force = -a[o] * p_f * m.normal[:, comp] * m.area
        force_nb = -a[nb] * p_f * m.normal[:, comp] * m.area
        src_i = fvm._interleave(o, nb)
        src_v = fvm._interleave(force, -force_nb)
        src_m = fvm._interleave(np.ones(m.n_faces, bool), internal)
        s.add_source(src_i[src_m], src_v[src_m])
        s.add_entries(idx, idx, K * m.volume)
        s.add_source(idx, K * m.volume * U_other[:, comp])
        s.add_source(idx, a * rho * self.g[comp] * m.volume)
        bvals = {nm: self.bv[fname][nm][:, comp] for nm in m.boundary_patches}
        fvm.apply_boundary_conditions(m, bvals, gamma, alpha_mf, s, self.bc[bckey])
        self._floor(s)
        fvm.under_relax(s, phi, self.alpha_u)
        x = spsolve(s.to_sparse().tocsc(), s.rhs)
        if np.any(np.isnan(x)):
            x = U[:, comp].copy()
        U[:, comp] = x
        aP_cur = np.maximum(s.diag.copy(), 1e-20)
        key = "l" if liquid else "g"
        self._aP[key] = aP_cur if (comp == 0 or key not in self._aP) else np.maximum(self._aP[key], aP_cur)
        return self._residual(s, x)

    # ---- pressure correction (models/two_fluid.py:641-725) ----
    def _pressure(self, mf_l, mf_g):
        m = self.mesh
        n = m.n_cells
        al, ag = self.v["alpha_l"], self.v["alpha_g"]
        aPl = self._aP.get("l", np.ones(n))
        aPg = self._aP.get("g", np.ones(n))
        s = fvm.System(n)
        internal = m.neighbour >= 0
        o = m.owner
        nb = np.where(internal, m.neighbour, o)
        d = fvm._norm_rows(m.ccenter[nb] - m.ccenter[o])
        keep_int = internal & ~(d < 1e-30)
        fi = np.nonzero(keep_int)[0]
        oi, ni = o[fi], nb[fi]
        al_f = 0.5 * (al[oi] + al[ni])
        ag_f = 0.5 * (ag[oi] + ag[ni])
        aPl_f = 0.5 * (aPl[oi] + aPl[ni])
        aPg_f = 0.5 * (aPg[oi] + aPg[ni])
        vol_f = 0.5 * (m.volume[oi] + m.volume[ni])
        cl = self.rho_l * al_f * vol_f / np.maximum(aPl_f, 1e-30)
        cg = self.rho_g * ag_f * vol_f / np.maximum(aPg_f, 1e-30)
        coeff = (cl + cg) * m.area[fi] / d[fi]
        s.add_entries(fvm._interleave(oi, ni, oi, ni), fvm._interleave(oi, ni, ni, oi),
                      fvm._interleave(coeff, coeff, -coeff, -coeff))
        total = mf_l * al[o] + mf_g * ag[o]
        take = keep_int | ~internal  # degenerate internal faces are skipped entirely
        src_i = fvm._interleave(o, nb)
        src_v = fvm._interleave(-total, total)
        src_m = fvm._interleave(take, keep_int)
        s.add_source(src_i[src_m], src_v[src_m])
        s.add_entries(np.array([0]), np.array([0]), np.array([1e10]))
        pp = spsolve(s.to_sparse().tocsc(), s.rhs)
        if np.any(np.isnan(pp)):
            pp = np.zeros_like(pp)
        self.v["p"] = self.v["p"] + self.alpha_p * pp
        nd = m.ndim
        grad = np.zeros((n, nd))
        it = np.nonzero(internal)[0]
        dp = pp[m.neighbour[it]] - pp[m.owner[it]]
        flux = dp[:, None] * m.normal[it, :nd] * m.area[it][:, None]
        gi = fvm._interleave(m.owner[it], m.neighbour[it])
        gv = np.stack([flux, -flux], axis=1).reshape(-1, nd)
        np.add.at(grad, gi, gv)
        ok = m.volume > 1e-30
        grad[ok] = grad[ok] / m.volume[ok][:, None]
        V = m.volume[:, None]
        corr_l = -al[:, None] * V / np.maximum(aPl, 1e-20)[:, None] * grad
        corr_g = -ag[:, None] * V / np.maximum(aPg, 1e-20)[:, None] * grad
        self.v["U_l"] = self.v["U_l"] + self.alpha_p * corr_l
        self.v["U_g"] = self.v["U_g"] + self.alpha_p * corr_g
        return float(np.linalg.norm(pp) / max(np.linalg.norm(self.v["p"]), 1e-15))

    # ---- volume fraction (models/two_fluid.py:727-783) ----
    def _volume_fraction(self, mf_g, dot_m):
        m = self.mesh
        n = m.n_cells
        s = fvm.System(n)
        gamma0 = np.full(n, 1e-6)
        fvm.convection_operator_upwind(m, mf_g, s)
        if "alpha_g" in self.old:
            fvm.temporal_operator(m, self.rho_g, self.dt, self.old["alpha_g"], s)
        idx = np.nonzero(np.abs(dot_m) > 1e-30)[0]
        s.add_source(idx, dot_m[idx] / self.rho_g * m.volume[idx])
        fvm.apply_boundary_conditions(m, self.bv["alpha_g"], gamma0, mf_g, s, self.bc["alpha"])
        self._floor(s)
        fvm.under_relax(s, self.v["alpha_g"], self.alpha_alpha)
        old = self.v["alpha_g"].copy()
        x = spsolve(s.to_sparse().tocsc(), s.rhs)
        if np.any(np.isnan(x)):
            x = old
        x = np.clip(x, 0.0, 1.0)
        self.v["alpha_g"] = x
        self.v["alpha_l"] = 1.0 - x
        ref = self.old.get("alpha_g", x)
        return float(np.max(np.abs(x - ref)))

    # ---- phase change and energy (models/two_fluid.py:334-518) ----
    def _phase_change(self):
        Tl, Tg = self.v["T_l"], self.v["T_g"]
        al, ag = self.v["alpha_l"], self.v["alpha_g"]
        r = self.r_phase_change
        ev = (Tl > self.T_sat) & (al > 1e-6)
        co = (Tg < self.T_sat) & (ag > 1e-6)
        dot_m = np.zeros(self.mesh.n_cells)
        dot_m = dot_m + np.where(ev, r * al * self.rho_l * (Tl - self.T_sat) / self.T_sat, 0.0)
        dot_m = dot_m - np.where(co, r * ag * self.rho_g * (self.T_sat - Tg) / self.T_sat, 0.0)
        return dot_m

    def _interfacial(self):
        u_rel = self.v["U_g"] - self.v["U_l"]
        u_rel_mag = np.sqrt(np.sum(u_rel ** 2, axis=1))
        u_rel_mag = np.maximum(u_rel_mag, 1e-15)
        Re_p = self.rho_l * u_rel_mag * self.d_b / self.mu_l
        Pr = self.mu_l * self.cp_l / self.k_l
        Nu = 2.0 + 0.6 * np.maximum(Re_p, 1e-10) ** 0.5 * Pr ** 0.333
        h_i = self.h_i_coeff * Nu * self.k_l / self.d_b
        a_i = self.a_i_coeff * 6.0 * self.v["alpha_g"] / np.maximum(self.d_b, 1e-15)
        return h_i, a_i

    def _energy(self, mf_l, mf_g, dot_m):
        h_i, a_i = self._interfacial()
        r_l = self._phase_energy("liquid", mf_l, h_i, a_i, dot_m)
        r_g = self._phase_energy("gas", mf_g, h_i, a_i, -dot_m)
        return max(r_l, r_g)

    def _phase_energy(self, phase, mf, h_i, a_i, dot_m):
        m = self.mesh
        n = m.n_cells
        liquid = phase == "liquid"
        a = self.v["alpha_l" if liquid else "alpha_g"]
        rho, cp, kc = (self.rho_l, self.cp_l, self.k_l) if liquid else (self.rho_g, self.cp_g, self.k_g)
        fT, fo = ("T_l", "T_g") if liquid else ("T_g", "T_l")
        s = fvm.System(n)
        gamma = a * kc
        fvm.diffusion_operator(m, gamma, s)
        internal = m.neighbour >= 0
        o = m.owner
        nb = np.where(internal, m.neighbour, o)
        a_face = np.where(internal & (mf < 0), a[nb], a[o])
        acm = mf * a_face * cp
        fvm.convection_operator_upwind(m, acm, s)
        idx = np.arange(n)
        if fT in self.old:
            coeff = a * rho * cp * m.volume / self.dt
            s.add_entries(idx, idx, coeff)
            s.add_source(idx, coeff * self.old[fT])
        hiai = h_i * a_i * m.volume
        s.add_source(idx, hiai * self.v[fo])
        s.add_entries(idx, idx, hiai)
        s.add_source(idx, -dot_m * self.h_fg * m.volume)
        for nm, q in self.wall_heat_flux.items():
            if nm in m.boundary_patches:
                fids = m.boundary_patches[nm]
                ow = m.owner[fids]
                w = self.v["alpha_l"][ow] if liquid else self.v["alpha_g"][ow]
                s.add_source(ow, q * m.area[fids] * w)
        fvm.apply_boundary_conditions(m, self.bv[fT], gamma, acm, s, self.bc[fT])
        self._floor(s)
        fvm.under_relax(s, self.v[fT], self.alpha_T)
        old = self.v[fT].copy()
        x = spsolve(s.to_sparse().tocsc(), s.rhs)
        if np.any(np.isnan(x)) or np.any(np.isinf(x)):
            x = old
        else:
            x = np.clip(x, 200.0, 800.0)
        self.v[fT] = x
        return self._residual(s, x)
