"""Two-fluid (Euler-Euler) solver on the device: the drop-in for models/two_fluid.py.

Public API as the reference's TwoFluidSolver (models/two_fluid.py:22-222): the
constructor takes a mesh; properties (rho_l, rho_g, mu_l, mu_g, cp_l, cp_g, k_l, k_g,
d_b, g, h_i_coeff, a_i_coeff, T_sat, h_fg, r_phase_change, alpha_T), relaxation
(alpha_u, alpha_p, alpha_alpha), max_outer_iter, tol, dt, solve_energy,
solve_momentum; initialize, set_inlet_bc, set_outlet_bc, set_wall_bc and
solve_transient; fields alpha_g, alpha_l, U_l, U_g, p, T_l, T_g whose .values are
host numpy arrays (copied from / to the device on access) with set_uniform /
set_boundary / min / max like core/fields.py.

One SIMPLE inner iteration (models/two_fluid.py:277-332) runs on the device:
zero-gradient boundary refresh, both mass fluxes, implicit drag, the liquid momentum
components one by one (Sato's viscosity is re-evaluated after each, as in the
reference), the gas components together (one matrix, ndim right-hand sides),
the two-phase pressure correction, the Lee phase-change rate, the gas volume
fraction and the two phase energy equations. Each system is assembled with the
generic FVM operators (operators.cu) and the two-fluid terms (two_fluid.cu) and
solved with the device BiCGSTAB + ILU(0) to a 1e-12 relative residual in place of
the reference's spsolve (method='direct'). The residuals of one inner iteration come
back to the host in one small copy for the reference's tolerance test.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _lib
from .device_mesh import BC_TYPES, DeviceMesh
from .mesh import Mesh, from_fvmesh
from .solver import DeviceCSR, Solver

DIRECT_RTOL = 1e-12


class _Field:
    """Device field with the reference field interface (core/fields.py)."""

    def __init__(self, owner, name, ncomp):
        # weak: the solver holds its fields (a strong reference would be a cycle)
        self._ref, self._name, self.ncomp = weakref.ref(owner), name, ncomp

    @property
    def _o(self):
        o = self._ref()
        if o is None:
            raise ReferenceError("the solver of this field no longer exists")
        return o

    @property
    def _t(self):
        return self._o._f[self._name]

    @property
    def values(self):
        return self._t.detach().cpu().numpy().copy()

    @values.setter
    def values(self, v):
        torch = _lib.require_cuda()
        t = self._t
        t.copy_(torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64).reshape(t.shape)))

    @property
    def old_values(self):
        t = self._o._old.get(self._name)
        return None if t is None else t.detach().cpu().numpy().copy()

    def set_uniform(self, value):
        torch = _lib.require_cuda()
        v = torch.as_tensor(np.asarray(value, dtype=np.float64), device=self._t.device)
        self._t[:] = v
        self._o._bv[self._name][:] = v

    def set_boundary(self, patch, value):
        slots = self._o.dm.patch_slots.get(patch)
        if slots is None:
            return
        torch = _lib.require_cuda()
        b = self._o._bv[self._name]
        idx = torch.from_numpy(np.asarray(slots, dtype=np.int64)).to(b.device)
        b[idx] = torch.as_tensor(np.asarray(value, dtype=np.float64), device=b.device)

    def boundary_values(self, patch):
        slots = self._o.dm.patch_slots[patch]
        return self._o._bv[self._name].detach().cpu().numpy()[slots]

    def min(self):
        return float(self._t.min())

    def max(self):
        return float(self._t.max())


class TwoFluidSolver:
    """p_precond: the pressure correction's preconditioner, 'ilu0' (as every other system)
    or 'amg' (the device multigrid, on the graph engine). precision 'mixed': the ILU(0)
    systems (momentum, volume fraction, energy, and p' with 'ilu0') run BiCGSTAB with
    FP32 vectors and values and FP64 residuals, iterate and stopping test (the graph
    engine's residual-replacement form on large meshes, FP32 inner iterations with FP64
    refinement on small ones); the multigrid p' keeps an FP64 Krylov iteration over an
    FP32 hierarchy, and an ILU(0) p' on a large mesh stays FP64. Every system still
    stops on its FP64 relative residual."""

    def __init__(self, mesh, device="cuda", rtol=DIRECT_RTOL, maxiter=20000, p_precond="ilu0", precision="fp64"):
        torch = _lib.require_cuda()
        if not isinstance(mesh, Mesh):
            mesh = from_fvmesh(mesh)
        self.mesh = mesh
        self.dm = dm = DeviceMesh(mesh, device)
        n, nd, Fb = mesh.n_cells, mesh.ndim, dm.n_boundary
        self.ndim = nd
        # properties and settings (models/two_fluid.py:35-95)
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
        self.bc_alpha, self.bc_u_l, self.bc_u_g, self.bc_p, self.bc_T_l, self.bc_T_g = {}, {}, {}, {}, {}, {}
        self.residuals, self.energy_residuals = [], []
        f64 = dict(dtype=torch.float64, device=device)
        self._f = {"alpha_g": torch.zeros(n, **f64), "alpha_l": torch.zeros(n, **f64),
                   "U_l": torch.zeros(n, nd, **f64), "U_g": torch.zeros(n, nd, **f64), "p": torch.zeros(n, **f64),
                   "T_l": torch.zeros(n, **f64), "T_g": torch.zeros(n, **f64)}
        self._bv = {k: torch.zeros((Fb, nd) if k.startswith("U") else (Fb,), **f64) for k in self._f}
        self._old = {}
        for k, nc in (("alpha_g", 1), ("alpha_l", 1), ("U_l", nd), ("U_g", nd), ("p", 1), ("T_l", 1), ("T_g", 1)):
            setattr(self, k, _Field(self, k, nc))
        self.alpha_l.set_uniform(0.95)
        self.alpha_g.set_uniform(0.05)
        self.T_l.set_uniform(300.0)
        self.T_g.set_uniform(300.0)
        # work arrays
        nnz = mesh.nnz
        self._vals = torch.zeros(nnz, **f64)
        self._diag = torch.zeros(n, **f64)
        self._rhs = torch.zeros(n * nd, **f64)
        self._x = torch.zeros(n * nd, **f64)
        self._xold = torch.zeros(n * nd, **f64)
        self._bcomp = torch.zeros(Fb * nd, **f64)
        self._zb = torch.zeros(Fb, **f64)
        self._mf_l = torch.zeros(dm.n_faces, **f64)
        self._mf_g = torch.zeros(dm.n_faces, **f64)
        self._flux = torch.zeros(dm.n_faces, **f64)
        self._gamma = torch.zeros(n, **f64)
        self._gamma0 = torch.full((n,), 1e-6, **f64)
        self._K = torch.zeros(n, **f64)
        self._hiai = torch.zeros(n, **f64)
        self._dot_m = torch.zeros(n, **f64)
        self._aP_l = torch.ones(n, **f64)
        self._aP_g = torch.ones(n, **f64)
        self._grad = torch.zeros(n * nd, **f64)
        self._flag = torch.zeros(1, dtype=torch.int32, device=device)
        self._scratch = torch.zeros(_lib.REDUCE_SCRATCH, **f64)
        # residual slots: [mom liquid (2 each)], [mom gas (2 each)], p (2), alpha (1), energy (2+2)
        self._res = torch.zeros(4 * nd + 2 + 1 + 4 + 2, **f64)
        self._A = DeviceCSR(dm.t["indptr"], dm.t["indices"], self._vals)
        levels = mesh.cell_color
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"unknown precision {precision!r}")
        mode = _lib.MODE_MIXED if precision == "mixed" else _lib.MODE_FP64
        self.precision = precision
        mixed = precision == "mixed"
        # mixed on large meshes: the graph engine's FP32 form for the momentum, volume
        # fraction and energy systems (well conditioned: every one has a time term)
        t1 = 3 if (mixed and n > 40000) else 0
        tg = 3 if (mixed and n * nd > 40000) else 0
        self._s1 = Solver(self._A, precond="ilu0", nrhs=1, rtol=rtol, atol=0.0, maxiter=maxiter, levels=levels,
                          mode=mode, team=t1)
        self._sg = Solver(self._A, precond="ilu0", nrhs=nd, rtol=rtol, atol=0.0, maxiter=maxiter, levels=levels,
                          mode=mode, team=tg)
        if p_precond == "amg":
            self._sp = Solver(self._A, precond="amg", nrhs=1, rtol=rtol, atol=0.0, maxiter=maxiter, mode=mode)
        elif p_precond == "ilu0":
            # the pinned p' (diag[0] += 1e10) is not well conditioned: in the mixed form
            # it keeps the FP64 Krylov iteration on large meshes
            self._sp = self._s1 if not t1 else Solver(self._A, precond="ilu0", nrhs=1, rtol=rtol, atol=0.0,
                                                      maxiter=maxiter, levels=levels)
        else:
            raise ValueError(f"unknown p' preconditioner {p_precond!r}")
        self._params = _lib.TfParams()
        # Krylov iterations since the last reset of the one-rhs ILU(0) solves, the
        # ndim-rhs solves and the multigrid p' solves (device counters, read by the
        # caller when it wants them)
        self.krylov = torch.zeros(3, dtype=torch.int64, device=device)

    # ---- set-up (models/two_fluid.py:97-165) ----
    def initialize(self, alpha_g_init=0.05):
        self.alpha_g.set_uniform(alpha_g_init)
        self.alpha_l.set_uniform(1.0 - alpha_g_init)

    def set_inlet_bc(self, patch, alpha_g, U_l, U_g, T_l=None, T_g=None):
        self.alpha_g.set_boundary(patch, alpha_g)
        self.alpha_l.set_boundary(patch, 1.0 - alpha_g)
        self.U_l.set_boundary(patch, U_l)
        self.U_g.set_boundary(patch, U_g)
        self.bc_alpha[patch] = {"type": "dirichlet"}
        self.bc_u_l[patch] = {"type": "dirichlet"}
        self.bc_u_g[patch] = {"type": "dirichlet"}
        self.bc_p[patch] = {"type": "zero_gradient"}
        if T_l is not None:
            self.T_l.set_boundary(patch, T_l)
            self.bc_T_l[patch] = {"type": "dirichlet"}
        if T_g is not None:
            self.T_g.set_boundary(patch, T_g)
            self.bc_T_g[patch] = {"type": "dirichlet"}

    def set_outlet_bc(self, patch, p_val=0.0):
        self.p.set_boundary(patch, p_val)
        self.bc_p[patch] = {"type": "dirichlet"}
        for d in (self.bc_u_l, self.bc_u_g, self.bc_alpha, self.bc_T_l, self.bc_T_g):
            d[patch] = {"type": "zero_gradient"}

    def set_wall_bc(self, patch, q_wall=None, T_wall=None):
        self.U_l.set_boundary(patch, np.zeros(self.ndim))
        self.bc_u_l[patch] = {"type": "dirichlet"}
        self.bc_u_g[patch] = {"type": "zero_gradient"}
        self.bc_p[patch] = {"type": "zero_gradient"}
        self.bc_alpha[patch] = {"type": "zero_gradient"}
        if q_wall is not None:
            self.wall_heat_flux[patch] = q_wall
            self.bc_T_l[patch] = {"type": "zero_gradient"}
            self.bc_T_g[patch] = {"type": "zero_gradient"}
        elif T_wall is not None:
            self.T_l.set_boundary(patch, T_wall)
            self.T_g.set_boundary(patch, T_wall)
            self.bc_T_l[patch] = {"type": "dirichlet"}
            self.bc_T_g[patch] = {"type": "dirichlet"}
        else:
            self.bc_T_l[patch] = {"type": "zero_gradient"}
            self.bc_T_g[patch] = {"type": "zero_gradient"}

    # ---- boundary arrays from the bc dicts ----
    def _bc_arrays(self):
        torch = _lib.require_cuda()
        dev = self._vals.device
        Fb = self.dm.n_boundary
        out = {}
        for key, d in (("alpha", self.bc_alpha), ("u_l", self.bc_u_l), ("u_g", self.bc_u_g), ("T_l", self.bc_T_l),
                       ("T_g", self.bc_T_g)):
            bt = np.zeros(Fb, np.int8)
            zg = np.zeros(Fb, np.int8)
            for nm, slots in self.dm.patch_slots.items():
                t = d.get(nm, {"type": "zero_gradient"})["type"]
                bt[slots] = BC_TYPES.get(t, -1)
                if nm in d and t == "zero_gradient":
                    zg[slots] = 1
            out[key] = (torch.from_numpy(bt).to(dev), torch.from_numpy(zg).to(dev))
        qm = np.zeros(Fb, np.int8)
        qb = np.zeros(Fb)
        for nm, q in self.wall_heat_flux.items():
            if nm in self.dm.patch_slots:
                qm[self.dm.patch_slots[nm]] = 1
                qb[self.dm.patch_slots[nm]] = float(q)
        out["q"] = (torch.from_numpy(qm).to(dev), torch.from_numpy(qb).to(dev))
        return out

    def _sync_params(self):
        P = self._params
        for k in ("rho_l", "rho_g", "mu_l", "mu_g", "cp_l", "cp_g", "k_l", "k_g", "d_b", "h_i_coeff", "a_i_coeff",
                  "T_sat", "h_fg", "r_phase_change", "dt"):
            setattr(P, k, float(getattr(self, k)))
        g = np.zeros(3)
        g[: self.ndim] = np.asarray(self.g, dtype=np.float64)[: self.ndim]
        for i in range(3):
            P.g[i] = float(g[i])

    # ---- time loop (models/two_fluid.py:167-222) ----
    def solve_transient(self, t_end, dt=None, report_interval=100, adaptive_dt=False, cfl_target=0.5,
                        dt_min=1e-8, dt_max=None, monitor=None):
        """models/two_fluid.py:167-258. With adaptive_dt the step after each SIMPLE
        solve comes from AdaptiveTimeControl on the liquid velocity (brought to the
        host once per step) and nu_l = mu_l / rho_l, shrinking when the step's residual
        is not below 10 tol; as in the reference, time advances by the new step."""
        if dt is not None:
            self.dt = dt
        ctrl = None
        if adaptive_dt:
            from .time_control import AdaptiveTimeControl
            ctrl = AdaptiveTimeControl(dt_init=self.dt, dt_min=dt_min, dt_max=dt_max if dt_max is not None else t_end,
                                       cfl_target=cfl_target)
        t, step = 0.0, 0
        self.residuals = []
        dt_history, cfl_history = [], []
        while t < t_end - 1e-15:
            max_res = self.step()
            if ctrl is not None:
                new_dt, info = ctrl.compute_dt(self.mesh, self.U_l.values, self.mu_l / self.rho_l,
                                               converged=(max_res < 10 * self.tol))
                self.dt = new_dt
                dt_history.append(new_dt)
                cfl_history.append(info["cfl_max"])
            t += self.dt
            step += 1
            self.residuals.append(max_res)
            if monitor is not None:
                monitor.update(step, t, max_res, dt=self.dt)
            if step % report_interval == 0:
                print(f"  Step {step}, t={t:.4f}, residual={max_res:.2e}, "
                      f"alpha_g: [{self.alpha_g.min():.4f}, {self.alpha_g.max():.4f}]")
        return {"time_steps": step, "final_time": t, "residuals": self.residuals, "dt_history": dt_history,
                "cfl_history": cfl_history}

    def step(self):
        """One time step: store the old fields, then the SIMPLE inner iterations."""
        names = ["alpha_g", "alpha_l", "U_l", "U_g"] + (["T_l", "T_g"] if self.solve_energy else [])
        for k in names:
            if k in self._old:
                self._old[k].copy_(self._f[k])
            else:
                self._old[k] = self._f[k].clone()
        return self._simple_iteration()

    # ---- helpers ----
    def _L(self):
        return _lib.lib()

    def _reset(self):
        self._vals.zero_()
        self._diag.zero_()
        self._rhs.zero_()

    def _solve(self, solver, x, rhs):
        solver.setup(self._A)
        solver.solve(self._A, rhs, x)
        k = 1 if solver is self._sg else (2 if (solver is self._sp and solver.precond == "amg") else 0)
        self.krylov[k] += solver.iters.max().to(self.krylov.dtype)

    def _simple_iteration(self):
        self._sync_params()
        bca = self._bc_arrays()
        n, nd = self.mesh.n_cells, self.ndim
        L, chk, P, st = self._L(), _lib.check, _lib.ptr, _lib.stream_handle()
        dmd = C.byref(self.dm.desc)
        prm = C.byref(self._params)
        f = self._f
        max_res = 0.0
        for _ in range(min(self.max_outer_iter, 30)):
            # zero-gradient boundary values := owner values
            zg = [("u_l", "U_l", nd), ("u_g", "U_g", nd)]
            if self.solve_energy:
                zg += [("T_l", "T_l", 1), ("T_g", "T_g", 1)]
            zg += [("alpha", "alpha_g", 1), ("alpha", "alpha_l", 1)]
            for key, fld, nc in zg:
                chk(L.kcfd_tf_zero_gradient(dmd, P(bca[key][1]), P(f[fld]), nc, P(self._bv[fld]), st), "zero_gradient")
            chk(L.kcfd_tf_mass_flux(dmd, self.rho_l, P(f["U_l"]), P(self._bv["U_l"]), P(self._mf_l), st), "mass_flux")
            chk(L.kcfd_tf_mass_flux(dmd, self.rho_g, P(f["U_g"]), P(self._bv["U_g"]), P(self._mf_g), st), "mass_flux")
            self._res.zero_()
            if self.solve_momentum:
                chk(L.kcfd_tf_drag(dmd, prm, P(f["alpha_g"]), P(f["U_g"]), P(f["U_l"]), P(self._K), st), "drag")
                for comp in range(nd):
                    self._momentum_liquid(comp, bca)
                self._momentum_gas(bca)
                self._pressure()
                if self.solve_energy:
                    chk(L.kcfd_tf_phase_change(dmd, prm, P(f["alpha_l"]), P(f["alpha_g"]), P(f["T_l"]), P(f["T_g"]),
                                               P(self._dot_m), st), "phase_change")
                else:
                    self._dot_m.zero_()
                self._volume_fraction(bca)
            else:
                if self.solve_energy:
                    chk(L.kcfd_tf_phase_change(dmd, prm, P(f["alpha_l"]), P(f["alpha_g"]), P(f["T_l"]), P(f["T_g"]),
                                               P(self._dot_m), st), "phase_change")
                    self._volume_fraction(bca)
                else:
                    self._dot_m.zero_()
            if self.solve_energy:
                chk(L.kcfd_tf_interfacial(dmd, prm, P(f["alpha_g"]), P(f["U_g"]), P(f["U_l"]), P(self._hiai), st),
                    "interfacial")
                self._energy("liquid", bca)
                self._energy("gas", bca)
            max_res = self._residual_max()
            if max_res < self.tol:
                break
        return max_res if np.isfinite(max_res) else 1e10

    def _residual_max(self):
        r = self._res.cpu().numpy()
        nd = self.ndim
        out = []
        k = 0
        if self.solve_momentum:
            for _ in range(2 * nd):
                out.append(np.sqrt(r[k]) / max(np.sqrt(r[k + 1]), 1e-15))
                k += 2
            out.append(np.sqrt(r[k]) / max(np.sqrt(r[k + 1]), 1e-15))  # p: ||p'|| / ||p||
        k = 4 * nd + 2
        res_alpha = r[k] if (self.solve_momentum or self.solve_energy) else 0.0
        if not self.solve_momentum:
            out.append(0.0)
        out.append(res_alpha)
        if self.solve_energy:
            el = np.sqrt(r[k + 1]) / max(np.sqrt(r[k + 2]), 1e-15)
            eg = np.sqrt(r[k + 3]) / max(np.sqrt(r[k + 4]), 1e-15)
            e = max(el, eg)
            self.energy_residuals.append(e)
            out.append(e)
        else:
            out.append(0.0)
        return max(v if np.isfinite(v) else 1e10 for v in out)

    # ---- momentum (models/two_fluid.py:520-639) ----
    def _momentum_liquid(self, comp, bca):
        L, chk, P, st = self._L(), _lib.check, _lib.ptr, _lib.stream_handle()
        dmd, prm, f = C.byref(self.dm.desc), C.byref(self._params), self._f
        n, nd, Fb = self.mesh.n_cells, self.ndim, self.dm.n_boundary
        self._reset()
        chk(L.kcfd_tf_gamma(dmd, prm, 1, P(f["alpha_l"]), self.mu_l, P(f["alpha_g"]), P(f["U_g"]), P(f["U_l"]),
                            P(self._gamma), st), "gamma")
        chk(L.kcfd_op_diffusion(dmd, P(self._gamma), P(self._vals), P(self._diag), st), "diffusion")
        chk(L.kcfd_tf_face_flux(dmd, 0, P(self._mf_l), P(f["alpha_l"]), 1.0, P(self._flux), st), "face_flux")
        chk(L.kcfd_op_convection_upwind(dmd, P(self._flux), P(self._vals), P(self._diag), st), "convection")
        old = self._old.get("U_l")
        chk(L.kcfd_tf_momentum_sources(dmd, prm, comp, 1, self.rho_l, P(f["alpha_l"]), P(f["p"]), P(self._K),
                                       P(f["U_g"]), P(old) if old is not None else None, P(self._vals),
                                       P(self._diag), P(self._rhs), st), "momentum_sources")
        x = self._x[:n]
        chk(L.kcfd_tf_copy(n, 1, P(f["U_l"]), nd, comp, P(x), 1, 0, st), "copy")
        chk(L.kcfd_tf_copy(Fb, 1, P(self._bv["U_l"]), nd, comp, P(self._bcomp), 1, 0, st), "copy")
        chk(L.kcfd_tf_boundary(dmd, P(bca["u_l"][0]), P(self._bcomp), P(self._zb), 1, P(self._gamma), P(self._flux),
                               P(self._vals), P(self._diag), P(self._rhs), st), "boundary")
        chk(L.kcfd_tf_relax(dmd, self.alpha_u, P(x), 1, 1, P(self._vals), P(self._diag), P(self._rhs), st), "relax")
        xo = self._xold[:n]
        xo.copy_(x)
        rhs = self._rhs[:n]
        self._solve(self._s1, x, rhs)
        chk(L.kcfd_tf_guard(n, P(x), P(xo), 0, 0.0, 0.0, P(self._flag), st), "guard")
        chk(L.kcfd_tf_copy(n, 1, P(x), 1, 0, P(f["U_l"]), nd, comp, st), "copy")
        chk(L.kcfd_tf_update_ap(dmd, P(self._diag), P(self._aP_l), 1 if comp == 0 else 0, st), "update_ap")
        chk(L.kcfd_residual_norms(C.byref(self._A.desc()), P(x), P(rhs), 1, P(self._res[2 * comp:]), P(self._scratch),
                                  st), "residual_norms")

    def _momentum_gas(self, bca):
        L, chk, P, st = self._L(), _lib.check, _lib.ptr, _lib.stream_handle()
        dmd, prm, f = C.byref(self.dm.desc), C.byref(self._params), self._f
        n, nd = self.mesh.n_cells, self.ndim
        self._reset()
        chk(L.kcfd_tf_gamma(dmd, prm, 0, P(f["alpha_g"]), self.mu_g, None, None, None, P(self._gamma), st), "gamma")
        chk(L.kcfd_op_diffusion(dmd, P(self._gamma), P(self._vals), P(self._diag), st), "diffusion")
        chk(L.kcfd_tf_face_flux(dmd, 0, P(self._mf_g), P(f["alpha_g"]), 1.0, P(self._flux), st), "face_flux")
        chk(L.kcfd_op_convection_upwind(dmd, P(self._flux), P(self._vals), P(self._diag), st), "convection")
        old = self._old.get("U_g")
        chk(L.kcfd_tf_momentum_sources(dmd, prm, 0, nd, self.rho_g, P(f["alpha_g"]), P(f["p"]), P(self._K),
                                       P(f["U_l"]), P(old) if old is not None else None, P(self._vals),
                                       P(self._diag), P(self._rhs), st), "momentum_sources")
        x = self._x[: n * nd]
        x.copy_(f["U_g"].reshape(-1))
        chk(L.kcfd_tf_boundary(dmd, P(bca["u_g"][0]), P(self._bv["U_g"]), P(self._zb), nd, P(self._gamma),
                               P(self._flux), P(self._vals), P(self._diag), P(self._rhs), st), "boundary")
        chk(L.kcfd_tf_relax(dmd, self.alpha_u, P(x), nd, 1, P(self._vals), P(self._diag), P(self._rhs), st), "relax")
        xo = self._xold[: n * nd]
        xo.copy_(x)
        rhs = self._rhs[: n * nd]
        self._solve(self._sg, x, rhs)
        chk(L.kcfd_tf_guard(n * nd, P(x), P(xo), 0, 0.0, 0.0, P(self._flag), st), "guard")
        f["U_g"].reshape(-1).copy_(x)
        chk(L.kcfd_tf_update_ap(dmd, P(self._diag), P(self._aP_g), 1, st), "update_ap")
        chk(L.kcfd_residual_norms(C.byref(self._A.desc()), P(x), P(rhs), nd, P(self._res[2 * nd:]), P(self._scratch),
                                  st), "residual_norms")

    # ---- two-phase pressure correction (models/two_fluid.py:641-725) ----
    def _pressure(self):
        L, chk, P, st = self._L(), _lib.check, _lib.ptr, _lib.stream_handle()
        dmd, prm, f = C.byref(self.dm.desc), C.byref(self._params), self._f
        n, nd = self.mesh.n_cells, self.ndim
        self._reset()
        chk(L.kcfd_tf_pressure_assemble(dmd, prm, P(f["alpha_l"]), P(f["alpha_g"]), P(self._aP_l), P(self._aP_g),
                                        P(self._mf_l), P(self._mf_g), P(self._vals), P(self._diag), P(self._rhs), st),
            "pressure_assemble")
        pp = self._x[:n]
        pp.zero_()
        self._solve(self._sp, pp, self._rhs[:n])
        chk(L.kcfd_tf_guard(n, P(pp), None, 2, 0.0, 0.0, P(self._flag), st), "guard")
        chk(L.kcfd_tf_correct(dmd, self.alpha_p, P(pp), P(f["alpha_l"]), P(f["alpha_g"]), P(self._aP_l),
                              P(self._aP_g), P(self._grad), P(f["U_l"]), P(f["U_g"]), P(f["p"]), st), "correct")
        k = 4 * nd
        chk(L.kcfd_vec_norms2(n, 1, P(pp), P(self._res[k:]), P(self._scratch), st), "norms")
        chk(L.kcfd_vec_norms2(n, 1, P(f["p"]), P(self._res[k + 1:]), P(self._scratch), st), "norms")

    # ---- volume fraction (models/two_fluid.py:727-783) ----
    def _volume_fraction(self, bca):
        L, chk, P, st = self._L(), _lib.check, _lib.ptr, _lib.stream_handle()
        dmd, f = C.byref(self.dm.desc), self._f
        n, nd = self.mesh.n_cells, self.ndim
        self._reset()
        chk(L.kcfd_op_convection_upwind(dmd, P(self._mf_g), P(self._vals), P(self._diag), st), "convection")
        old = self._old.get("alpha_g")
        if old is not None:
            chk(L.kcfd_op_cells(dmd, 0, self.rho_g, self.dt, P(old), None, P(self._vals), P(self._diag),
                                P(self._rhs), st), "temporal")
        chk(L.kcfd_tf_alpha_source(dmd, self.rho_g, P(self._dot_m), P(self._rhs), st), "alpha_source")
        chk(L.kcfd_op_boundary(dmd, P(bca["alpha"][0]), P(self._bv["alpha_g"]), P(self._zb), P(self._gamma0),
                               P(self._mf_g), P(self._vals), P(self._diag), P(self._rhs), st), "boundary")
        ag = f["alpha_g"]
        chk(L.kcfd_tf_relax(dmd, self.alpha_alpha, P(ag), 1, 1, P(self._vals), P(self._diag), P(self._rhs), st),
            "relax")
        xo = self._xold[:n]
        xo.copy_(ag)
        self._solve(self._s1, ag, self._rhs[:n])
        chk(L.kcfd_tf_guard(n, P(ag), P(xo), 0, 0.0, 0.0, P(self._flag), st), "guard")
        ref = old if old is not None else xo
        chk(L.kcfd_tf_alpha_finish(n, P(ag), P(f["alpha_l"]), P(ref), P(self._res[4 * nd + 2:]), st), "alpha_finish")
        if old is None:
            # the reference compares with the new values when no old values exist
            chk(L.kcfd_tf_alpha_finish(n, P(ag), P(f["alpha_l"]), P(ag), P(self._res[4 * nd + 2:]), st),
                "alpha_finish")

    # ---- phase energy (models/two_fluid.py:412-518) ----
    def _energy(self, phase, bca):
        L, chk, P, st = self._L(), _lib.check, _lib.ptr, _lib.stream_handle()
        dmd, prm, f = C.byref(self.dm.desc), C.byref(self._params), self._f
        n, nd = self.mesh.n_cells, self.ndim
        liquid = phase == "liquid"
        a = f["alpha_l" if liquid else "alpha_g"]
        rho, cp, kc = (self.rho_l, self.cp_l, self.k_l) if liquid else (self.rho_g, self.cp_g, self.k_g)
        fT, fo = ("T_l", "T_g") if liquid else ("T_g", "T_l")
        mf = self._mf_l if liquid else self._mf_g
        self._reset()
        chk(L.kcfd_tf_gamma(dmd, prm, 0, P(a), kc, None, None, None, P(self._gamma), st), "gamma")
        chk(L.kcfd_op_diffusion(dmd, P(self._gamma), P(self._vals), P(self._diag), st), "diffusion")
        chk(L.kcfd_tf_face_flux(dmd, 1, P(mf), P(a), cp, P(self._flux), st), "face_flux")
        chk(L.kcfd_op_convection_upwind(dmd, P(self._flux), P(self._vals), P(self._diag), st), "convection")
        old = self._old.get(fT)
        qm, qb = bca["q"]
        chk(L.kcfd_tf_energy_sources(dmd, prm, rho, cp, P(a), P(old) if old is not None else None, P(f[fo]),
                                     P(self._hiai), P(self._dot_m), 1.0 if liquid else -1.0, P(qm), P(qb), P(a),
                                     P(self._vals), P(self._diag), P(self._rhs), st), "energy_sources")
        chk(L.kcfd_op_boundary(dmd, P(bca[fT][0]), P(self._bv[fT]), P(self._zb), P(self._gamma), P(self._flux),
                               P(self._vals), P(self._diag), P(self._rhs), st), "boundary")
        T = f[fT]
        chk(L.kcfd_tf_relax(dmd, self.alpha_T, P(T), 1, 1, P(self._vals), P(self._diag), P(self._rhs), st), "relax")
        xo = self._xold[:n]
        xo.copy_(T)
        rhs = self._rhs[:n]
        self._solve(self._s1, T, rhs)
        chk(L.kcfd_tf_guard(n, P(T), P(xo), 1, 200.0, 800.0, P(self._flag), st), "guard")
        k = 4 * nd + 3 + (0 if liquid else 2)
        chk(L.kcfd_residual_norms(C.byref(self._A.desc()), P(T), P(rhs), 1, P(self._res[k:]), P(self._scratch), st),
            "residual_norms")
