"""SIMPLE solver on the device: the drop-in for models/single_phase.py SIMPLESolver.

Public API as in the reference (models/single_phase.py:16-121): SIMPLESolver(mesh,
rho, mu), set_velocity_bc, set_pressure_bc, alpha_u, alpha_p, max_outer_iter, tol,
solve_steady() -> {'converged', 'iterations', 'residuals'}, and U / p fields whose
.values are host numpy arrays (copied from / to the device on access).

One outer iteration (models/single_phase.py:77-92) runs entirely on the device:
  mass flux -> [Green-Gauss of U] -> momentum assembly (one matrix, ndim rhs) ->
  one BiCGSTAB+Jacobi launch for all components -> post-solve residual norms ->
  mass flux -> p' assembly -> ILU(0)/Jacobi set-up -> BiCGSTAB launch for p' ->
  Green-Gauss of p' -> velocity/pressure correction -> residual bookkeeping.
No step reads back to the host; with graph=True the iteration is captured once in a
CUDA graph and replayed.

Linear solves: the reference calls spsolve; here BiCGSTAB runs to a relative
residual `rtol` (1e-8 by default) from the current field (momentum) or zero (p').
precision='mixed' keeps FP64 assembly values for the outer residual and an FP32
copy (written by the same kernels) for the inner iterations. On large meshes the
momentum solve runs the graph engine's FP32 form (FP32 vectors and values, FP64
iterate, residual replacement against the FP64 matrix); the p' solve keeps an FP64
Krylov iteration over an FP32 multigrid hierarchy with precond_p='amg'; with ILU(0)
or Jacobi it runs FP32 inner iterations with FP64 refinement up to 4,096 cells and
FP64 above (FP32 inner iterations cannot resolve the pinned p' operator on large
meshes).
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _lib
from .device_mesh import BoundaryConditions, DeviceMesh
from .mesh import Mesh, from_fvmesh
from .solver import DeviceCSR, Solver


class _Field:
    """values: host numpy view of a device tensor (read copies, assignment uploads)."""

    def __init__(self, owner, name):
        # a weak reference: the solver holds its fields, so a strong one would make a
        # cycle that keeps the solver's device memory until the garbage collector runs
        self._ref, self._name = weakref.ref(owner), name

    @property
    def _owner(self):
        o = self._ref()
        if o is None:
            raise ReferenceError("the solver of this field no longer exists")
        return o

    @property
    def values(self):
        return getattr(self._owner, self._name).detach().cpu().numpy().copy()

    @values.setter
    def values(self, v):
        t = getattr(self._owner, self._name)
        torch = _lib.require_cuda()
        t.copy_(torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64).reshape(t.shape)))


class SIMPLESolver:
    def __init__(self, mesh, rho=1.0, mu=1e-3, precision="fp64", precond_p="jacobi", ilu_order="color",
                 rtol=1e-8, maxiter=10000, muscl=None, nonorth=False, graph=False, team=0, lanes=0,
                 inner_rtol=1e-3, inner_maxiter=400, device="cuda"):
        torch = _lib.require_cuda()
        if not isinstance(mesh, Mesh):
            mesh = from_fvmesh(mesh)
        self.mesh = mesh
        self.dm = DeviceMesh(mesh, device)
        self.bcs = BoundaryConditions(self.dm, device)
        self.rho, self.mu = float(rho), float(mu)
        self.alpha_u, self.alpha_p = 0.7, 0.3
        self.max_outer_iter, self.tol = 500, 1e-6
        self.residuals = []
        self.transient, self.dt = False, 0.01
        self.precision = precision
        self.muscl = muscl
        self.nonorth = bool(nonorth)
        self.graph = graph
        n, D, nnz = mesh.n_cells, mesh.ndim, mesh.nnz
        self.ndim = D
        f64 = dict(dtype=torch.float64, device=device)
        self.U_t = torch.zeros(n, D, **f64)
        self.U_old_t = torch.zeros(n, D, **f64)
        self.p_t = torch.zeros(n, **f64)
        self.pp_t = torch.zeros(n, **f64)
        self.mf_t = torch.zeros(mesh.n_faces, **f64)
        self.aP_t = torch.zeros(n, **f64)
        self.dP_t = torch.zeros(n, **f64)
        self.b_m = torch.zeros(n, D, **f64)
        self.b_p = torch.zeros(n, **f64)
        self.gU_t = torch.zeros(n, D, D, **f64) if (muscl or nonorth) else None
        self.gpp_t = torch.zeros(n, D, **f64)
        self.mom_norms = torch.zeros(2 * D, **f64)
        self.p_norms = torch.zeros(2, **f64)
        self.scratch = torch.zeros(_lib.REDUCE_SCRATCH, **f64)
        self.state = torch.zeros(2, **f64)
        self.it_dev = torch.zeros(1, dtype=torch.int32, device=device)
        self.hist_cap = 1 << 16
        self.hist = torch.zeros(self.hist_cap, **f64)
        self.chist = torch.zeros(self.hist_cap, **f64)   # ||b_p'|| per outer iteration
        self.bp_norm2 = torch.zeros(1, **f64)
        mixed = precision == "mixed"
        self.mode = _lib.MODE_MIXED if mixed else _lib.MODE_FP64
        ip, ix = self.dm.t["indptr"], self.dm.t["indices"]
        self.A_m = DeviceCSR(ip, ix, torch.zeros(nnz, **f64),
                             torch.zeros(nnz, dtype=torch.float32, device=device) if mixed else None)
        self.A_p = DeviceCSR(ip, ix, torch.zeros(nnz, **f64),
                             torch.zeros(nnz, dtype=torch.float32, device=device) if mixed else None)
        # mixed momentum solves on large meshes: the graph engine's FP32 form (residual
        # replacement against the FP64 matrix; these systems are well conditioned)
        team_m = team if team else (3 if (mixed and n * D > 40000) else 0)
        self.s_m = Solver(self.A_m, precond="jacobi", mode=self.mode, nrhs=D, maxiter=maxiter, rtol=rtol,
                          team=team_m, lanes=lanes, inner_rtol=inner_rtol, inner_maxiter=inner_maxiter)
        levels = None
        if precond_p == "ilu0":
            levels = mesh.cell_color if ilu_order == "color" else mesh.level_natural
        # p' in the mixed form: an FP32 multigrid hierarchy under an FP64 Krylov iteration
        # ('amg'); FP32 inner iterations with FP64 refinement up to 4,096 cells; FP64
        # above, where the FP32 inner iterations cannot resolve the pinned operator
        # (its conditioning grows with the mesh; measured: BREAKDOWN on a 256^2 cavity,
        # and divergence of the engine's FP32 recursion on the 128^3 cavity, with ILU(0)
        # and with Jacobi)
        mode_p = self.mode if (precond_p == "amg" or n <= 4096) else _lib.MODE_FP64
        self.s_p = Solver(self.A_p, precond=precond_p, mode=mode_p, nrhs=1, maxiter=maxiter, rtol=rtol,
                          team=team, lanes=lanes, inner_rtol=inner_rtol, inner_maxiter=inner_maxiter, levels=levels)
        self.U = _Field(self, "U_t")
        self.p = _Field(self, "p_t")
        self._graph = None
        self._params = _lib.MomParams()

    # ---- boundary conditions (models/single_phase.py:55-68) ----
    def set_velocity_bc(self, patch, bc_type, value=None):
        self.bcs.set_velocity(patch, bc_type, value)
        self._graph = None

    def set_pressure_bc(self, patch, bc_type, value=None):
        self.bcs.set_pressure(patch, bc_type, value)
        self._graph = None

    # ---- one outer iteration, all on the device ----
    def _step(self):
        L = _lib.lib()
        chk = _lib.check
        st = _lib.stream_handle()
        dm = C.byref(self.dm.desc)
        bc = C.byref(self.bcs.desc)
        P = _lib.ptr
        prm = self._params
        prm.rho, prm.mu, prm.alpha_u = self.rho, self.mu, self.alpha_u
        prm.dt = self.dt if self.transient else 0.0
        prm.limiter = _lib.LIMITERS[self.muscl]
        prm.nonorth = 1 if self.nonorth else 0
        chk(L.kcfd_mass_flux(dm, bc, P(self.U_t), self.rho, P(self.mf_t), st), "mass_flux")
        if self.gU_t is not None:
            chk(L.kcfd_gg_gradient(dm, self.ndim, P(self.U_t), P(self.bcs.tensor("u_type")),
                                   P(self.bcs.tensor("u_val")), P(self.gU_t), st), "gg_gradient U")
        chk(L.kcfd_momentum_assemble(dm, bc, C.byref(prm), P(self.U_t), P(self.U_old_t), P(self.p_t), P(self.mf_t),
                                     P(self.gU_t), P(self.aP_t), P(self.A_m.vals64), P(self.A_m.vals32),
                                     P(self.b_m), P(self.dP_t), st), "momentum_assemble")
        self.s_m.setup(self.A_m)
        self.s_m.solve(self.A_m, self.b_m, self.U_t)
        am = self.A_m.desc()
        chk(L.kcfd_residual_norms(C.byref(am), P(self.U_t), P(self.b_m), self.ndim, P(self.mom_norms),
                                  P(self.scratch), st), "residual_norms")
        chk(L.kcfd_mass_flux(dm, bc, P(self.U_t), self.rho, P(self.mf_t), st), "mass_flux")
        chk(L.kcfd_pressure_assemble(dm, bc, self.rho, P(self.dP_t), P(self.mf_t), P(self.aP_t),
                                     P(self.A_p.vals64), P(self.A_p.vals32), P(self.b_p), st), "pressure_assemble")
        chk(L.kcfd_vec_norms2(self.dm.n_cells, 1, P(self.b_p), P(self.bp_norm2), P(self.scratch), st),
            "vec_norms2")
        chk(L.kcfd_record_norm(P(self.bp_norm2), P(self.chist), P(self.it_dev), self.hist_cap, st), "record_norm")
        self.s_p.setup(self.A_p)
        self.pp_t.zero_()
        self.s_p.solve(self.A_p, self.b_p, self.pp_t)
        chk(L.kcfd_gg_gradient(dm, 1, P(self.pp_t), P(self.bcs.tensor("pp_type")), P(self.bcs.tensor("pp_val")),
                               P(self.gpp_t), st), "gg_gradient p'")
        chk(L.kcfd_simple_correct(dm, self.alpha_p, P(self.pp_t), P(self.gpp_t), P(self.dP_t), P(self.U_t),
                                  P(self.p_t), P(self.p_norms), P(self.scratch), st), "simple_correct")
        chk(L.kcfd_simple_residual(self.ndim, P(self.mom_norms), P(self.p_norms), P(self.state), P(self.hist),
                                   P(self.it_dev), self.hist_cap, st), "simple_residual")

    def iterate(self, n=1):
        """Run n outer iterations (graph replay when graph=True). Solvers that run as
        their own graph (large FP64 systems) are not captured: for those the outer
        iteration is launched directly, its few kernel launches cost little beside
        the solves."""
        torch = _lib.require_cuda()
        self.bcs.upload()
        if self.graph and not (self.s_m.graph_engine or self.s_p.graph_engine):
            if self._graph is None:
                s = torch.cuda.Stream()
                s.wait_stream(torch.cuda.current_stream())
                with torch.cuda.stream(s):
                    self._step()      # warm-up outside capture (loads kernels, no allocations)
                torch.cuda.current_stream().wait_stream(s)
                g = torch.cuda.CUDAGraph()
                # thread-local capture: other host threads (a server building the next
                # case) may allocate and copy meanwhile
                with torch.cuda.graph(g, capture_error_mode="thread_local"):
                    self._step()
                self._graph = g
                n -= 1
            for _ in range(n):
                self._graph.replay()
        else:
            for _ in range(n):
                self._step()

    def reset_history(self):
        self.state.zero_()
        self.it_dev.zero_()
        self.hist.zero_()
        self.chist.zero_()

    def continuity_residual(self, k):
        """||b_p'|| of outer iteration k normalised by the first one (host read)."""
        c = self.chist[: k + 1].cpu().numpy()
        return float(c[k] / c[0]) if c[0] > 0 else 0.0

    def solve_steady(self):
        """models/single_phase.py:70-101 semantics; the residual history is kept on the
        device and read back once (and per iteration only when tol > 0)."""
        torch = _lib.require_cuda()
        self.reset_history()
        self.residuals = []
        done = 0
        converged = False
        while done < self.max_outer_iter:
            step = 1 if self.tol > 0 else self.max_outer_iter - done
            self.iterate(step)
            done += step
            if self.tol > 0:
                r = float(self.hist[done - 1].item())
                if r < self.tol:
                    converged = True
                    break
        torch.cuda.synchronize()
        self.residuals = self.hist[:done].cpu().numpy().tolist()
        return {"converged": converged, "iterations": done, "residuals": self.residuals}

    def solve_transient(self, t_end, dt=None):
        """models/single_phase.py:103-121: up to 30 SIMPLE iterations per step, stopping
        when the p' residual falls below 10 tol."""
        torch = _lib.require_cuda()
        if dt:
            self.dt = dt
        self.transient = True
        self._graph = None
        t, steps = 0.0, 0
        while t < t_end - 1e-15:
            self.U_old_t.copy_(self.U_t)
            for _ in range(30):
                self.iterate(1)
                pn = self.p_norms.cpu().numpy()
                rp = np.sqrt(pn[0]) / max(np.sqrt(pn[1]) + 1e-10, 1e-10)
                if rp < self.tol * 10:
                    break
            t += self.dt
            steps += 1
        self.transient = False
        self._graph = None
        return {"time_steps": steps, "final_time": t}

    # ---- profiles (models/single_phase.py:390-425) ----
    def _spacing(self, axis):
        """Centre distance along `axis` across the first internal face (in face order)
        where it exceeds 1e-10; 0.05 if there is none."""
        m = self.mesh
        cc = np.asarray(m.ccenter)
        internal = np.flatnonzero(np.asarray(m.neighbour) >= 0)
        d = np.abs(cc[np.asarray(m.owner)[internal], axis] - cc[np.asarray(m.neighbour)[internal], axis])
        big = np.flatnonzero(d > 1e-10)
        return float(d[big[0]]) if len(big) else 0.05

    def _profile(self, axis, target):
        cc = np.asarray(self.mesh.ccenter)
        sel = np.flatnonzero(np.abs(cc[:, axis] - target) < self._spacing(axis) * 1.5)
        pos = cc[sel, 1 - axis]
        U = self.U.values
        idx = np.argsort(pos)
        return pos[idx], U[sel, 0][idx], U[sel, 1][idx]

    def get_velocity_at_y(self, x_target, n_points=50):
        """(y, u, v) of the cells within 1.5 cell widths of x = x_target, sorted by y."""
        return self._profile(0, x_target)

    def get_velocity_at_x(self, y_target):
        """(x, u, v) of the cells within 1.5 cell heights of y = y_target, sorted by x."""
        return self._profile(1, y_target)

    def face_mass_flux(self):
        """Current face mass flux in reference face order (host)."""
        return self.dm.to_reference_faces(self.mf_t)

    def solver_stats(self):
        """Iterations / status of the last momentum and p' solves (host)."""
        return {"mom_iters": self.s_m.iters.cpu().numpy().tolist(), "mom_status": self.s_m.status.cpu().numpy().tolist(),
                "p_iters": int(self.s_p.iters[0]), "p_status": int(self.s_p.status[0])}
