"""Served SIMPLE requests: a continuous-batching request loop on one GPU.

Each request is a lid-driven cavity (2D quads N^2 or 3D hexes N^3, Reynolds number
Re, mu = 1/Re, lid speed 1) to be run until its continuity residual
||b_p'|| / ||b_p'(first iteration)|| falls below `cont_tol`. The reference has no such
definition (it tracks ||p'|| / ||p||, models/single_phase.py:377); b_p' is the mass
imbalance the pressure-correction equation removes.

Continuous batching: requests are admitted while free slots and the HBM budget allow
(footprint estimated from the mesh size), every admitted case keeps its mesh,
matrices and fields resident and gets its own CUDA stream (and, for cases small
enough for the single-CTA solver, a CUDA graph of one outer iteration), and the
scheduler enqueues `iters_per_tick` iterations per case and polls events without
blocking. Cases are built (host mesh, device set-up) on a worker thread, so the host
work of the next case overlaps the GPU work of the running ones. Admission takes
the queued request with the least estimated work first (policy "sjf", cells x a
dimension factor) or in arrival order ("fifo"). A case's result does not depend on
what runs beside it (its solves reduce in a fixed order on its own buffers), so it is
the same alone and in the mix.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib


@dataclass
class Request:
    rid: int
    ndim: int
    N: int
    Re: float
    arrival: float  # seconds after the start of the run


@dataclass
class Result:
    rid: int
    ndim: int
    N: int
    cells: int
    arrival: float
    admitted: float
    finished: float
    iterations: int
    converged: bool
    continuity: float
    fields: dict = field(default_factory=dict, repr=False)

    @property
    def latency(self):
        return self.finished - self.arrival


def make_requests(count, rate, seed=0, n2d=(32, 512), n3d=(16, 96), re=(100.0, 1000.0)):
    """Poisson arrivals at `rate` req/s; half 2D, half 3D (per request coin flip);
    N uniform in the given ranges; Re uniform."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    out = []
    for i in range(count):
        ndim = 2 if rng.random() < 0.5 else 3
        lo, hi = n2d if ndim == 2 else n3d
        N = int(rng.integers(lo, hi + 1))
        out.append(Request(i, ndim, N, float(rng.uniform(*re)), float(t[i])))
    return out


AMG_MIN_CELLS = 32768   # precond_p "auto": multigrid p' above this many cells, ILU(0) below


def p_precond_for(cells, precond_p):
    """The p' preconditioner of a case: precond_p, or for "auto" the multigrid for cases
    above AMG_MIN_CELLS cells (their p' solves run on the graph engine, where the
    multigrid takes an order of magnitude fewer Krylov iterations than ILU(0)) and
    ILU(0) for the small ones (one CTA each, so that concurrent cases overlap)."""
    if precond_p != "auto":
        return precond_p
    return "amg" if cells > AMG_MIN_CELLS else "ilu0"


def footprint_bytes(ndim, N, precision="mixed", precond_p="ilu0"):
    """Device bytes a resident case holds (mesh, two matrices, solver scratch, fields;
    a multigrid hierarchy at about 1.6 kB a cell, measured 3.3 GB at 128^3)."""
    n = N ** ndim
    F = ndim * n + ndim * N ** (ndim - 1)
    nnz = n + 2 * ndim * n
    mesh = F * (4 + 4 + 8 + 2 * 8 * ndim + 8 * 3 + 4 * 3) + n * (8 * ndim + 8 + 4 + 4) + nnz * 4
    mats = 2 * nnz * 8 + (2 * nnz * 4 if precision == "mixed" else 0)
    vw = 4 if precision == "mixed" else 8
    solver = 9 * n * ndim * vw + 9 * n * vw + n * ndim * 8 + nnz * (8 + 4 + 4 + vw) + 4 * n * 8
    fields = n * (ndim * 4 + 8) * 8 + F * 8 + n * ndim * ndim * 8
    amg = 1600 * n if p_precond_for(n, precond_p) == "amg" else 0
    return int(1.15 * (mesh + mats + solver + fields + amg)) + (8 << 20)


class Case:
    def __init__(self, req, precision="fp64", graph=True, precond_p="ilu0", rtol=1e-8, device="cuda",
                 small_team=1):
        torch = _lib.require_cuda()
        from .mesh import build_mesh
        from .meshgen import CAVITY_2D_NAMES, CAVITY_3D_NAMES, hex_box_arrays, quad_box_arrays
        from .simple import SIMPLESolver
        self.req = req
        N = req.N
        if req.ndim == 2:
            nodes, cells, bd = quad_box_arrays(0.0, 0.0, 1.0, 1.0, N, N, CAVITY_2D_NAMES)
            m = build_mesh(nodes, cells, bd)
        else:
            nodes, cells, cf, bd = hex_box_arrays(1.0, 1.0, 1.0, N, N, N, CAVITY_3D_NAMES)
            m = build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
        self.stream = torch.cuda.Stream()
        with torch.cuda.stream(self.stream):
            # small_team=1: one CTA per solve for the small cases, so that concurrent cases
            # overlap on the device (0: the library's choice, best for one case alone);
            # the large ones take the grid-wide solvers either way
            team = small_team if m.n_cells * m.ndim <= 40000 else 0
            # 'mixed' takes effect above 40,000 cells (the engine's FP32 momentum solve,
            # the multigrid p' hierarchy in FP32); the small cases run latency-bound
            # single-CTA solves, where FP32 storage saves nothing, in FP64
            prec = precision if (precision != "mixed" or m.n_cells > 40000) else "fp64"
            s = SIMPLESolver(m, rho=1.0, mu=1.0 / req.Re, precision=prec,
                             precond_p=p_precond_for(m.n_cells, precond_p), rtol=rtol, graph=graph, team=team)
            for nm in m.boundary_patches:
                lid = [1.0] + [0.0] * (m.ndim - 1)
                s.set_velocity_bc(nm, "dirichlet", lid if nm == "lid" else [0.0] * m.ndim)
                s.set_pressure_bc(nm, "zero_gradient")
            s.alpha_u, s.alpha_p, s.tol = 0.7, 0.3, 0.0
            s.reset_history()
        self.solver = s
        self.cells = m.n_cells
        self.done_iters = 0
        self.pending = None
        self.host = torch.zeros(2, dtype=torch.float64).pin_memory()
        self.event = None

    def launch(self, k):
        torch = _lib.require_cuda()
        with torch.cuda.stream(self.stream):
            self.solver.iterate(k)
            self.done_iters += k
            self.host[0:1].copy_(self.solver.chist[0:1], non_blocking=True)
            self.host[1:2].copy_(self.solver.chist[self.done_iters - 1:self.done_iters], non_blocking=True)
            self.event = torch.cuda.Event()
            self.event.record(self.stream)

    def ready(self):
        return self.event is None or self.event.query()

    def continuity(self):
        c0, c = float(self.host[0]), float(self.host[1])
        return c / c0 if c0 > 0 else 0.0

    def fields(self):
        return {"U": self.solver.U.values, "p": self.solver.p.values}


def work_estimate(req):
    """Relative work of a request for shortest-job-first admission."""
    return req.N ** req.ndim * (1.5 if req.ndim == 3 else 1.0)


class Server:
    def __init__(self, budget_bytes=150e9, max_active=64, iters_per_tick=10, max_iters=3000, cont_tol=1e-6,
                 precision="fp64", graph=True, precond_p="ilu0", keep_fields=False, verbose=False,
                 policy="fifo", builders=1, small_team=1):
        self.budget = budget_bytes
        self.max_active = max_active
        self.k = iters_per_tick
        self.max_iters = max_iters
        self.cont_tol = cont_tol
        self.precision, self.graph, self.precond_p = precision, graph, precond_p
        self.keep_fields = keep_fields
        self.verbose = verbose
        if policy not in ("fifo", "sjf"):
            raise ValueError(f"unknown admission policy {policy!r}")
        self.policy = policy
        self.builders = max(1, int(builders))
        # solver team of the cases up to 40,000 unknowns when served beside others: 1 (one
        # CTA per solve) or 0 (the library's choice, the grid kernel above 1,024 unknowns)
        self.small_team = int(small_team)

    def run(self, requests, serial=False, case_factory=None):
        """Serve `requests` in real time (arrival times honoured). serial=True runs one
        case at a time (the serial comparator). Returns a list of Result; `last_stats`
        then holds the peak admitted footprint and the peak number of resident cases.

        case_factory(request) -> case replaces the device-resident `Case` (same members:
        req, cells, done_iters, launch(k), ready(), continuity(), fields()); the default
        builds a Case on the current GPU."""
        from concurrent.futures import ThreadPoolExecutor
        if case_factory is None:
            torch = _lib.require_cuda()
            dev = torch.cuda.current_device()

            def build(r):
                torch.cuda.set_device(dev)
                # alone, a case takes the library's fastest single-case solvers
                return Case(r, self.precision, self.graph, self.precond_p, small_team=0 if serial else self.small_team)

            finish = torch.cuda.synchronize
        else:
            build, finish = case_factory, (lambda: None)
        reqs = sorted(requests, key=lambda r: r.arrival)
        pending = list(reqs)
        queue, building, active, results = [], [], [], []
        used = peak_used = peak_resident = 0
        max_active = 1 if serial else self.max_active

        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=self.builders) as pool:
            while pending or queue or building or active:
                now = time.perf_counter() - t0
                while pending and pending[0].arrival <= now:
                    queue.append(pending.pop(0))
                progressed = False
                # admission: while a slot and the HBM budget allow; the case is built
                # on a worker thread
                while queue and len(active) + len(building) < max_active:
                    pick = 0
                    if self.policy == "sjf":
                        pick = min(range(len(queue)), key=lambda i: work_estimate(queue[i]))
                    r = queue[pick]
                    fp = footprint_bytes(r.ndim, r.N, self.precision, self.precond_p)
                    if (active or building) and used + fp > self.budget:
                        break
                    queue.pop(pick)
                    used += fp
                    building.append((r, fp, time.perf_counter() - t0, pool.submit(build, r)))
                    peak_used = max(peak_used, used)
                    peak_resident = max(peak_resident, len(active) + len(building))
                    progressed = True
                # built cases start their first tick
                still_b = []
                for r, fp, adm, fut in building:
                    if not fut.done():
                        still_b.append((r, fp, adm, fut))
                        continue
                    c = fut.result()
                    c.admitted, c.fp = adm, fp
                    c.launch(self.k)
                    active.append(c)
                    progressed = True
                building = still_b
                # progress: poll without blocking; finished cases leave, others continue
                still = []
                for c in active:
                    if not c.ready():
                        still.append(c)
                        continue
                    progressed = True
                    cont = c.continuity()
                    if cont < self.cont_tol or c.done_iters >= self.max_iters:
                        fin = time.perf_counter() - t0
                        res = Result(c.req.rid, c.req.ndim, c.req.N, c.cells, c.req.arrival, c.admitted, fin,
                                     c.done_iters, cont < self.cont_tol, cont,
                                     c.fields() if self.keep_fields else {})
                        results.append(res)
                        used -= c.fp
                        if self.verbose:
                            print(f"  done rid={res.rid} {res.ndim}D N={res.N} iters={res.iterations} "
                                  f"latency={res.latency:.3f}s cont={cont:.2e}", flush=True)
                        del c
                    else:
                        c.launch(self.k)
                        still.append(c)
                active = still
                if not progressed:
                    time.sleep(0.0002)
        finish()
        self.last_stats = {"peak_bytes": peak_used, "peak_resident": peak_resident}
        return results


def summarize(results):
    lat = np.array([r.latency for r in results])
    t_end = max(r.finished for r in results)
    t_start = min(r.arrival for r in results)
    return {"cases": len(results), "converged": int(sum(r.converged for r in results)),
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "cases_per_s": float(len(results) / max(t_end - t_start, 1e-9)),
            "mean_iterations": float(np.mean([r.iterations for r in results]))}
