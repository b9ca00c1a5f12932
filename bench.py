"""Benchmark: SIMPLE outer iterations per second on the 3D jittered lid-driven cavity.

Workload (the headline config that fits one GPU): 128^3 hexahedra (2,097,152 cells) on
the unit cube, interior nodes jittered by U(-0.2, 0.2) x spacing (seed 0), Re = 400
(rho = 1, mu = 0.0025), MUSCL van Leer deferred correction, over-relaxed
non-orthogonal correction, Green-Gauss gradients, BiCGSTAB + Jacobi for u, v, w and
BiCGSTAB for p' preconditioned by the device smoothed-aggregation multigrid (one V-cycle
per apply; --p-precond ilu0 takes the red-black ILU(0) instead), each solve to a 1e-8
relative residual; alpha_u = 0.7, alpha_p = 0.3. FP64 throughout; the solves run on the
graph engine (phase kernels in one CUDA graph per solve with a device-side WHILE loop).

A "step" is one SIMPLE outer iteration. Inputs (mesh, matrices, fields: several GB)
are far larger than the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--size S]

The line also carries, measured in the same run: the config's own p' preconditioner
(ILU(0)) as `ilu0_variant`; the mixed form (FP32 multigrid hierarchy and momentum inner
iterations, FP64 Krylov residuals) with its relative L2 error against the FP64 fields
per component (u, v, w, p, p'); a bounded batched leg of C4 (1,024-system p' batch:
its first systems, batched against the plain drop-in) and a short served leg of C5
(Poisson-arriving cavities, served against serial); and the CPU baseline: one full
outer iteration of the same 128^3 workload by the oracle on the host, measured, not
scaled.

Multi-GPU: one mesh does not shard without a halo exchange, so N > 1 runs N
independent replicas (one per rank, torch.distributed over NCCL for the barrier and
the max-over-ranks timing); value = total iterations / max time.

--impl reference times the oracle (the numpy/scipy restatement of the reference's
path, with the device's red-black ILU(0) for p') on the host cores on the full 128^3
workload, as many whole outer iterations as fit its time budget.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "k-cfd_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "SIMPLE outer iterations/s (3D jittered cavity, 1e-8 relative residual per solve)"
UNIT = "iters/s"
REF_BUDGET_S = 160.0   # reference arm: whole 128^3 outer iterations while the timed work stays below this


def cavity_arrays(N, seed=0):
    from kcfd import meshgen
    nodes, cells, cf, bd = meshgen.hex_box_arrays(1.0, 1.0, 1.0, N, N, N, meshgen.CAVITY_3D_NAMES)
    nodes = meshgen.jitter_interior(nodes, (N, N, N), (1.0 / N,) * 3, 0.2, seed=seed)
    return nodes, cells, cf, bd


def make_solver(N, precision="fp64", graph=True, p_precond="amg", mesh=None):
    from kcfd import mesh as km
    from kcfd.simple import SIMPLESolver
    if mesh is None:
        nodes, cells, cf, bd = cavity_arrays(N)
        mesh = km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
    s = SIMPLESolver(mesh, rho=1.0, mu=0.0025, precision=precision, precond_p=p_precond, ilu_order="color",
                     rtol=1e-8, maxiter=20000, muscl="van_leer", nonorth=True, graph=graph)
    for nm in mesh.boundary_patches:
        s.set_velocity_bc(nm, "dirichlet", [1.0, 0.0, 0.0] if nm == "lid" else [0.0, 0.0, 0.0])
        s.set_pressure_bc(nm, "zero_gradient")
    s.alpha_u, s.alpha_p, s.tol = 0.7, 0.3, 0.0
    return s


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.gpu = gpu_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one p' Krylov iteration
# on the 128^3 cavity, from an ncu launch list of one solve on the graph engine
# (KCFD_ENGINE_EAGER=1, every kernel of the solve captured, one pass each), divided
# by the solve's Krylov count; the roofline's traffic is this times the timed solve's
# count. Keyed by preconditioner; None where no capture was made.
NCU_P_ITER_DRAM_BYTES_128 = {"ilu0": 857019136, "amg": 2471459375}


def amg_levels(solver):
    """Rows, entries and prolongator entries of each level of an AMG handle."""
    return solver.amg_levels() if solver.precond == "amg" else None


def vcycle_bytes(levels, w):
    """Algorithmic bytes of one V(1,1) cycle (each array once per kernel): per level l
    above the coarsest, the pre-smoothing and residual (W values and columns, b, omega
    D^-1, x and r written), the restriction (P^T values and columns, row pointers, r,
    the coarse right-hand side), the prolongation (P values and columns, row pointers,
    the coarse correction, x read and written) and the post-smoothing (A values and
    columns, x, b, omega D^-1, y); at the coarsest level the dense inverse and two
    vectors. Level 0's b and y are the Krylov FP64 vectors."""
    b = 0
    L = len(levels)
    for l in range(L - 1):
        n, nnz, pn = levels[l]["rows"], levels[l]["nnz"], levels[l]["p_nnz"]
        nc = levels[l + 1]["rows"]
        wi = 8 if l == 0 else w
        b += nnz * (w + 4) + n * (wi + 3 * w)                 # pre + residual
        b += pn * (w + 4) + 4 * (nc + 1) + n * w + nc * w     # restriction
        b += pn * (w + 4) + 4 * (n + 1) + nc * w + 2 * n * w  # prolongation
        b += nnz * (w + 4) + n * (2 * w + 2 * wi)             # post-smoothing
    nc = levels[-1]["rows"]
    wi = 8 if L == 1 else w
    return b + nc * nc * w + 2 * nc * wi


def solver_bytes(n, nnz, iters, precond, w, nrhs=1, amg=None):
    """Algorithmic bytes of BiCGSTAB iterations (each array counted once per use):
    SpMV nnz(w+4) + 4(n+1) + 2 n w nrhs; ILU(0) apply nnz(w+4) + 8(n+1) + 4 n w;
    Jacobi iteration 2 SpMV + 21 n w nrhs; ILU iteration 2 SpMV + 2 ILU + 19 n w;
    multigrid iteration 2 FP64 SpMV + 2 V-cycles (vcycle_bytes, hierarchy value width w)
    + 17 n 8 (the engine's FP64 vector streams: p update 4, v.rhat 1, s 3, s read 1,
    x and r update 8)."""
    spmv = nnz * (w + 4) + 4 * (n + 1) + 2 * n * w * nrhs
    if precond == "amg":
        spmv8 = nnz * 12 + 4 * (n + 1) + 16 * n
        return iters * (2 * spmv8 + 2 * vcycle_bytes(amg, w) + 17 * n * 8)
    if precond == "ilu0":
        ilu = nnz * (w + 4) + 8 * (n + 1) + 4 * n * w
        return iters * (2 * spmv + 2 * ilu + 19 * n * w)
    return iters * (2 * spmv + 21 * n * w * nrhs)


def outer_step_bytes(n, Fi, Fb, nnz, ndim, its_m, its_p, p_precond="amg", amg=None, w=8):
    """Algorithmic bytes of one SIMPLE outer iteration by the fixed formulas (each
    array counted once per use): mass flux twice, Green-Gauss of U (ndim components)
    and of p', MUSCL and momentum assembly per component, p' assembly, the momentum
    solve (Jacobi, ndim right-hand sides) and the p' solve at the step's Krylov counts.
    The correction, residual bookkeeping and preconditioner set-up are left out."""
    F = Fi + Fb
    mass_flux = F * (8 + 8 + (1 + ndim) * 8 + 8) + n * ndim * 8
    gg = Fi * (8 + ndim * 8 + 8) + Fb * (4 + ndim * 8 + 8) + n * (16 + ndim * 8)
    muscl = Fi * (8 + 8 + ndim * 8) + n * (8 + 2 * ndim * 8 + 8)
    asm = Fi * (8 + (1 + ndim) * 8 + 16 + 8 + 2 * w) + Fb * (4 + (1 + ndim) * 8 + 8 + 8 + 8) + n * (32 + 2 * w)
    b = 2 * mass_flux + (ndim + 1) * gg + ndim * (muscl + asm) + asm
    b += solver_bytes(n, nnz, its_m, "jacobi", w, nrhs=ndim)
    b += solver_bytes(n, nnz, its_p, p_precond, w, amg=amg)
    return b


def solve_launches(solver, iters):
    """Kernels one solve launches: the persistent kernels launch once; the graph
    engine launches the value fill, init, final and the two copies plus, per loop
    trip, the phase kernels (5), 2 (nlev - 1) ILU sweeps for each of phat and shat, or
    two V-cycles (4 kernels per level above the coarsest and the coarse solve)."""
    if not solver.graph_engine:
        return 1
    info = solver.info()
    body = 5
    if solver.precond == "ilu0":
        body += 4 * (info["levels"] - 1)
    elif solver.precond == "amg":
        L = info["levels"]
        body += 2 * (1 if L == 1 else 4 * (L - 1) + 1)
    return 5 + body * int(iters)


def setup_launches(solver, power_iters=8):
    """Kernels of one preconditioner set-up: Jacobi 1; ILU(0) permute + factor (+ 2
    SELL fills on the graph engine); AMG per level above the coarsest 9 (level 0) or
    10 + power iterations, and 2 for the coarsest."""
    if solver.precond == "jacobi":
        return 1
    if solver.precond == "ilu0":
        return 2 + (2 if solver.graph_engine else 0)
    if solver.precond == "amg":
        L = solver.info()["levels"]
        return (9 if L > 1 else 0) + max(0, L - 2) * (10 + power_iters) + 2
    return 0


def launches_per_step(s, its_m, its_p):
    """Kernels of libkcfd launched by one outer iteration (excluding memsets), with
    the Krylov counts of that iteration."""
    nci, ncb = s.dm.desc.n_colors_int, s.dm.desc.n_colors_bnd
    per_colour_pass = nci + ncb
    gg = per_colour_pass + 1
    mom = per_colour_pass + 1
    pp = per_colour_pass + 1
    n = 2                       # mass flux x2
    n += gg if s.gU_t is not None else 0
    n += mom + 2                # momentum assembly, residual norms (2)
    n += pp + 2                 # p' assembly, norm + record
    n += gg + 2 + 1             # GG p', correction (2), residual bookkeeping
    n += setup_launches(s.s_m) + setup_launches(s.s_p)
    n += solve_launches(s.s_m, its_m)
    n += solve_launches(s.s_p, its_p)
    return n


def p_solve_roofline(s, peak, reps=3):
    """The p' solve timed alone with CUDA events on its stream (after its set-up, which
    is timed on its own); algorithmic bytes from its Krylov count. Also the FP64 SpMV
    kernel alone on the same matrix."""
    import torch
    n, nnz = s.mesh.n_cells, s.mesh.nnz
    pc = s.s_p.precond
    mixed = s.mode == 1
    w = 4 if mixed else 8
    amg = amg_levels(s.s_p)
    times, byts, setups = [], [], []
    for _ in range(reps):
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        s.s_p.setup(s.A_p)
        e1.record()
        s.pp_t.zero_()
        torch.cuda.synchronize()
        e1b = torch.cuda.Event(enable_timing=True)
        e1b.record()
        s.s_p.solve(s.A_p, s.b_p, s.pp_t)
        e2.record()
        torch.cuda.synchronize()
        it = int(s.s_p.iters[0])
        b = solver_bytes(n, nnz, it, pc, w, amg=amg)
        if mixed and pc != "amg":  # outer FP64 residuals (about one per 40 inner iterations) + updates
            nref = max(2, it // 40)
            b += nref * (nnz * 12 + 4 * (n + 1) + 2 * n * 8 + 5 * n * 8)
        times.append(e1b.elapsed_time(e2) / 1e3)
        setups.append(e0.elapsed_time(e1) / 1e3)
        byts.append(b)
    t = float(np.mean(times))
    ach = float(np.mean(byts)) / t / 1e9
    info = s.s_p.info()
    prec_name = {"amg": f"smoothed-aggregation multigrid ({info['levels']} levels, one V(1,1) cycle per apply)",
                 "ilu0": "ILU(0), red-black levels", "jacobi": "Jacobi"}[pc]
    kern = (f"graph engine: g_p, V-cycle/ILU sweeps, g_spmv_v, g_s, g_spmv_t, g_xr per Krylov iteration "
            f"(p' BiCGSTAB + {prec_name}, {'FP32 hierarchy / FP64 Krylov' if mixed else 'FP64'})"
            if info["team"] == 3 else f"solve_grid_kernel (p' BiCGSTAB + {prec_name})")
    # SpMV alone: nnz (8 + 4) + 4 (n + 1) + 8 n (x) + 8 n (y)
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(3):
        s.A_p.spmv(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    K = 50
    e0.record()
    for _ in range(K):
        s.A_p.spmv(x, y)
    e1.record()
    torch.cuda.synchronize()
    ts = e0.elapsed_time(e1) / 1e3 / K
    sb = nnz * 12 + 4 * (n + 1) + 16 * n
    spmv = {"kernel": "spmv_row_kernel<double> (kcfd_spmv_f64, row per thread, entries loaded before the x gathers)",
            "bytes": int(sb), "launch_us": round(ts * 1e6, 2), "achieved": round(sb / ts / 1e9, 1),
            "frac": round(sb / ts / 1e9 / peak[0], 3)}
    it = int(s.s_p.iters[0])
    per_it = solver_bytes(n, nnz, 1, pc, w, amg=amg)
    moved = None
    if pc == "ilu0" and info["team"] == 3 and info["levels"] >= 2:
        # on ILU level 0 A M^-1 q = q, so two SpMVs skip those rows' values, columns
        # and row pointers, and v = p, t = s there are neither stored nor read back
        lev = np.asarray(s.mesh.cell_color)
        rl = np.diff(np.asarray(s.mesh.indptr))
        n0, nnz0 = int((lev == 0).sum()), int(rl[lev == 0].sum())
        mv = per_it - 2 * (nnz0 * (w + 4) + 4 * n0) - 4 * n0 * w
        moved = {"bytes_per_krylov_iter": int(mv), "achieved": round(mv * it / t / 1e9, 1),
                 "frac": round(mv * it / t / 1e9 / peak[0], 3)}
    ncu = NCU_P_ITER_DRAM_BYTES_128.get(pc) if (n == 128 ** 3 and info["team"] == 3 and not mixed) else None
    return {"bound": "hbm", "kernel": kern, "unit_of_work": "one p' solve (Krylov iterations x bytes/iteration)",
            "achieved": round(ach, 1), "peak": peak[0], "unit": "GB/s", "frac": round(ach / peak[0], 3),
            "moved": moved, "peak_source": peak[1],
            "traffic": int(ncu * it) if ncu else None,
            "traffic_source": "ncu launch list of one solve (DRAM bytes per Krylov iteration) x Krylov count"
            if ncu else None,
            "launch_ms": round(t * 1e3, 3), "setup_ms": round(float(np.mean(setups)) * 1e3, 3),
            "krylov_iters": it, "bytes_per_krylov_iter": int(per_it),
            "hierarchy": amg, "spmv": spmv}


def timed_iterations(s, steps):
    """Run `steps` outer iterations between CUDA events; keeps each step's Krylov
    counts (device copies, read after the timed region)."""
    import torch
    its = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        s.iterate(1)
        its.append((s.s_m.iters.max().clone(), s.s_p.iters[0].clone()))
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3, [(int(a), int(b)) for a, b in its]


def fields_of(s):
    return {"u": s.U.values[:, 0], "v": s.U.values[:, 1], "w": s.U.values[:, 2], "p": s.p.values,
            "pp": s.pp_t.detach().cpu().numpy().copy()}


def field_errors(ref, test):
    """Relative L2 error of each field of `test` against `ref`."""
    return {k: float(np.linalg.norm(test[k] - ref[k]) / max(np.linalg.norm(ref[k]), 1e-300)) for k in ref}


def start_cpu_sample(N):
    """The CPU baseline in a separate host process (it runs beside the GPU legs that
    follow the timed region): one full outer iteration of the same workload by the
    oracle. BLAS threads capped at 8 so it cannot crowd the launching thread."""
    env = dict(os.environ, OMP_NUM_THREADS="8", OPENBLAS_NUM_THREADS="8", MKL_NUM_THREADS="8")
    return subprocess.Popen([sys.executable, os.path.abspath(__file__), "--impl", "cpu-sample", "--size", str(N)],
                            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, env=env)


def collect_cpu_sample(proc, timeout_s=900.0):
    if proc is None:
        return None
    try:
        out, _ = proc.communicate(timeout=timeout_s)
    except subprocess.TimeoutExpired:
        proc.kill()
        proc.communicate()
        return {"unavailable": f"the host oracle did not finish within {timeout_s:.0f} s"}
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    if proc.returncode != 0 or not lines:
        return {"unavailable": f"the host oracle exited with {proc.returncode}"}
    r = json.loads(lines[-1])
    return cpu_baseline_entry(r)


def cpu_baseline_entry(r):
    t = float(np.mean([x["s"] for x in r["steps"]]))
    kry = [x["p_krylov"] for x in r["steps"]]
    return {"value": round(1.0 / t, 6), "unit": UNIT, "cores": 1, "kind": "port",
            "host_cores_available": r["host_cores"],
            "sample": f"the oracle (numpy/scipy restatement of the reference path: BiCGSTAB + Jacobi for u, v, w, "
                      f"BiCGSTAB + ILU(0) in the device's red-black order for p', rtol 1e-8, MUSCL van Leer, "
                      f"non-orthogonal correction) on the full {r['N']}^3 workload: {len(r['steps'])} whole outer "
                      f"iteration(s) from the initial state, {t:.1f} s each (p' Krylov counts {kry}); mesh build "
                      f"{r['build_s']:.0f} s and colouring not timed; single-threaded sparse kernels",
            "seconds_per_step": [round(x["s"], 2) for x in r["steps"]], "p_krylov": kry}


def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=900))
    dev = torch.cuda.current_device()
    N = args.size
    t_setup = time.time()
    s = make_solver(N, precision="mixed" if args.mixed else "fp64", graph=True, p_precond=args.p_precond)
    setup_s = time.time() - t_setup
    if args.iterate_only:
        # a fixed number of outer iterations from the initial state and nothing else:
        # the command the committed ncu launch lists are taken on (no timing here)
        s.iterate(args.iterate_only)
        torch.cuda.synchronize()
        print(json.dumps({"iterated": args.iterate_only, "setup_s": round(setup_s, 2), **s.solver_stats()}))
        return
    mesh = s.mesh
    n_faces, nnz = int(mesh.n_faces), int(mesh.nnz)
    s.reset_history()
    s.iterate(args.warmup)
    torch.cuda.synchronize()
    # the state the timed region starts from (U, p: everything else is rebuilt from
    # them each outer iteration); the e2e leg replays the same steps from it
    D = 3
    Uh = torch.empty(mesh.n_cells, D, dtype=torch.float64).pin_memory()
    ph = torch.empty(mesh.n_cells, dtype=torch.float64).pin_memory()
    Uh.copy_(s.U_t.cpu())
    ph.copy_(s.p_t.cpu())
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as cs:
        t, its = timed_iterations(s, args.steps)
    if world > 1:
        dist.barrier()
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    clocks = cs.summary()
    value = world * args.steps / t
    fields64 = fields_of(s)
    stats = s.solver_stats()
    launches = sum(launches_per_step(s, a, b) for a, b in its)
    res_hist = s.hist[: args.warmup + args.steps].cpu().numpy()
    # e2e through the reference-facing API with host buffers: the same steps as the
    # timed region (from the same state), each taking U, p from pinned host memory
    # and returning them there
    torch.cuda.synchronize()
    ke = args.steps
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(ke):
        s.U_t.copy_(Uh, non_blocking=True)
        s.p_t.copy_(ph, non_blocking=True)
        s.iterate(1)
        Uh.copy_(s.U_t, non_blocking=True)
        ph.copy_(s.p_t, non_blocking=True)
        torch.cuda.synchronize()
    te = time.perf_counter() - t0
    if world > 1:
        tt = torch.tensor([te], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        te = float(tt.item())
    e2e = {"value": round(world * ke / te, 3), "unit": UNIT, "h2d_bytes_per_step": int(mesh.n_cells * (D + 1) * 8),
           "d2h_bytes_per_step": int(mesh.n_cells * (D + 1) * 8), "steps": ke}
    cpu_proc = start_cpu_sample(N) if (rank == 0 and world == 1 and not args.no_cpu) else None
    roof = p_solve_roofline(s, measured_peak()) if rank == 0 else None
    if roof is not None:
        # the whole outer iteration against the same peak
        Fi = int(mesh.n_internal_faces)
        amg = roof["hierarchy"]
        ob = sum(outer_step_bytes(mesh.n_cells, Fi, n_faces - Fi, nnz, 3, a, b, args.p_precond, amg) for a, b in its)
        roof["outer_iteration"] = {"bytes_per_step": int(ob / len(its)), "achieved": round(ob / t / 1e9, 1),
                                   "frac": round(ob / t / 1e9 / roof["peak"], 3),
                                   "note": "formula bytes of all assembly, gradient, mass-flux and solve work of "
                                           "the timed steps (their Krylov counts; preconditioner set-up not "
                                           "counted) / the timed region"}
    del s
    torch.cuda.empty_cache()
    variants = {}
    if args.plain and rank == 0:
        # the mixed form on the same mesh, the same number of outer iterations from the
        # same initial state: rate and each field's error against the FP64 fields
        sm = make_solver(N, precision="mixed", graph=True, p_precond=args.p_precond, mesh=mesh)
        sm.iterate(args.warmup)
        torch.cuda.synchronize()
        tm, its_m = timed_iterations(sm, args.steps)
        variants["mixed_precision_variant"] = {
            "value": round(args.steps / tm, 3), "unit": UNIT, "steps": args.steps, "krylov_iters_per_step": its_m,
            "field_error": field_errors(fields64, fields_of(sm)),
            "desc": "same workload, mixed form: momentum BiCGSTAB + Jacobi with FP32 inner iterations and FP64 "
                    "refinement; p' multigrid hierarchy and V-cycles stored in FP32 (FP64 arithmetic) under an "
                    "FP64 Krylov iteration; field_error = relative L2 against the FP64 run after the same "
                    f"{args.warmup + args.steps} outer iterations (u, v, w, p, and p' of the last iteration)"}
        del sm
        torch.cuda.empty_cache()
        if args.p_precond != "ilu0":
            si = make_solver(N, precision="fp64", graph=True, p_precond="ilu0", mesh=mesh)
            si.iterate(args.warmup)
            torch.cuda.synchronize()
            k = args.steps
            ti, its_i = timed_iterations(si, k)
            variants["ilu0_variant"] = {
                "value": round(k / ti, 3), "unit": UNIT, "steps": k, "krylov_iters_per_step": its_i,
                "field_error_vs_main": field_errors(fields64, fields_of(si)),
                "desc": "same workload with the config's named p' preconditioner: BiCGSTAB + ILU(0) (red-black "
                        "levels) on the graph engine, FP64; field_error_vs_main: two FP64 runs whose p' solves "
                        "stop at the same 1e-8 residual with different preconditioners, the noise floor of the "
                        "field errors at this tolerance"}
            del si
            torch.cuda.empty_cache()
    legs = {}
    if rank == 0 and world == 1 and args.legs:
        if "c4" in args.legs:
            legs["batched_c4"] = c4_measure(count=args.leg_systems, steps=1, warmup=1, mode="fp64", plain=True,
                                            plain_budget_s=20.0, cpu=False)
        if "c5" in args.legs:
            legs["served_c5"] = c5_measure(requests=args.leg_requests, rate=args.rate, cont_tol=args.cont_tol,
                                           max_iters=args.max_iters, max_active=args.max_active,
                                           policy=args.policy, serial=True)
    cpu = collect_cpu_sample(cpu_proc)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        pname = {"amg": "smoothed-aggregation multigrid", "ilu0": "ILU(0) red-black"}.get(args.p_precond,
                                                                                           args.p_precond)
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * t / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"3D jittered lid-driven cavity {N}^3 hex ({N**3} cells), Re 400, MUSCL van Leer, "
                                   f"over-relaxed non-orthogonal, BiCGSTAB + {pname} p' / Jacobi u,v,w, rtol 1e-8, "
                                   "FP64, graph-engine solves",
                       "cells": N ** 3, "faces": n_faces, "nnz": nnz, "p_precond": args.p_precond,
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "working set >> 126 MB L2; no flush needed", "setup_s": round(setup_s, 2)},
            "clocks": clocks, "e2e": e2e, "roofline": roof, "cpu_baseline": cpu,
            "gpu_launches": launches, "krylov_iters_per_step": its,
            "solver_stats_last_step": stats,
            "residual_first_last": [float(res_hist[0]), float(res_hist[-1])],
        }
        line.update(variants)
        line.update(legs)
        print(json.dumps(line))


C4_METRIC = "p' systems solved/s (1,024 Delaunay systems, 1e-8 relative residual each)"
C4_TOTAL = 1024


def _c4_bytes(n, nnz, iters, mixed):
    """Algorithmic bytes of one system's batched solve: BiCGSTAB + Jacobi iterations
    (w = 4 mixed, 8 FP64) plus, mixed, about one FP64 refinement step (residual SpMV
    and 5 vector streams) per 40 inner iterations."""
    w = 4 if mixed else 8
    b = solver_bytes(n, nnz, iters, "jacobi", w)
    if mixed:
        nref = max(2, iters // 40)
        b += nref * (nnz * 12 + 4 * (n + 1) + 2 * n * 8 + 5 * n * 8)
    return b


def c4_measure(count=C4_TOTAL, steps=1, warmup=1, mode="fp64", plain=True, plain_budget_s=60.0, cpu=True,
               restarts=20, world=1, rank=0):
    """The first `count` of the 1,024 C4 systems (cell counts log-uniform in [2e3, 2e5],
    seed 0; the same systems whatever the count) solved together: BiCGSTAB + Jacobi to
    1e-8 per system, one persistent launch per size tier, a system whose rho or omega
    breaks down restarted (up to `restarts` times). Returns the measurements: batched
    solves/s over converged systems, e2e with host buffers, the plain FP64 drop-in per
    system over a bounded prefix, the CPU scipy path over a bounded prefix."""
    import torch
    import torch.distributed as dist
    from scipy import sparse
    from kcfd.batch import BatchSolver, lpt_shards, p_prime_batch, p_prime_sizes
    sizes = p_prime_sizes(C4_TOTAL, 2000, 200000, 0)[:count]
    mine = lpt_shards(sizes * 4, world)[rank] if world > 1 else list(range(count))
    workers = max(1, min(os.cpu_count() or 1, 64) // max(world, 1))
    t0 = time.time()
    from kcfd.batch import _p_prime_host
    if workers > 1 and len(mine) > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            host = list(ex.map(_p_prime_host, mine, [sizes[k] for k in mine], [0] * len(mine), chunksize=2))
    else:
        host = [_p_prime_host(k, sizes[k], 0) for k in mine]
    gen_s = time.time() - t0
    pats, vals, rhs, _ = p_prime_batch(len(mine), host=host)
    n_sys = np.array([len(ip) - 1 for ip, _ in pats])
    nnz_sys = np.array([len(ix) for _, ix in pats])
    mixed = mode == "mixed"
    bs = BatchSolver(pats, mode=mode, precond="jacobi", rtol=1e-8, maxiter=20000, restarts=restarts)
    v = torch.cat(vals)
    b = bs.pack(rhs)
    x = torch.zeros_like(b)
    for _ in range(warmup):
        x.zero_()
        bs.solve(v, b, x)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    dev = torch.cuda.current_device()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as cs:
        e0.record()
        for _ in range(steps):
            x.zero_()
            bs.solve(v, b, x)
        e1.record()
        torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    if world > 1:
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    clocks = cs.summary()
    its = bs.iters.cpu().numpy()
    st = bs.status.cpu().numpy()
    xs = bs.unpack(x)
    # parity: true FP64 residual of every system (host scipy CSR)
    true_rel = []
    for k in range(len(mine)):
        A = sparse.csr_matrix((vals[k].cpu().numpy(), pats[k][1], pats[k][0]), shape=(n_sys[k], n_sys[k]))
        true_rel.append(float(np.linalg.norm(rhs[k] - A @ xs[k]) / np.linalg.norm(rhs[k])))
    true_rel = np.asarray(true_rel)
    ok = (st == 0) & (true_rel <= 1.5e-8)
    byts = sum(_c4_bytes(int(n_sys[k]), int(nnz_sys[k]), int(its[k]), mixed) for k in range(len(mine)))
    launch = t / steps
    peak = measured_peak()
    tiers = bs.tiers()
    roof = {"bound": "hbm", "kernel": f"batch_cluster_kernel<MIXED={int(mixed)}, JACOBI> ({tiers['cluster']} systems on "
                                      f"thread-block clusters of 2-{tiers['cluster_size']} CTAs graded by size) + "
                                      f"batch_kernel<MIXED={int(mixed)}, JACOBI, 512 | 256> (one CTA per system), "
                                      "largest first, one persistent launch per tier",
            "unit_of_work": "one launch solving all systems", "achieved": round(byts / launch / 1e9, 1),
            "peak": peak[0], "unit": "GB/s", "frac": round(byts / launch / 1e9 / peak[0], 3),
            "peak_source": peak[1], "traffic": None, "launch_ms": round(launch * 1e3, 3)}
    # e2e through the public batch API with host buffers: values and right-hand
    # sides from pinned host memory, solutions back, every step
    vh = v.cpu().pin_memory()
    bh = b.cpu().pin_memory()
    xh = torch.empty_like(bh).pin_memory()
    torch.cuda.synchronize()
    te0 = time.perf_counter()
    for _ in range(steps):
        v.copy_(vh, non_blocking=True)
        b.copy_(bh, non_blocking=True)
        x.zero_()
        bs.solve(v, b, x)
        xh.copy_(x, non_blocking=True)
        torch.cuda.synchronize()
    te = time.perf_counter() - te0
    if world > 1:
        tt = torch.tensor([te], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        te = float(tt.item())
    n_ok = int(ok.sum())
    if world > 1:
        nt = torch.tensor([n_ok], device="cuda", dtype=torch.int64)
        dist.all_reduce(nt)
        n_ok_all = int(nt.item())
    else:
        n_ok_all = n_ok
    e2e = {"value": round(n_ok_all * steps / te, 3), "unit": "solves/s",
           "h2d_bytes_per_step": int(vh.numel() * 8 + bh.numel() * 8), "d2h_bytes_per_step": int(xh.numel() * 8)}
    # plain FP64 drop-in (solve_linear_system, host CSR in, ndarray out) once per
    # system, over a bounded prefix of this rank's systems (rank 0 only)
    plain_d = None
    if rank == 0 and plain:
        from kcfd.fvm_operators import FVMSystem
        from kcfd.linear_solver import solve_linear_system
        host_sys = [(sparse.csr_matrix((vals[k].cpu().numpy(), pats[k][1], pats[k][0]),
                                       shape=(n_sys[k], n_sys[k])), rhs[k]) for k in range(len(mine))]
        solve_linear_system(FVMSystem.from_csr(*host_sys[0]), None, "bicgstab", 0.0, 20000, "b200", "jacobi",
                            rtol=1e-8)
        torch.cuda.synchronize()
        tp0 = time.perf_counter()
        done = 0
        for A, r in host_sys:
            solve_linear_system(FVMSystem.from_csr(A, r), None, "bicgstab", 0.0, 20000, "b200", "jacobi", rtol=1e-8)
            done += 1
            if time.perf_counter() - tp0 > plain_budget_s:
                break
        tp = time.perf_counter() - tp0
        frac = float(nnz_sys[:done].sum() / nnz_sys.sum())
        plain_d = {"value": round(len(mine) * frac / tp, 3) if done < len(mine) else round(done / tp, 3),
                   "unit": "solves/s", "systems_timed": done, "seconds": round(tp, 2),
                   "desc": "plain FP64 drop-in: kcfd solve_linear_system(backend='b200', bicgstab + jacobi, "
                           "rtol 1e-8) once per system, host CSR in / ndarray out"
                           + ("" if done == len(mine) else "; the timed prefix's rate weighted by its share of "
                              "the entries")}
    cpu_d = None
    if rank == 0 and world == 1 and cpu:
        import scipy.sparse.linalg as spla
        tc0 = time.perf_counter()
        done = 0
        for k in range(len(mine)):
            A = sparse.csr_matrix((vals[k].cpu().numpy(), pats[k][1], pats[k][0]), shape=(n_sys[k], n_sys[k]))
            d = A.diagonal()
            dinv = np.where(np.abs(d) > 1e-30, 1.0 / np.where(d == 0, 1.0, d), 0.0)
            M = spla.LinearOperator(A.shape, matvec=lambda y, dinv=dinv: dinv * y)
            spla.bicgstab(A, rhs[k], rtol=1e-8, atol=0.0, maxiter=20000, M=M)
            done += 1
            if time.perf_counter() - tc0 > 20.0:
                break
        tc = time.perf_counter() - tc0
        frac = float(nnz_sys[:done].sum() / nnz_sys.sum())
        cpu_d = {"value": round(len(mine) / (tc / frac), 4), "unit": "solves/s", "cores": 1, "kind": "port",
                 "sample": f"scipy bicgstab + Jacobi (the reference's create_preconditioner 'jacobi' path) on the "
                           f"first {done} systems ({tc:.1f} s, {100 * frac:.1f}% of the entries), weighted by "
                           f"entries to all {len(mine)}"}
    value = n_ok_all * steps / t
    return {"value": round(value, 3), "unit": "solves/s", "systems": int(count), "steps": steps, "warmup": warmup,
            "ms_per_step": round(1e3 * t / steps, 3), "mixed": mixed, "clocks": clocks, "e2e": e2e,
            "roofline": roof, "plain_fp64_dropin": plain_d, "cpu_baseline": cpu_d,
            "batched_over_plain": round(value / plain_d["value"], 2) if plain_d else None,
            "gpu_launches": (1 + sum(1 for k in ("cluster", "big", "small") if tiers[k] > 0)) * steps,
            "tiers": tiers, "status_ok": int((st == 0).sum()), "breakdown": int((st == 2).sum()),
            "converged": n_ok, "restarts_allowed": restarts, "max_true_relres": float(true_rel.max()),
            "krylov_iters": {"min": int(its.min()), "median": int(np.median(its)), "max": int(its.max())},
            "cells_this_rank": int(n_sys.sum()), "nnz_this_rank": int(nnz_sys.sum()),
            "generation_s": round(gen_s, 1),
            "desc": f"the first {count} of the 1,024 p' systems on Delaunay triangle meshes (n log-uniform in "
                    "[2e3, 2e5], seed 0), diffusion (harmonic, Gamma log-uniform [0.1, 10]) + one Dirichlet side, "
                    "RHS N(0,1); batched " + ("FP32 BiCGSTAB + Jacobi with FP64 refinement" if mixed else
                                              "FP64 BiCGSTAB + Jacobi") +
                    f", rtol 1e-8, breakdown restarts <= {restarts}, one persistent launch per size tier; value "
                    "counts converged systems only"}


def run_c4(args):
    """C4: 1,024 pressure-correction systems on Delaunay triangle meshes solved
    together (c4_measure). Multi-GPU: systems are spread over ranks by LPT on nnz, no
    data-path collective."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=900))
    r = c4_measure(count=args.systems, steps=args.steps, warmup=args.warmup, mode=args.c4_mode, plain=bool(args.plain),
                   cpu=not args.no_cpu, world=world, rank=rank)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": C4_METRIC, "value": r["value"], "unit": "solves/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None,
                "dtype": "fp32-inner/fp64-refine" if r["mixed"] else "f64", "data": "synthetic",
                "config": {"workload": r["desc"], "cells_this_rank": r["cells_this_rank"],
                           "nnz_this_rank": r["nnz_this_rank"],
                           "parallelism": f"LPT shards x{world}" if world > 1 else "1 GPU",
                           "l2": "working set >> 126 MB L2; no flush needed", "generation_s": r["generation_s"]}}
        for k in ("clocks", "e2e", "roofline", "cpu_baseline", "plain_fp64_dropin", "batched_over_plain",
                  "gpu_launches", "tiers", "status_ok", "breakdown", "converged", "restarts_allowed",
                  "max_true_relres", "krylov_iters"):
            line[k] = r[k]
        print(json.dumps(line))


C5_METRIC = "served SIMPLE cavities/s (Poisson arrivals, continuous batching)"


def c5_measure(requests=40, rate=20.0, cont_tol=1e-2, max_iters=1500, max_active=4, policy="sjf", serial=True,
               small_team=1):
    """Poisson-arriving cavity requests (half 2D N^2, N in [32, 512]; half 3D N^3, N in
    [16, 96]; Re in [100, 1000]; seed 0) served by the continuous-batching loop
    (kcfd.serve.Server: HBM-budget admission, one stream and graph per case), each run
    to a continuity residual ||b_p'|| / ||b_p'(first)|| below cont_tol; the comparator
    serves the same requests one case at a time."""
    import torch
    from kcfd.serve import Request, Server, make_requests, summarize
    reqs = make_requests(requests, rate, seed=0)
    common = dict(budget_bytes=150e9, iters_per_tick=10, max_iters=max_iters, cont_tol=cont_tol,
                  graph=True, precond_p="auto", keep_fields=True)
    # warm-up: one small case of each dimension (kernel loading, allocator)
    Server(precision="fp64", **common).run([Request(0, 2, 32, 400.0, 0.0), Request(1, 3, 16, 400.0, 0.0)])
    torch.cuda.synchronize()
    dev = torch.cuda.current_device()
    with ClockSampler(dev) as cs:
        res = Server(max_active=max_active, policy=policy, builders=2, precision="fp64", small_team=small_team,
                     **common).run(reqs)
    clocks = cs.summary()
    ours = summarize(res)
    d2h = int(sum(r.cells * (r.ndim + 1) * 8 for r in res))
    serial_d = None
    if serial:
        sres = Server(max_active=1, policy="fifo", precision="fp64", **common).run(reqs, serial=True)
        serial_d = summarize(sres)
        # the serial run takes the library's single-case solvers (the grid kernel for
        # small cases), the served run one CTA per small case: same algorithm, other
        # reduction partition, so the fields agree to the solver tolerance
        diffs = [float(np.linalg.norm(a.fields["U"] - b.fields["U"]) / max(np.linalg.norm(b.fields["U"]), 1e-300))
                 for a, b in zip(sorted(res, key=lambda r: r.rid), sorted(sres, key=lambda r: r.rid))]
        serial_d["max_rel_l2_U_vs_batched"] = max(diffs)
    return {"value": round(ours["cases_per_s"], 3), "unit": "cases/s", "requests": len(reqs), "rate": rate,
            "clocks": clocks, "p50_ms": round(ours["p50_ms"], 1), "p99_ms": round(ours["p99_ms"], 1),
            "converged": ours["converged"], "mean_iterations": ours["mean_iterations"],
            "d2h_bytes_per_case": int(d2h / max(len(res), 1)), "serial_comparator": serial_d,
            "served_over_serial": round(ours["cases_per_s"] / serial_d["cases_per_s"], 2) if serial_d else None,
            "desc": f"{len(reqs)} cavity requests at {rate} req/s (Poisson, seed 0): 2D N^2 N~U{{32..512}}, 3D N^3 "
                    f"N~U{{16..96}}, Re~U(100,1000); each to continuity {cont_tol:g} (max {max_iters} outer "
                    f"iterations); p' by the multigrid above 32,768 cells and ILU(0) below, HBM budget 150 GB; "
                    f"FP64; served: continuous batching (max {max_active} resident, {policy} admission, cases built "
                    f"on 2 host threads); serial comparator: one case at a time"}


def run_c5(args):
    r = c5_measure(args.requests, args.rate, args.cont_tol, args.max_iters, args.max_active, args.policy,
                   bool(args.plain), args.small_team)
    line = {
        "metric": C5_METRIC, "value": r["value"], "unit": "cases/s", "n_gpus": 1,
        "steps": r["requests"], "warmup": 2, "ms_per_step": round(1e3 / max(r["value"], 1e-9), 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": r["desc"], "parallelism": "1 GPU, continuous batching"},
        "clocks": r["clocks"], "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"],
        "converged": r["converged"], "mean_iterations": r["mean_iterations"],
        "e2e": {"value": r["value"], "unit": "cases/s", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": r["d2h_bytes_per_case"],
                "note": "the served loop is end to end already: host mesh arrays in, fields out per case"},
        "serial_comparator": r["serial_comparator"], "served_over_serial": r["served_over_serial"],
        "roofline": None, "cpu_baseline": None,
    }
    print(json.dumps(line))


C1_METRIC = "SIMPLE outer iterations/s (2D lid-driven cavity 64^2, Re 100, 500 outer iterations)"


def run_c1(args):
    """C1, the reference's own CPU-runnable case: 64^2 quad cavity (generate_cavity_mesh
    geometry), rho 1, mu 0.01, upwind, alpha_u 0.7, alpha_p 0.3, BiCGSTAB + Jacobi to
    rtol 1e-8 for momentum and p', exactly 500 outer iterations, one outer iteration
    captured as a CUDA graph. The oracle (same solver semantics) runs the same 500
    iterations on the host for the parity figure and the CPU baseline."""
    import torch
    from kcfd import mesh as km, meshgen
    from kcfd.simple import SIMPLESolver
    from oracle import mesh as om, simple as osim
    N, iters = 64, args.c1_iters
    nodes, cells, bd = meshgen.quad_box_arrays(0, 0, 1, 1, N, N, meshgen.CAVITY_2D_NAMES)
    m = km.build_mesh(nodes, cells, bd)

    def make():
        s = SIMPLESolver(m, rho=1.0, mu=0.01, precision="fp64", precond_p="jacobi", rtol=1e-8, maxiter=20000,
                         graph=True)
        for nm in m.boundary_patches:
            s.set_velocity_bc(nm, "dirichlet", [1.0, 0.0] if nm == "lid" else [0.0, 0.0])
            s.set_pressure_bc(nm, "zero_gradient")
        s.alpha_u, s.alpha_p, s.tol = 0.7, 0.3, 0.0
        s.reset_history()
        return s

    w = make()
    w.iterate(args.warmup)  # warm-up run (graph capture, kernel loading), then a fresh solver
    torch.cuda.synchronize()
    s = make()
    dev = torch.cuda.current_device()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as cs:
        e0.record()
        s.iterate(iters)
        e1.record()
        torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    clocks = cs.summary()
    U = s.U.values
    # e2e through the drop-in: solve_steady (host residual history read once), fields out
    s2 = make()
    s2.max_outer_iter = iters
    torch.cuda.synchronize()
    te0 = time.perf_counter()
    s2.solve_steady()
    U2 = s2.U.values
    te = time.perf_counter() - te0
    parity = cpu = None
    if not args.no_cpu:
        o = osim.Simple(om.build_2d(nodes, cells, bd), rho=1.0, mu=0.01)
        osim.cavity_setup(o)
        o.solver, o.rtol, o.precond_u, o.precond_p = "bicgstab", 1e-8, "jacobi", "jacobi"
        o.alpha_u, o.alpha_p, o.max_outer_iter, o.tol = 0.7, 0.3, iters, 0.0
        tc0 = time.perf_counter()
        o.solve_steady()
        tc = time.perf_counter() - tc0
        parity = float(np.linalg.norm(U - o.U) / np.linalg.norm(o.U))
        cpu = {"value": round(iters / tc, 3), "unit": "iters/s", "cores": 1, "kind": "port",
               "sample": f"the oracle (numpy/scipy restatement, bicgstab + Jacobi) on the full workload: "
                         f"{iters} outer iterations in {tc:.1f} s"}
    line = {
        "metric": C1_METRIC, "value": round(iters / t, 2), "unit": "iters/s", "n_gpus": 1, "steps": iters,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t / iters, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "2D lid-driven cavity 64^2 quads, rho 1, mu 0.01, upwind, alpha_u 0.7, alpha_p 0.3, "
                               "BiCGSTAB + Jacobi rtol 1e-8, 500 outer iterations, CUDA graph per iteration",
                   "cells": int(m.n_cells), "parallelism": "1 GPU",
                   "l2": "small case: the working set stays in L2 (no flush; latency-bound)"},
        "clocks": clocks,
        "e2e": {"value": round(iters / te, 2), "unit": "iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(U2.nbytes / iters),
                "note": "solve_steady through the drop-in: residual history and U read back once"},
        "cpu_baseline": cpu, "roofline": None, "parity_U_rel_l2_vs_oracle": parity,
    }
    print(json.dumps(line))


C3_METRIC = "two-fluid time steps/s (Delaunay tets, 10 SIMPLE inner iterations per step, 6-equation energy)"


def c3_solver(n_target, seed=0, oracle=False, p_precond="amg", precision="fp64", arrays=None):
    """The two-fluid workload: a 0.2 x 0.2 x 1.0 m box of Delaunay tetrahedra
    (jittered lattice, ~n_target cells), bottom 'inlet_gas', top 'outlet', 'wall'
    elsewhere; water / air (rho 998 / 1.2, mu 1e-3 / 1.8e-5, cp_l 4182), d_b = 3 mm,
    Lee rate 0.1 1/s, T_sat 373.15 K; inlet superficial gas velocity 0.01 m/s at
    alpha_in = 0.05 (u_g = 0.2 m/s); alpha_g ~ U(0.02, 0.08), T_l = T_g = 370 + U(0, 6) K;
    dt = 1e-3, 10 inner iterations, energy on. oracle=True builds the numpy oracle.
    arrays: the (nodes, cells, cf, bd) of an earlier call with the same n_target and seed
    (the mesh is not generated again; the initial fields are the same draws)."""
    from kcfd import meshgen
    rng = np.random.default_rng(seed)
    if arrays is None:
        arrays = meshgen.delaunay_tet_arrays((0.2, 0.2, 1.0), n_target, rng)
    else:
        rng.integers(0, 2**31)   # the generator's one draw (its jitter seed)
    nodes, cells, cf, bd = arrays
    if oracle:
        from oracle import mesh as om
        from oracle.two_fluid import TwoFluid
        m = om.build_3d(nodes, cells, cf, bd)
        sv = TwoFluid(m)
        setf = lambda k, v: sv.v.__setitem__(k, np.array(v, dtype=np.float64))  # noqa: E731
    else:
        from kcfd import mesh as km
        from kcfd.two_fluid import TwoFluidSolver
        m = km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
        sv = TwoFluidSolver(m, p_precond=p_precond, precision=precision)
        setf = lambda k, v: setattr(getattr(sv, k), "values", v)  # noqa: E731
    sv.rho_l, sv.mu_l, sv.cp_l = 998.0, 1e-3, 4182.0
    sv.rho_g, sv.mu_g = 1.2, 1.8e-5
    sv.d_b, sv.r_phase_change, sv.T_sat = 0.003, 0.1, 373.15
    sv.solve_energy, sv.max_outer_iter, sv.tol, sv.dt = True, 10, 1e-12, 1e-3
    sv.initialize(0.05)
    sv.set_inlet_bc("inlet_gas", 0.05, U_l=[0.0, 0.0, 0.0], U_g=[0.0, 0.0, 0.01 / 0.05], T_l=372.0, T_g=373.15)
    sv.set_outlet_bc("outlet", 0.0)
    sv.set_wall_bc("wall")
    n = len(cells)
    ag = rng.uniform(0.02, 0.08, n)
    T = 370.0 + rng.uniform(0.0, 6.0, n)
    setf("alpha_g", ag)
    setf("alpha_l", 1.0 - ag)
    setf("T_l", T)
    setf("T_g", T.copy())
    sv._arrays = arrays
    return sv, m


def _c3_tensors(sv):
    """Every device tensor of a TwoFluidSolver that carries state between steps."""
    import torch
    out = {}
    for name, v in vars(sv).items():
        if isinstance(v, torch.Tensor):
            out[name] = v
        elif isinstance(v, dict):
            for k, t in v.items():
                if isinstance(t, torch.Tensor):
                    out[f"{name}.{k}"] = t
    return out


def run_c3(args):
    """C3: the two-fluid system set on ~1 M Delaunay tets (one GPU; a single mesh is
    not sharded, so N > 1 would run replicas). The reference model diverges on this
    workload within a few steps, and solves on non-finite fields end at once, so every
    timed pass starts from the initial state (restored after the warm-up) and only
    the steps whose fields are still finite are counted, each timed on its own."""
    import torch
    t0 = time.time()
    sv, m = c3_solver(args.tets, p_precond=args.p_precond)
    arrays = sv._arrays
    setup_s = time.time() - t0
    state0 = {k: t.clone() for k, t in _c3_tensors(sv).items()}

    def restore():
        cur = _c3_tensors(sv)
        for k, t in state0.items():
            if k in cur:
                cur[k].copy_(t)

    for _ in range(args.warmup):
        sv.step()
    torch.cuda.synchronize()
    restore()
    torch.cuda.synchronize()
    dev = torch.cuda.current_device()
    res, evs, fin, kry = [], [], [], [sv.krylov.clone()]
    with ClockSampler(dev) as cs:
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            res.append(sv.step())
            b.record()
            evs.append((a, b))
            kry.append(sv.krylov.clone())
            fin.append(torch.stack([torch.isfinite(t).all() for t in sv._f.values()]).all())
        torch.cuda.synchronize()
    clocks = cs.summary()
    fin = [bool(f) for f in fin]
    n_ok = fin.index(False) if False in fin else len(fin)
    t = sum(a.elapsed_time(b) for a, b in evs[:n_ok]) / 1e3
    umax = float(max(sv._f["U_l"].abs().max(), sv._f["U_g"].abs().max()))
    # roofline of the solves (80 per step, the dominant work): BiCGSTAB + ILU(0)
    # formula bytes at each step's Krylov counts (one-rhs and 3-rhs solves)
    roof = None
    if n_ok:
        k = [v.cpu().numpy() for v in kry[: n_ok + 1]]
        it1, itg, itp = (int(k[-1][j] - k[0][j]) for j in range(3))
        nnz = int(m.nnz)
        amg = amg_levels(sv._sp) if args.p_precond == "amg" else None
        byts = solver_bytes(m.n_cells, nnz, it1, "ilu0", 8) + solver_bytes(m.n_cells, nnz, itg, "ilu0", 8, nrhs=3)
        if amg:
            byts += solver_bytes(m.n_cells, nnz, itp, "amg", 8, amg=amg)
        peak = measured_peak()
        roof = {"bound": "hbm", "kernel": "graph engine BiCGSTAB solves (all 80 systems of a step: ILU(0), and the "
                                          "multigrid for p')",
                "unit_of_work": "the solves of the counted steps (formula bytes x Krylov iterations)",
                "krylov_iters": {"one_rhs_ilu0": it1, "three_rhs_ilu0": itg, "p_multigrid": itp},
                "achieved": round(byts / t / 1e9, 1), "peak": peak[0], "unit": "GB/s",
                "frac": round(byts / t / 1e9 / peak[0], 3), "peak_source": peak[1], "traffic": None,
                "note": "the time is the whole step (assembly, closures and set-up included), so this is a "
                        "lower bound on the solves' own fraction"}
    # e2e: every step the fields come in from host arrays and go back out
    names = ("alpha_g", "alpha_l", "U_l", "U_g", "p", "T_l", "T_g")
    restore()
    host = {k: getattr(sv, k).values for k in names}
    nbytes = sum(v.nbytes for v in host.values())
    torch.cuda.synchronize()
    te, ne = 0.0, 0
    for _ in range(args.steps):
        te0 = time.perf_counter()
        for k in names:
            getattr(sv, k).values = host[k]
        sv.step()
        host = {k: getattr(sv, k).values for k in names}
        dt_e = time.perf_counter() - te0
        if not all(np.isfinite(v).all() for v in host.values()):
            break
        te += dt_e
        ne += 1
    # the mixed form (the multigrid p' hierarchy in FP32) from the same initial state,
    # its fields after the same finite steps against FP64's
    mixed = None
    if args.plain and args.p_precond == "amg" and n_ok:
        # the steps before the model's divergence shows (residual below 1e3): past it
        # both runs' fields grow without bound and their difference says nothing
        ncmp = max(1, next((i for i, r in enumerate(res[:n_ok]) if not (float(r) < 1e3)), n_ok))
        restore()
        for _ in range(ncmp):
            sv.step()
        ref = {k: getattr(sv, k).values for k in ("alpha_g", "U_l", "U_g", "p", "T_l", "T_g")}
        del sv
        torch.cuda.empty_cache()
        sm, _ = c3_solver(args.tets, p_precond="amg", precision="mixed", arrays=arrays)
        cur = _c3_tensors(sm)
        for k2, t2 in state0.items():
            if k2 in cur and cur[k2].shape == t2.shape:
                cur[k2].copy_(t2)
        torch.cuda.synchronize()
        tm0 = time.perf_counter()
        for _ in range(ncmp):
            sm.step()
        torch.cuda.synchronize()
        tm = time.perf_counter() - tm0
        errs = {k2: float(np.linalg.norm(getattr(sm, k2).values - v) / max(np.linalg.norm(v), 1e-300))
                for k2, v in ref.items()}
        t64 = sum(a.elapsed_time(b) for a, b in evs[:ncmp]) / 1e3
        mixed = {"value": round(ncmp / tm, 4), "unit": "steps/s", "steps": ncmp, "field_error": errs,
                 "fp64_same_steps": round(ncmp / t64, 4) if t64 > 0 else None,
                 "desc": "the same workload in the mixed form: the momentum, volume-fraction and energy systems "
                         "(ILU(0)) on the graph engine's FP32 form (FP32 vectors and values, FP64 iterate, residual "
                         "replacement against the FP64 matrix, the same 1e-12 FP64 stopping test), the multigrid p' "
                         "hierarchy stored in FP32 under an FP64 Krylov iteration; wall time of the steps with a "
                         "device synchronize on both sides; field_error = relative L2 against the FP64 run after "
                         "the same steps from the same initial state (alpha_g, U_l, U_g, p, T_l, T_g), over the "
                         "steps before the model's residual passes 1e3"}
    cpu = None
    if not args.no_cpu:
        so, mo = c3_solver(args.cpu_tets, oracle=True)
        so.step()  # warm-up
        tc0 = time.perf_counter()
        so.step()
        tc = time.perf_counter() - tc0
        scale = m.n_cells / mo.n_cells
        cpu = {"value": round(1.0 / (tc * scale), 6), "unit": "steps/s", "cores": 1, "kind": "port",
               "sample": f"the oracle (numpy + scipy spsolve, as the reference's method='direct') on the same "
                         f"workload at {mo.n_cells} tets: one step {tc:.2f} s, scaled linearly by cells "
                         f"(x{scale:.1f}); the direct solves grow faster than linearly, so this favours the CPU"}
    line = {
        "metric": C3_METRIC, "value": round(n_ok / t, 4) if n_ok else None, "unit": "steps/s", "n_gpus": 1,
        "steps": n_ok, "steps_run": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t / n_ok, 2) if n_ok else None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"two-fluid bubble column, {m.n_cells} Delaunay tets in 0.2x0.2x1.0 m, water/air, "
                               "d_b 3 mm, Lee phase change, dt 1e-3, 10 inner SIMPLE iterations per step, energy on; "
                               "every system BiCGSTAB to 1e-12: ILU(0), and for p' "
                               + ("the multigrid" if args.p_precond == "amg" else "ILU(0)"),
                   "cells": int(m.n_cells), "faces": int(m.n_faces), "setup_s": round(setup_s, 1),
                   "parallelism": "1 GPU", "l2": "working set >> 126 MB L2; no flush needed"},
        "clocks": clocks,
        "e2e": {"value": round(ne / te, 4) if ne else None, "unit": "steps/s", "h2d_bytes_per_step": int(nbytes),
                "d2h_bytes_per_step": int(nbytes), "steps": ne},
        "cpu_baseline": cpu, "roofline": roof, "mixed_precision_variant": mixed,
        "finite_steps": n_ok, "max_residual_per_step": [float(r) for r in res],
        "max_abs_velocity_after_all_steps": umax,
        "note": "the reference two-fluid model diverges on this workload within a few steps (its numpy "
                "restatement, run with spsolve, reaches |U| ~ 1e11 by step 2); both legs start from the initial "
                "state and count only the steps whose fields are still finite (value = those steps / their "
                "summed device time)",
    }
    print(json.dumps(line))




def oracle_cavity(N):
    """The oracle on the same workload: BiCGSTAB + Jacobi for u, v, w and BiCGSTAB +
    structural ILU(0) in the greedy (red-black) cell colouring for p' -- the device's
    ILU(0) ordering; the reference's own 'ilu0' (SuperLU spilu, COLAMD) needs about
    twice the Krylov iterations on these systems -- each to rtol 1e-8."""
    from oracle import mesh as om, simple as osim
    nodes, cells, cf, bd = cavity_arrays(N)
    m = om.build_3d(nodes, cells, cf, bd)
    o = osim.Simple(m, rho=1.0, mu=0.0025)
    osim.cavity_setup(o)
    o.muscl, o.nonorth = "van_leer", True
    o.solver, o.rtol, o.precond_u, o.precond_p = "bicgstab", 1e-8, "jacobi", "ilu0"
    o.alpha_u, o.alpha_p = 0.7, 0.3
    return o


def cpu_outer_iterations(N, max_steps, budget_s):
    """Whole outer iterations of the N^3 workload by the oracle from the initial state,
    timed one by one; stops after max_steps or when another step would take the timed
    work past budget_s (at least one step). The mesh build and the ILU(0) colouring
    (pattern only) are set-up, not timed; an 8^3 copy runs one iteration first."""
    from oracle import linsolve, mesh as om
    w = oracle_cavity(8)
    w.iterate()
    t0 = time.time()
    o = oracle_cavity(N)
    ip, ix = om.csr_pattern(o.mesh)
    from scipy import sparse
    o._colour = linsolve.greedy_colouring(sparse.csr_matrix((np.ones(len(ix)), ix, ip), shape=(len(ip) - 1,) * 2))
    build_s = time.time() - t0
    steps = []
    while len(steps) < max_steps:
        ts = time.perf_counter()
        o.iterate()
        dt = time.perf_counter() - ts
        log = dict(o.iters_log[-4:])
        steps.append({"s": dt, "p_krylov": int(log.get("p", 0)), "mom_krylov": [int(log.get(f"u{c}", 0)) for c in range(3)]})
        if sum(x["s"] for x in steps) + dt > budget_s:
            break
    return {"N": N, "build_s": build_s, "steps": steps, "host_cores": os.cpu_count(),
            "colours": int(o._colour.max()) + 1}


def run_cpu_sample(args):
    print(json.dumps(cpu_outer_iterations(args.size, max_steps=1, budget_s=0.0)))


def run_reference(args):
    """The reference's path on the host cores: the oracle on the full workload, whole
    outer iterations (as many of the requested steps as fit REF_BUDGET_S of timed
    work, at least one), measured one by one; nothing is scaled."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    N = args.size
    r = cpu_outer_iterations(N, max_steps=args.steps, budget_s=REF_BUDGET_S)
    cb = cpu_baseline_entry(r)
    t = 1.0 / cb["value"]
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": 1,
            "steps": len(r["steps"]), "steps_requested": args.steps, "warmup": 1,
            "ms_per_step": round(1e3 * t, 1), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"3D jittered lid-driven cavity {N}^3 hex ({N**3} cells), Re 400, MUSCL van Leer, "
                                   "over-relaxed non-orthogonal, BiCGSTAB + ILU(0) (red-black) p' / Jacobi u,v,w, "
                                   "rtol 1e-8, FP64, the oracle (numpy/scipy) on the host cores",
                       "cells": N ** 3, "warmup_note": "one outer iteration of an 8^3 copy of the workload",
                       "setup_s": round(r["build_s"], 1), "ilu0_colours": r["colours"]},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "cpu-sample"])
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--p-precond", default="amg", choices=["amg", "ilu0"], help="c2: p' preconditioner")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: 128^3 cavity SIMPLE (default); c3: two-fluid on ~1M tets; c4: 1,024 batched p' "
                         "systems; c5: served cavities")
    ap.add_argument("--legs", default="c4,c5", help="c2: bounded C4 / C5 legs in the same line ('' for none)")
    ap.add_argument("--leg-systems", type=int, default=128, help="c2: C4 leg systems (the first of the 1,024)")
    ap.add_argument("--leg-requests", type=int, default=12, help="c2: C5 leg requests")
    ap.add_argument("--tets", type=int, default=1000000, help="c3: target tetrahedra")
    ap.add_argument("--c1-iters", type=int, default=500, help="c1: outer iterations")
    ap.add_argument("--cpu-tets", type=int, default=6000, help="c3: oracle sample size")
    ap.add_argument("--requests", type=int, default=40, help="c5: number of requests")
    ap.add_argument("--rate", type=float, default=20.0, help="c5: arrival rate (req/s)")
    ap.add_argument("--cont-tol", type=float, default=1e-2, help="c5: continuity residual to serve to")
    ap.add_argument("--max-iters", type=int, default=1500, help="c5: outer iteration cap per case")
    ap.add_argument("--max-active", type=int, default=4, help="c5: resident cases at most")
    ap.add_argument("--small-team", type=int, default=1, help="c5: solver team of the served small cases (1 or 0)")
    ap.add_argument("--policy", default="sjf", choices=["sjf", "fifo"], help="c5: admission order")
    ap.add_argument("--systems", type=int, default=1024, help="c4: number of systems")
    ap.add_argument("--c4-mode", default="fp64", choices=["fp64", "mixed"], help="c4: batched solve precision")
    ap.add_argument("--plain", type=int, default=1, help="also time the variants (rank 0)")
    ap.add_argument("--iterate-only", type=int, default=0,
                    help="c2: run this many outer iterations from the initial state and exit (for profilers)")
    ap.add_argument("--mixed", action="store_true", help="c2 with --iterate-only: the mixed form")
    args = ap.parse_args()
    args.legs = [x for x in args.legs.split(",") if x]
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.impl == "cpu-sample":
        run_cpu_sample(args)
    elif args.config == "c1":
        run_c1(args)
    elif args.config == "c3":
        run_c3(args)
    elif args.config == "c4":
        run_c4(args)
    elif args.config == "c5":
        run_c5(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
