"""Batched solves: many independent systems of uneven size in one persistent launch.

BatchSolver packs the systems' CSR (local row pointers and column indices per system,
concatenated) once and then solves all of them in one launch of the batched kernel
(libkcfd kcfd_batch_*): each CTA takes the next system from a largest-first queue and
solves it alone, so a system's result is the same whatever runs beside it.

The pressure-correction batch of the benchmark configs is built here too:
p_prime_batch() makes Delaunay triangle meshes with cell counts log-uniform in
[n_min, n_max], per-cell diffusivity log-uniform in [0.1, 10], one Dirichlet
segment and a N(0, 1) right-hand side, assembled on the device with the generic
operators (kcfd.assembly).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class BatchOpts(C.Structure):
    _fields_ = [("precond", C.c_int32), ("stop", C.c_int32), ("mode", C.c_int32), ("maxiter", C.c_int32),
                ("lanes", C.c_int32), ("max_refine", C.c_int32), ("inner_maxiter", C.c_int32), ("big_rows", C.c_int32),
                ("cluster_rows", C.c_int32), ("cluster_size", C.c_int32),
                ("rtol", C.c_double), ("atol", C.c_double), ("inner_rtol", C.c_double), ("restarts", C.c_int32)]


class BatchSolver:
    """patterns: list of (indptr, indices) host arrays (one per system).

    Tiers by system size. Cluster teams (one thread-block cluster per system):
    graded with cluster_size 0 -- 8, 4 or 2 CTAs from 8R, 4R or 2R rows, R =
    cluster_rows (0: 16384) -- or one tier of cluster_size CTAs from cluster_rows rows
    (0: 131072); negative cluster_rows: none. Then at least big_rows rows (0: 16384,
    negative: none) by one 512-thread CTA; the rest by one 256-thread CTA. tiers()
    reports the split (cluster_size: the largest team).

    restarts: with the scipy stopping rule, a system whose rho or omega breaks down
    restarts from its current iterate (rhat = r, p = r) up to this many times (0: it
    stops with BREAKDOWN, as scipy's bicgstab does)."""

    def __init__(self, patterns, mode="mixed", precond="jacobi", rtol=1e-8, atol=0.0, maxiter=20000, lanes=1,
                 inner_rtol=1e-3, inner_maxiter=400, max_refine=60, stop=_lib.STOP_SCIPY, big_rows=0,
                 cluster_rows=0, cluster_size=0, restarts=20, device="cuda"):
        torch = _lib.require_cuda()
        self.nsys = len(patterns)
        self.n = np.array([len(ip) - 1 for ip, _ in patterns], dtype=np.int32)
        self.nnz = np.array([len(ix) for _, ix in patterns], dtype=np.int32)
        ip = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.int32) for p, _ in patterns]))
        ix = np.ascontiguousarray(np.concatenate([np.asarray(i, dtype=np.int32) for _, i in patterns]))
        self.row_off = np.concatenate([[0], np.cumsum(self.n.astype(np.int64))])
        self.nnz_off = np.concatenate([[0], np.cumsum(self.nnz.astype(np.int64))])
        o = BatchOpts()
        o.precond = _lib.PREC[precond]
        o.stop = stop
        o.mode = _lib.MODE_MIXED if mode == "mixed" else _lib.MODE_FP64
        o.maxiter, o.lanes, o.max_refine, o.inner_maxiter = int(maxiter), int(lanes), int(max_refine), int(inner_maxiter)
        o.rtol, o.atol, o.inner_rtol = float(rtol), float(atol), float(inner_rtol)
        o.big_rows = int(big_rows)
        o.cluster_rows, o.cluster_size = int(cluster_rows), int(cluster_size)
        o.restarts = int(restarts)
        h = C.c_void_p()
        _lib.check(_lib.lib().kcfd_batch_create(self.nsys, self.n.ctypes.data, self.nnz.ctypes.data, ip.ctypes.data,
                                                ix.ctypes.data, C.byref(o), C.byref(h)), "kcfd_batch_create")
        self._h = h
        info = np.zeros(4, dtype=np.int64)
        _lib.check(_lib.lib().kcfd_batch_info(h, info.ctypes.data_as(_lib.P_i64)), "kcfd_batch_info")
        self.n_total, self.nnz_total, self.ctas = int(info[1]), int(info[2]), int(info[3])
        dev = device
        self.iters = torch.zeros(self.nsys, dtype=torch.int32, device=dev)
        self.relres = torch.zeros(self.nsys, dtype=torch.float64, device=dev)
        self.status = torch.zeros(self.nsys, dtype=torch.int32, device=dev)

    def tiers(self):
        """dict(cluster, big, small, clusters, cluster_size): systems per tier, clusters launched."""
        v = np.zeros(5, dtype=np.int32)
        _lib.check(_lib.lib().kcfd_batch_tiers(self._h, v.ctypes.data_as(_lib.P_i32)), "kcfd_batch_tiers")
        return dict(zip(("cluster", "big", "small", "clusters", "cluster_size"), (int(t) for t in v)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.release("kcfd_batch_destroy", h)
            except Exception:   # interpreter shutdown: the module may be gone already
                pass
            self._h = None

    def solve(self, vals64, rhs, x, stream=None):
        """Packed device arrays; x holds x0 on entry. One kernel launch."""
        _lib.check(_lib.lib().kcfd_batch_solve(self._h, _lib.ptr(vals64), _lib.ptr(rhs), _lib.ptr(x),
                                               _lib.ptr(self.iters), _lib.ptr(self.relres), _lib.ptr(self.status),
                                               _lib.stream_handle(stream)), "kcfd_batch_solve")
        return self.iters, self.relres, self.status

    def pack(self, arrays, what="rows"):
        """List of per-system host arrays -> one packed device tensor."""
        torch = _lib.require_cuda()
        return torch.from_numpy(np.ascontiguousarray(np.concatenate([np.asarray(a, dtype=np.float64)
                                                                     for a in arrays]))).cuda()

    def unpack(self, t):
        v = t.detach().cpu().numpy()
        return [v[self.row_off[s]:self.row_off[s + 1]] for s in range(self.nsys)]


def plan_teams(sizes, sm_count=148, cluster_rows=0, cluster_size=0, big_rows=0):
    """The team each system of a batch of these row counts gets (kcfd_batch_plan, host
    only): CTAs of its thread-block cluster (2, 4, 8), 1 for one 512-thread CTA, 0 for one
    256-thread CTA."""
    n = np.ascontiguousarray(sizes, dtype=np.int32)
    o = BatchOpts()
    o.cluster_rows, o.cluster_size, o.big_rows = int(cluster_rows), int(cluster_size), int(big_rows)
    team = np.zeros(len(n), dtype=np.int32)
    _lib.check(_lib.lib().kcfd_batch_plan(len(n), n.ctypes.data, C.byref(o), int(sm_count), team.ctypes.data),
               "kcfd_batch_plan")
    return team


def lpt_shards(weights, nranks):
    """Greedy longest-processing-time assignment of systems to ranks (largest first,
    each to the currently lightest rank). Returns a list of index lists."""
    order = np.argsort(-np.asarray(weights), kind="stable")
    load = np.zeros(nranks)
    out = [[] for _ in range(nranks)]
    for i in order:
        r = int(np.argmin(load))
        out[r].append(int(i))
        load[r] += weights[i]
    return [sorted(o) for o in out]


def _p_prime_host(k, n_k, seed):
    """Host part of system k: Delaunay triangles of ~n_k/2 points, per-cell
    diffusivity and right-hand side, all from its own generator (seed, k), so the
    systems do not depend on how many processes make them. Each side of the square
    carries sqrt(n_k/2) equally spaced points, so the Dirichlet side (x = 0) is a
    chain of faces of the local mesh size rather than one edge under a sliver."""
    from .meshgen import delaunay_tri_arrays
    rng = np.random.default_rng((seed, k))
    npts = max(int(n_k) // 2, 4)
    pts, cells, bd = delaunay_tri_arrays(npts, rng, side_points=int(np.ceil(np.sqrt(npts))))
    n_cells = len(cells)
    gamma = np.exp(rng.uniform(np.log(0.1), np.log(10.0), n_cells))
    rhs = rng.normal(size=n_cells)
    return pts, cells, bd, gamma, rhs


def p_prime_sizes(count, n_min=2000, n_max=200000, seed=0):
    """Requested cell counts, log-uniform in [n_min, n_max]."""
    rng = np.random.default_rng(seed)
    return np.round(np.exp(rng.uniform(np.log(n_min), np.log(n_max), count))).astype(np.int64)


def p_prime_host(count, n_min=2000, n_max=200000, seed=0, workers=0):
    """Host inputs of the batch (list of (pts, cells, bd, gamma, rhs)); workers > 0
    makes them in a pool of spawned processes (Delaunay dominates: ~16 us a point)."""
    sizes = p_prime_sizes(count, n_min, n_max, seed)
    if workers and workers > 1 and count > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_p_prime_host, range(count), sizes, [seed] * count, chunksize=4)), sizes
    return [_p_prime_host(k, sizes[k], seed) for k in range(count)], sizes


def p_prime_batch(count, n_min=2000, n_max=200000, seed=0, device="cuda", workers=0, host=None):
    """Pressure-correction systems on Delaunay triangle meshes, assembled on the device.

    Returns (patterns, vals_list [device], rhs_list [host], sizes). Cell counts are
    log-uniform in [n_min, n_max]; each mesh triangulates ~n/2 uniform points plus the
    unit square's corners and sqrt(n/2) points on each side; the 'dirichlet' side
    (x = 0) has p' = 0, the other hull edges are zero-gradient. The diffusivity is log-uniform in [0.1, 10] per
    cell, the right-hand side N(0, 1). `host` takes the output of p_prime_host.
    """
    torch = _lib.require_cuda()
    from .assembly import DeviceSystem, boundary_arrays
    from .device_mesh import DeviceMesh
    from .mesh import build_mesh
    if host is None:
        host, sizes = p_prime_host(count, n_min, n_max, seed, workers)
    else:
        sizes = p_prime_sizes(count, n_min, n_max, seed)
    patterns, vals, rhs = [], [], []
    for pts, cells, bd, gamma_h, rhs_h in host:
        m = build_mesh(pts, cells, bd)
        dm = DeviceMesh(m, device)
        gamma = torch.from_numpy(gamma_h).to(device)
        s = DeviceSystem(dm)
        s.diffusion_operator(gamma)
        mf = torch.zeros(m.n_faces, dtype=torch.float64, device=device)
        bt, bv, bg = boundary_arrays(dm, {"dirichlet": {"type": "dirichlet"}, "wall": {"type": "zero_gradient"}}, {})
        s.apply_boundary_conditions(bt, bv, bg, gamma, mf)
        patterns.append((m.indptr, m.indices))
        vals.append(s.vals)
        rhs.append(rhs_h)
    return patterns, vals, rhs, sizes
