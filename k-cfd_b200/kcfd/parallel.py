"""Single-mesh partitioning, halo exchange and a distributed BiCGSTAB over torch.distributed.

Public API as in the reference (parallel/partitioning.py:11-143):

- GeometricPartitioner(mesh).partition(n_parts): recursive coordinate bisection of
  the cell centres. At depth d the cells are split on axis d % ndim at the median
  (np.median; cells with coordinate <= median go left, at least one cell each side),
  the left half taking n_parts // 2 parts and the right half the rest
  (partitioning.py:20-79). Part ids are the reference's, bit for bit.
- GhostCellLayer(mesh, part_ids): for every rank, the cells of each other rank that
  share an internal face with it, sorted (partitioning.py:82-143); get_local_cells,
  get_ghost_cells.

Beyond the reference (which exchanges ghosts with mpi4py point-to-point messages,
parallel/mpi_solver.py:56-103):

- HaloPlan(indptr, indices, part_ids, rank): the rank's rows (its cells, ascending), its
  ghost columns (ordered by owning rank, then cell id), the local CSR with columns
  renumbered to [own rows | ghosts], and per peer the rows it sends and the ghost
  slots it receives.
- HaloExchange(plan, group): fills the ghost part of an extended vector from the
  peers' rows with one all_to_all_single per exchange (NCCL on GPUs, gloo on CPU);
  each rank packs its send rows with index_select.
- DistributedBiCGSTAB: scipy's BiCGSTAB loop with Jacobi (the reference's
  preconditioner 'jacobi') or block-Jacobi ILU(0), the dot products all_reduced over
  the group, one halo exchange before each local SpMV. The local SpMV is the device
  kernel (kcfd_spmv_f64 on the extended local CSR); a caller may pass another operator.

A partitioned solve needs one exchange per SpMV and three all_reduces per iteration:
the dot products that do not depend on one another are reduced together as one short
vector, (||r||, rt.r), (rt.v) and (||s||, t.s, t.t). Ranks take the same collective
steps in the same order.
"""
from __future__ import annotations

import numpy as np


def _centres(mesh):
    c = getattr(mesh, "ccenter", None)
    if c is not None:
        return np.asarray(c, dtype=np.float64)
    return np.array([cell.center for cell in mesh.cells], dtype=np.float64)


def _internal_faces(mesh):
    """(owner, neighbour) of the internal faces."""
    own = getattr(mesh, "owner", None)
    if own is not None and not callable(own):
        own = np.asarray(mesh.owner)
        nb = np.asarray(mesh.neighbour)
    else:
        own = np.array([f.owner for f in mesh.faces])
        nb = np.array([f.neighbour for f in mesh.faces])
    keep = nb >= 0
    return own[keep], nb[keep]


def _row_entries(indptr, rows):
    """Positions of the CSR entries of the given rows, row after row."""
    lens = indptr[rows + 1] - indptr[rows]
    if not len(rows):
        return np.zeros(0, np.int64), lens
    first = np.repeat(indptr[rows] - (np.cumsum(lens) - lens), lens)
    return first + np.arange(int(lens.sum())), lens


class GeometricPartitioner:
    """Recursive coordinate bisection (parallel/partitioning.py:11-79)."""

    def __init__(self, mesh):
        self.mesh = mesh

    def partition(self, n_parts: int) -> np.ndarray:
        ndim = getattr(self.mesh, "ndim", 2)
        centres = _centres(self.mesh)[:, :ndim]
        n = len(centres)
        part_ids = np.zeros(n, dtype=int)
        self._split(centres, np.arange(n), part_ids, 0, int(n_parts), 0, ndim)
        return part_ids

    def _split(self, centres, cells, part_ids, first, n_parts, depth, ndim):
        if n_parts <= 1 or len(cells) == 0:
            part_ids[cells] = first
            return
        coords = centres[cells, depth % ndim]
        left = coords <= np.median(coords)
        if not left.any():
            left[0] = True
        if left.all():
            left[-1] = False
        n_left = n_parts // 2
        self._split(centres, cells[left], part_ids, first, n_left, depth + 1, ndim)
        self._split(centres, cells[~left], part_ids, first + n_left, n_parts - n_left, depth + 1, ndim)


class GhostCellLayer:
    """Ghost cells of each partition (parallel/partitioning.py:82-143)."""

    def __init__(self, mesh, part_ids):
        self.mesh = mesh
        self.part_ids = np.asarray(part_ids)
        self.n_parts = int(self.part_ids.max()) + 1
        self.ghost_map = {r: {} for r in range(self.n_parts)}
        own, nb = _internal_faces(mesh)
        po, pn = self.part_ids[own], self.part_ids[nb]
        cut = po != pn
        # in the owner's partition the neighbour is a ghost, and the other way round
        for me, other, cell in ((po[cut], pn[cut], nb[cut]), (pn[cut], po[cut], own[cut])):
            for r in np.unique(me):
                sel = me == r
                for q in np.unique(other[sel]):
                    cells = set(int(c) for c in cell[sel & (other == q)])
                    prev = self.ghost_map[int(r)].get(int(q), [])
                    self.ghost_map[int(r)][int(q)] = sorted(set(prev) | cells)
        self.send_map = {r: {} for r in range(self.n_parts)}
        self.recv_map = {r: {} for r in range(self.n_parts)}

    def get_local_cells(self, rank: int) -> np.ndarray:
        return np.where(self.part_ids == rank)[0]

    def get_ghost_cells(self, rank: int) -> dict:
        return self.ghost_map.get(rank, {})


class HaloPlan:
    """One rank's share of a partitioned system.

    indptr/indices: the global CSR pattern (host arrays). rows: this rank's rows
    (ascending); ghosts: the other ranks' rows its rows reference, ordered by owner
    then id; local_indptr/local_indices: its rows with columns renumbered to
    [0, n_own) for its rows and n_own + k for ghost k; send[q]: its rows that rank q
    needs (positions in rows, ascending by row id); recv[q]: slice of the ghost block
    that rank q fills."""

    def __init__(self, indptr, indices, part_ids, rank):
        indptr = np.asarray(indptr, dtype=np.int64)
        indices = np.asarray(indices, dtype=np.int64)
        part = np.asarray(part_ids)
        self.rank, self.n_ranks = int(rank), int(part.max()) + 1
        rows = np.flatnonzero(part == rank)
        self.rows = rows
        n = len(part)
        local_of = -np.ones(n, dtype=np.int64)
        local_of[rows] = np.arange(len(rows))
        take, lens = _row_entries(indptr, rows)
        cols = indices[take]
        self.src = take  # positions of this rank's entries in the global value array
        remote = np.unique(cols[part[cols] != rank])
        order = np.lexsort((remote, part[remote]))
        ghosts = remote[order]
        self.ghosts = ghosts
        ghost_of = -np.ones(n, dtype=np.int64)
        ghost_of[ghosts] = len(rows) + np.arange(len(ghosts))
        self.local_indptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        self.local_indices = np.where(part[cols] == rank, local_of[cols], ghost_of[cols]).astype(np.int32)
        self.n_own, self.n_ghost = len(rows), len(ghosts)
        gp = part[ghosts]
        self.recv = {}
        for q in range(self.n_ranks):
            idx = np.flatnonzero(gp == q)
            if len(idx):
                self.recv[q] = slice(int(idx[0]), int(idx[-1]) + 1)
        # what each peer needs from me: my rows among its ghosts, in the peer's order
        # (ascending id, the same order as my rows), so send lists are positions
        self.send = {}
        for q in range(self.n_ranks):
            if q == rank:
                continue
            q_take, _ = _row_entries(indptr, np.flatnonzero(part == q))
            need = np.unique(indices[q_take][part[indices[q_take]] == rank])
            if len(need):
                self.send[q] = local_of[need]


class HaloExchange:
    """Fills x_ext[n_own:] (the ghosts) from the peers with one all_to_all_single."""

    def __init__(self, plan, group=None):
        import torch
        import torch.distributed as dist
        self.plan, self.group, self.dist = plan, group, dist
        R = plan.n_ranks
        if dist.is_initialized() and dist.get_world_size(group) != R:
            raise ValueError(f"HaloExchange: the group has {dist.get_world_size(group)} ranks, the partition {R} parts")
        self.send_counts = [len(plan.send.get(q, ())) for q in range(R)]
        self.recv_counts = [(plan.recv[q].stop - plan.recv[q].start) if q in plan.recv else 0 for q in range(R)]
        order = [plan.send[q] for q in range(R) if q in plan.send]
        self._send_idx_np = np.concatenate(order).astype(np.int64) if order else np.zeros(0, np.int64)
        self._torch = torch
        self._send_idx = {}

    def exchange(self, x_ext):
        if self.plan.n_ranks == 1:
            return x_ext  # a single rank has no ghosts
        torch = self._torch
        dev = x_ext.device
        if dev not in self._send_idx:
            self._send_idx[dev] = torch.from_numpy(self._send_idx_np).to(dev)
        n_own = self.plan.n_own
        sendbuf = x_ext[:n_own].index_select(0, self._send_idx[dev])
        recvbuf = x_ext[n_own:]
        self.dist.all_to_all_single(recvbuf, sendbuf, output_split_sizes=self.recv_counts,
                                    input_split_sizes=self.send_counts, group=self.group)
        return x_ext


class DistributedBiCGSTAB:
    """scipy's BiCGSTAB loop (stop at ||r|| < max(atol, rtol ||b||)) over the ranks of a
    group. vals: this rank's entries (plan.src order); b: its rows. spmv(x_ext, y) computes
    y = A_local x_ext; default: the device kernel.

    precond: 'jacobi', or 'block_ilu0' -- ILU(0) of this rank's diagonal block (its own
    rows and columns; the couplings to other ranks' rows are left out of the
    preconditioner, block Jacobi over the ranks), so a preconditioner apply needs no
    exchange. local_precond(r, z) -> z replaces the block's apply; default: the device
    ILU(0) (kcfd_solver_apply_precond)."""

    def __init__(self, plan, vals, group=None, spmv=None, device=None, precond="jacobi", local_precond=None):
        import torch
        self.torch = torch
        self.plan = plan
        self.group = group
        self.halo = HaloExchange(plan, group)
        self.device = device if device is not None else vals.device
        ip = np.asarray(plan.local_indptr)
        rows_of = np.repeat(np.arange(plan.n_own), np.diff(ip))
        diag = np.zeros(plan.n_own)
        v = vals.detach().cpu().numpy()
        on_diag = np.asarray(plan.local_indices) == rows_of
        np.add.at(diag, rows_of[on_diag], v[on_diag])
        dinv = np.where(np.abs(diag) > 1e-30, 1.0 / np.where(diag == 0, 1.0, diag), 0.0)
        self.dinv = torch.from_numpy(dinv).to(self.device)
        if spmv is None:
            from .solver import DeviceCSR
            csr = DeviceCSR(torch.from_numpy(ip).to(self.device),
                            torch.from_numpy(np.asarray(plan.local_indices)).to(self.device), vals.to(self.device))
            csr.n = plan.n_own
            spmv = lambda x, y: csr.spmv(x, y)
        self._spmv = spmv
        if precond not in ("jacobi", "block_ilu0"):
            raise ValueError(f"unknown distributed preconditioner {precond!r}")
        self.precond = precond
        if precond == "block_ilu0" and local_precond is None:
            local_precond = self._device_block_ilu0(ip, np.asarray(plan.local_indices), v)
        self._local_precond = local_precond

    def _device_block_ilu0(self, ip, ix, v):
        """The device ILU(0) of the own diagonal block (columns < n_own, natural-order levels)."""
        torch = self.torch
        from .solver import DeviceCSR, Solver
        n = self.plan.n_own
        keep = ix < n
        rows_of = np.repeat(np.arange(n), np.diff(ip))
        bip = np.zeros(n + 1, dtype=np.int32)
        np.add.at(bip, rows_of[keep] + 1, 1)
        bip = np.cumsum(bip).astype(np.int32)
        csr = DeviceCSR(torch.from_numpy(bip).to(self.device),
                        torch.from_numpy(np.ascontiguousarray(ix[keep], dtype=np.int32)).to(self.device),
                        torch.from_numpy(np.ascontiguousarray(v[keep], dtype=np.float64)).to(self.device))
        csr.n = n
        s = Solver(csr, precond="ilu0")
        s.setup(csr)
        self._block = (csr, s)
        return lambda r, z: s.apply_precond(csr, r, z)

    def _apply(self, q):
        if self.precond == "jacobi":
            return self.dinv * q
        return self._local_precond(q.contiguous(), self.torch.empty_like(q))

    def _dot(self, a, b):
        return self._dots((a, b))[0]

    def _dots(self, *pairs):
        """The global dot products of the pairs with one all_reduce (one host sync). The
        local sums keep the elementwise-product-then-sum form, so each value rounds as a
        single dot's did (late in a tight solve rho = rt.r sits near scipy's absolute
        eps**2 breakdown test, where the last bits decide)."""
        torch = self.torch
        t = torch.stack([(a * b).sum() for a, b in pairs])
        torch.distributed.all_reduce(t, group=self.group)
        return t.tolist()

    def _matvec(self, x_own, x_ext, y):
        x_ext[: self.plan.n_own].copy_(x_own)
        self.halo.exchange(x_ext)
        self._spmv(x_ext, y)
        return y

    def solve(self, b, x=None, rtol=1e-8, atol=0.0, maxiter=1000):
        """Returns (x, info, iterations): info 0 converged, > 0 not converged, < 0
        breakdown (scipy's codes)."""
        torch = self.torch
        p = self.plan
        b = b.to(self.device, torch.float64)
        x = torch.zeros_like(b) if x is None else x.to(self.device, torch.float64).clone()
        x_ext = torch.zeros(p.n_own + p.n_ghost, dtype=torch.float64, device=self.device)
        tmp = torch.empty_like(b)
        bnrm = self._dot(b, b) ** 0.5
        if bnrm == 0.0:
            return b.clone(), 0, 0
        atol = max(float(atol), float(rtol) * bnrm)
        r = b - self._matvec(x, x_ext, tmp) if self._dot(x, x) > 0 else b.clone()
        rt = r.clone()
        eps2 = np.finfo(np.float64).eps ** 2
        rho_prev = omega = alpha = None
        pvec = v = None
        for it in range(maxiter):
            rr, rho = self._dots((r, r), (rt, r))
            if rr ** 0.5 < atol:
                return x, 0, it
            if abs(rho) < eps2:
                return x, -10, it
            if it > 0:
                if abs(omega) < eps2:
                    return x, -11, it
                beta = (rho / rho_prev) * (alpha / omega)
                pvec = (pvec - omega * v) * beta + r
            else:
                pvec = r.clone()
            ph = self._apply(pvec)
            v = self._matvec(ph, x_ext, torch.empty_like(b))
            rv = self._dot(rt, v)
            if rv == 0:
                return x, -11, it + 1
            alpha = rho / rv
            r = r - alpha * v
            # ||s|| is reduced with (t, s) and (t, t): the half-step exit costs one more
            # product on the last iteration, and the loop one all_reduce less per iteration
            sh = self._apply(r)
            t = self._matvec(sh, x_ext, torch.empty_like(b))
            ss, ts, tt = self._dots((r, r), (t, r), (t, t))
            if ss ** 0.5 < atol:
                x = x + alpha * ph
                return x, 0, it + 1
            # t = 0 (s = 0 under a zero stop threshold, or a singular operator): omega = 0,
            # and the next iteration ends in one of scipy's breakdowns (-10 when s = 0,
            # else -11) instead of a division by zero
            omega = ts / tt if tt != 0.0 else 0.0
            x = x + alpha * ph + omega * sh
            r = r - omega * t
            rho_prev = rho
        return x, maxiter, maxiter
