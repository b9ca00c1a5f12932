"""Single-mesh partitioning (kcfd.parallel) against the reference's parallel/partitioning.py,
and the partitioned solve on world-size-2 gloo ranks (host code; the local SpMV is a
scipy stand-in injected by the test, the device kernel being the product's).

- RCB part ids and ghost maps equal the reference's on every fixture mesh for 2-5
  parts (tests/golden/part_*.npz, written by tests/golden/make_golden.py from the
  reference itself).
- Each rank's local CSR times [its x | ghost x] equals the global product on its rows.
- The two-rank distributed BiCGSTAB + Jacobi reaches rtol 1e-10, matches spsolve to
  1e-8 and takes the oracle's iteration count within 10% (at least 2)."""
import os

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch.multiprocessing as mp
from scipy import sparse

from case16 import channel_mesh, convdiff_system
from conftest import golden_inputs, load_golden
from kcfd import mesh as km
from kcfd.parallel import GeometricPartitioner, GhostCellLayer, HaloPlan

MESHES = ["quad", "cavity", "tri", "hex", "hybrid"]


def _mesh(name):
    d = load_golden("mesh_" + name)
    nodes, cells, bdict, cfl = golden_inputs(d)
    return km.build_mesh(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl)


@pytest.mark.parametrize("name", MESHES)
def test_rcb_and_ghosts_match_reference(name):
    m = _mesh(name)
    ref = load_golden("part_" + name)
    for n_parts in (2, 3, 4, 5):
        part = GeometricPartitioner(m).partition(n_parts)
        np.testing.assert_array_equal(part, ref[f"part{n_parts}"])
        g = GhostCellLayer(m, part)
        trip = [(r, q, c) for r in sorted(g.ghost_map) for q in sorted(g.ghost_map[r]) for c in g.ghost_map[r][q]]
        np.testing.assert_array_equal(np.asarray(trip, dtype=np.int64).reshape(-1, 3), ref[f"ghost{n_parts}"])
        for r in range(n_parts):
            np.testing.assert_array_equal(g.get_local_cells(r), np.flatnonzero(part == r))


@pytest.mark.parametrize("n_parts", [2, 3, 4])
def test_halo_plan_local_products(n_parts):
    m = _mesh("cavity")
    ip, ix = np.asarray(m.indptr), np.asarray(m.indices)
    n = m.n_cells
    rng = np.random.default_rng(n_parts)
    A = sparse.csr_matrix((rng.standard_normal(len(ix)), ix, ip), shape=(n, n))
    x = rng.standard_normal(n)
    y = A @ x
    part = GeometricPartitioner(m).partition(n_parts)
    covered = np.zeros(n, bool)
    for r in range(n_parts):
        p = HaloPlan(ip, ix, part, r)
        Al = sparse.csr_matrix((A.data[p.src], p.local_indices, p.local_indptr), shape=(p.n_own, p.n_own + p.n_ghost))
        xe = np.concatenate([x[p.rows], x[p.ghosts]])
        np.testing.assert_allclose(Al @ xe, y[p.rows], rtol=0, atol=1e-14)
        assert set(p.ghosts) == {c for cells in GhostCellLayer(m, part).get_ghost_cells(r).values() for c in cells}
        for q, sl in p.recv.items():
            peer = HaloPlan(ip, ix, part, q)
            np.testing.assert_array_equal(peer.rows[peer.send[r]], p.ghosts[sl])
        covered[p.rows] = True
    assert covered.all()


def _solve_worker(rank, world, port, out, precond="jacobi"):
    import torch
    import torch.distributed as dist
    from kcfd.parallel import DistributedBiCGSTAB
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    A, b = convdiff_system(channel_mesh(24, 18))
    A = sparse.csr_matrix(A)
    n = A.shape[0]
    # partition on the cell index (a stand-in geometry for this matrix)
    part = (np.arange(n) * world) // n
    p = HaloPlan(A.indptr, A.indices, part, rank)
    vals = torch.from_numpy(A.data[p.src].copy())
    Al = sparse.csr_matrix((A.data[p.src], p.local_indices, p.local_indptr), shape=(p.n_own, p.n_own + p.n_ghost))

    def spmv(x_ext, y):
        y.copy_(torch.from_numpy(Al @ x_ext.numpy()))
        return y

    local = None
    if precond == "block_ilu0":
        # host stand-in for the device ILU(0) of the own diagonal block (the oracle's)
        from oracle.linsolve import ilu0_factor, ilu0_apply
        Bf, perm = ilu0_factor(Al[:, : p.n_own].tocsr())

        def local(r, z):
            z.copy_(torch.from_numpy(ilu0_apply(Bf, perm, r.numpy())))
            return z
    solver = DistributedBiCGSTAB(p, vals, spmv=spmv, device=torch.device("cpu"), precond=precond,
                                 local_precond=local)
    reduce, calls = dist.all_reduce, []

    def counted(*a, **k):
        calls.append(1)
        return reduce(*a, **k)
    dist.all_reduce = counted
    try:
        x, info, its = solver.solve(torch.from_numpy(b[p.rows].copy()), rtol=1e-10, maxiter=2000)
    finally:
        dist.all_reduce = reduce
    full = torch.zeros(n, dtype=torch.float64)
    full[torch.from_numpy(p.rows)] = x
    dist.all_reduce(full)
    if rank == 0:
        out.put((full.numpy().tolist(), info, its, len(calls)))
    dist.barrier()
    dist.destroy_process_group()


def _run_two_ranks(precond, port):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_solve_worker, args=(r, 2, port, q, precond)) for r in range(2)]
    for p in ps:
        p.start()
    res = q.get(timeout=180)
    for p in ps:
        p.join(timeout=120)
    return res


def test_two_rank_block_ilu0():
    """Block-Jacobi ILU(0) over the two ranks (each factors its own diagonal block, no
    exchange in an apply) converges to the direct solution in fewer iterations than
    Jacobi."""
    x, info, its, _ = _run_two_ranks("block_ilu0", 29700 + (os.getpid() + 500) % 1000)
    xj, infoj, itsj, _ = _run_two_ranks("jacobi", 29700 + (os.getpid() + 700) % 1000)
    A, b = convdiff_system(channel_mesh(24, 18))
    xd = spla.spsolve(sparse.csc_matrix(A), b)
    assert info == 0 and infoj == 0
    assert np.linalg.norm(np.asarray(x) - xd) / np.linalg.norm(xd) < 1e-8
    assert its < itsj, (its, itsj)


def test_two_rank_distributed_bicgstab():
    from oracle.linsolve import bicgstab_scipy, jacobi
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    ps = [ctx.Process(target=_solve_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    x, info, its, n_reduce = q.get(timeout=180)
    for p in ps:
        p.join(timeout=120)
    A, b = convdiff_system(channel_mesh(24, 18))
    x = np.asarray(x)
    assert info == 0
    # ||b|| and x.x, then three all_reduces per iteration (one more if the exit is at the top)
    assert n_reduce <= 3 * its + 3, (n_reduce, its)
    xd = spla.spsolve(sparse.csc_matrix(A), b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-8
    _, info_o, its_o = bicgstab_scipy(A, b, np.zeros(len(b)), rtol=1e-10, atol=0.0, maxiter=2000, M=jacobi(A))
    assert info_o == 0 and abs(its - its_o) <= max(2, its_o // 10), (its, its_o)


def _exchange_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from kcfd.parallel import HaloExchange
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A, _ = convdiff_system(channel_mesh(24, 18))
        A = sparse.csr_matrix(A)
        n = A.shape[0]
        part = np.random.default_rng(7).integers(0, world, n)   # scattered: every rank talks to every peer
        p = HaloPlan(A.indptr, A.indices, part, rank)
        x = np.sin(np.arange(n) * 0.37) + 2.0
        x_ext = torch.zeros(p.n_own + p.n_ghost, dtype=torch.float64)
        x_ext[: p.n_own] = torch.from_numpy(x[p.rows])
        HaloExchange(p).exchange(x_ext)
        Al = sparse.csr_matrix((A.data[p.src], p.local_indices, p.local_indptr), shape=(p.n_own, p.n_own + p.n_ghost))
        ok_ghost = np.array_equal(x_ext[p.n_own:].numpy(), x[p.ghosts])
        ok_prod = np.allclose(Al @ x_ext.numpy(), (A @ x)[p.rows], rtol=1e-14, atol=0.0)
        out.put((rank, bool(ok_ghost), bool(ok_prod), p.n_own, p.n_ghost, sorted(p.recv), sorted(p.send)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_three_rank_exchange_on_a_scattered_partition():
    """Three gloo ranks, cells scattered over them at random (ragged counts, every rank
    exchanging with both peers): after one exchange every ghost holds its owner's value and
    every rank's local product equals its rows of the global product."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() + 300) % 1000
    ps = [ctx.Process(target=_exchange_worker, args=(r, 3, port, q)) for r in range(3)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(3))
    for p in ps:
        p.join(timeout=120)
    assert [r[0] for r in res] == [0, 1, 2]
    for rank, ok_ghost, ok_prod, n_own, n_ghost, recv, send in res:
        assert ok_ghost and ok_prod, (rank, ok_ghost, ok_prod)
        peers = [q for q in range(3) if q != rank]
        assert recv == peers and send == peers, (rank, recv, send)
    assert sum(r[3] for r in res) == 24 * 18 and len({r[3] for r in res}) > 1


def _exact_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from kcfd.parallel import DistributedBiCGSTAB
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 6
        A = sparse.csr_matrix(sparse.identity(n) * 2.0)    # solved exactly in one half-step
        part = (np.arange(n) * world) // n
        p = HaloPlan(A.indptr, A.indices, part, rank)
        Al = sparse.csr_matrix((A.data[p.src], p.local_indices, p.local_indptr), shape=(p.n_own, p.n_own + p.n_ghost))

        def spmv(x_ext, y):
            y.copy_(torch.from_numpy(Al @ x_ext.numpy()))
            return y
        s = DistributedBiCGSTAB(p, torch.from_numpy(A.data[p.src].copy()), spmv=spmv, device=torch.device("cpu"))
        b = torch.ones(p.n_own, dtype=torch.float64)
        x, info, its = s.solve(b, rtol=0.0, atol=0.0, maxiter=5)
        out.put((rank, x.tolist(), info, its))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_zero_threshold_exact_solve_ends_without_dividing_by_zero():
    """With rtol = atol = 0 an exactly solved system (s = 0, t = 0) ends, with the exact
    solution, as scipy's loop orders it: rho = rt.r = 0 at the next iteration (-10),
    on every rank alike, without dividing by t.t = 0."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() + 900) % 1000
    ps = [ctx.Process(target=_exact_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in ps:
        p.join(timeout=120)
    for rank, x, info, its in res:
        assert info == -10 and its == 1, (rank, info, its)
        assert np.allclose(x, 0.5, rtol=0, atol=0), x
