"""Edge cases of the device solver and batch paths: the smallest systems, zero
right-hand sides, an iteration cap of zero, rejected malformed CSR, every team on a
2-right-hand-side system, and a batch of one system and of systems on both tiers."""
import numpy as np
import pytest
from scipy import sparse

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def _dev(torch, A):
    from kcfd.solver import DeviceCSR
    return DeviceCSR.from_scipy(A)


def _poisson(n):
    return sparse.diags([-np.ones(n - 1), 2.5 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1]).tocsr()


@pytest.mark.parametrize("team", [1, 2, 3])
def test_one_row_system(torch_cuda, team):
    from kcfd.solver import Solver
    torch = torch_cuda
    A = sparse.csr_matrix(np.array([[4.0]]))
    d = _dev(torch, A)
    s = Solver(d, precond="jacobi", rtol=1e-12, maxiter=10, team=team)
    s.setup(d)
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    it, rr, st = s.solve(d, torch.tensor([2.0], dtype=torch.float64, device="cuda"), x)
    assert int(st[0]) == 0 and abs(float(x[0]) - 0.5) < 1e-15


@pytest.mark.parametrize("team", [1, 2, 3])
def test_zero_rhs_returns_zero_with_no_iterations(torch_cuda, team):
    from kcfd.solver import Solver
    torch = torch_cuda
    d = _dev(torch, _poisson(5000))
    s = Solver(d, precond="jacobi", rtol=1e-10, maxiter=100, team=team)
    s.setup(d)
    x = torch.ones(5000, dtype=torch.float64, device="cuda")
    it, rr, st = s.solve(d, torch.zeros(5000, dtype=torch.float64, device="cuda"), x)
    # scipy returns b (== 0) for a zero right-hand side
    assert int(st[0]) == 0 and int(it[0]) == 0 and float(x.abs().max()) == 0.0


@pytest.mark.parametrize("team", [1, 2, 3])
def test_maxiter_zero(torch_cuda, team):
    from kcfd import _lib
    from kcfd.solver import Solver
    torch = torch_cuda
    d = _dev(torch, _poisson(3000))
    s = Solver(d, precond="jacobi", rtol=1e-10, maxiter=0, team=team)
    s.setup(d)
    x = torch.zeros(3000, dtype=torch.float64, device="cuda")
    it, rr, st = s.solve(d, torch.ones(3000, dtype=torch.float64, device="cuda"), x)
    assert int(st[0]) == _lib.MAXITER and int(it[0]) == 0 and float(x.abs().max()) == 0.0


def test_malformed_csr_is_rejected(torch_cuda):
    from kcfd import _lib
    from kcfd.solver import DeviceCSR, Solver
    torch = torch_cuda
    ip = torch.tensor([0, 2, 3], dtype=torch.int32, device="cuda")
    bad_col = DeviceCSR(ip, torch.tensor([0, 5, 1], dtype=torch.int32, device="cuda"),
                        torch.ones(3, dtype=torch.float64, device="cuda"))
    with pytest.raises(_lib.KcfdError) as e:
        Solver(bad_col, precond="jacobi")
    assert e.value.status == _lib.BAD_INPUT
    bad_ptr = DeviceCSR(torch.tensor([0, 3, 2], dtype=torch.int32, device="cuda"),
                        torch.tensor([0, 1, 1], dtype=torch.int32, device="cuda"),
                        torch.ones(3, dtype=torch.float64, device="cuda"))
    with pytest.raises(_lib.KcfdError):
        Solver(bad_ptr, precond="jacobi")
    no_diag = DeviceCSR(ip, torch.tensor([1, 1, 0], dtype=torch.int32, device="cuda"),
                        torch.ones(3, dtype=torch.float64, device="cuda"))
    with pytest.raises(_lib.KcfdError):
        Solver(no_diag, precond="ilu0")


@pytest.mark.parametrize("team", [1, 2, 3])
def test_two_right_hand_sides_every_team(torch_cuda, team):
    from kcfd.solver import Solver
    torch = torch_cuda
    n = 30000
    A = _poisson(n)
    d = _dev(torch, A)
    rng = np.random.default_rng(3)
    B = rng.normal(size=(n, 2))
    s = Solver(d, precond="jacobi", rtol=1e-10, maxiter=5000, team=team, nrhs=2)
    s.setup(d)
    x = torch.zeros(n, 2, dtype=torch.float64, device="cuda")
    it, rr, st = s.solve(d, torch.from_numpy(B).cuda(), x)
    assert list(st.cpu().numpy()) == [0, 0]
    X = x.cpu().numpy()
    for c in range(2):
        assert np.linalg.norm(B[:, c] - A @ X[:, c]) / np.linalg.norm(B[:, c]) < 2e-10


def test_batch_single_system_and_both_tiers(torch_cuda):
    from kcfd.batch import BatchSolver
    torch = torch_cuda
    sizes = [50, 20000, 300, 17000]   # two systems on each tier (threshold 16,384 rows)
    mats = [_poisson(n) for n in sizes]
    rng = np.random.default_rng(5)
    rhs = [rng.normal(size=n) for n in sizes]
    for pick in ([0], list(range(4))):
        pats = [(mats[k].indptr, mats[k].indices) for k in pick]
        bs = BatchSolver(pats, mode="fp64", precond="jacobi", rtol=1e-10, maxiter=20000)
        v = torch.cat([torch.from_numpy(mats[k].data).cuda() for k in pick])
        b = bs.pack([rhs[k] for k in pick])
        x = torch.zeros_like(b)
        it, rr, st = bs.solve(v, b, x)
        assert list(st.cpu().numpy()) == [0] * len(pick)
        for xs, k in zip(bs.unpack(x), pick):
            assert np.linalg.norm(rhs[k] - mats[k] @ xs) / np.linalg.norm(rhs[k]) < 2e-10
