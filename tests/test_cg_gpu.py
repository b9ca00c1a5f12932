"""Device conjugate gradients (the graph engine's CG, KCFD_METHOD_CG) against scipy's cg,
the reference's solve_pressure_correction branch (core/linear_solver.py:73-93).

Same algorithm and stopping rule (||r|| < max(atol, rtol ||b||) tested before every
iteration), so on a symmetric positive definite diffusion system the Krylov counts agree
within 1 (only the reduction order differs) and the solutions within 1e-8 relative L2;
with the device-only preconditioners (ILU(0), multigrid) the true residual meets the
tolerance."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _diffusion_system(nx, seed):
    """Diffusion (harmonic, Gamma log-uniform) + a time term (dt 0.1) on a jittered nx^3 hex box:
    SPD, with a condition number of a few hundred (a tolerance of 1e-10 is attainable)."""
    from kcfd import meshgen
    from oracle import mesh as om, fvm
    n, c, f, b = meshgen.hex_box_arrays(1, 1, 1, nx, nx, nx, meshgen.CAVITY_3D_NAMES)
    n = meshgen.jitter_interior(n, (nx, nx, nx), (1.0 / nx,) * 3, 0.2, seed=seed)
    m = om.build_3d(n, c, f, b)
    rng = np.random.default_rng(seed)
    s = fvm.System(m.n_cells)
    fvm.diffusion_operator(m, np.exp(rng.uniform(np.log(0.1), np.log(10.0), m.n_cells)), s)
    fvm.temporal_operator(m, 1.0, 0.1, np.zeros(m.n_cells), s)
    A = s.to_sparse()
    return A, rng.normal(size=m.n_cells), (n, c, f, b)


def _device_cg(A, b, precond, atol, rtol, maxiter, levels=None):
    import torch
    from kcfd import _lib
    from kcfd.solver import DeviceCSR, Solver
    d = DeviceCSR.from_scipy(A)
    s = Solver(d, precond=precond, stop=_lib.STOP_SCIPY, rtol=rtol, atol=atol, maxiter=maxiter, method="cg",
               levels=levels)
    assert s.info()["team"] == 3
    s.setup(d)
    x = torch.zeros(d.n, dtype=torch.float64, device="cuda")
    it, rr, st = s.solve(d, torch.from_numpy(b).cuda(), x)
    return x.cpu().numpy(), int(it[0]), int(st[0])


@pytest.mark.parametrize("precond", ["none", "jacobi"])
def test_cg_matches_scipy(precond):
    A, b, _ = _diffusion_system(24, seed=3)
    atol = 1e-10 * np.linalg.norm(b)
    M = None
    if precond == "jacobi":
        dinv = 1.0 / A.diagonal()
        M = spla.LinearOperator(A.shape, matvec=lambda v: dinv * v)
    count = [0]
    xs, info = spla.cg(A, b, atol=atol, rtol=0.0, maxiter=5000, M=M, callback=lambda xk: count.__setitem__(0, count[0] + 1))
    assert info == 0 and np.linalg.norm(b - A @ xs) < 1.01 * atol
    xd, its, st = _device_cg(A, b, precond, atol, 0.0, 5000)
    assert st == 0
    assert abs(its - count[0]) <= 1, (its, count[0])
    assert np.linalg.norm(b - A @ xd) < 1.01 * atol
    assert _rel(xd, xs) < 1e-8


@pytest.mark.parametrize("precond", ["ilu0", "amg"])
def test_cg_device_preconditioners_converge(precond):
    from kcfd import mesh as km
    A, b, arrays = _diffusion_system(24, seed=5)
    n, c, f, bd = arrays
    levels = km.build_mesh(n, c, bd, ndim=3, cell_face_node_list=f).cell_color if precond == "ilu0" else None
    atol = 1e-9 * np.linalg.norm(b)
    _, none_its, _ = _device_cg(A, b, "none", atol, 0.0, 5000)
    xd, its, st = _device_cg(A, b, precond, atol, 0.0, 5000, levels=levels)
    assert st == 0
    assert np.linalg.norm(b - A @ xd) < 1.01 * atol
    assert its < none_its, (precond, its, none_its)


def test_cg_maxiter_reports_like_scipy():
    """scipy tests before each iteration only: after maxiter iterations it reports maxiter."""
    A, b, _ = _diffusion_system(16, seed=7)
    xd, its, st = _device_cg(A, b, "jacobi", 0.0, 1e-14, 5)
    assert st == 1 and its == 5
    x5, info = spla.cg(A, b, atol=0.0, rtol=1e-14, maxiter=5,
                       M=spla.LinearOperator(A.shape, matvec=lambda v: v / A.diagonal()))
    assert info == 5
    assert _rel(xd, x5) < 1e-10


def test_solve_pressure_correction_runs_cg_on_the_device():
    """The drop-in's iterative branch: cg from zero with atol=tol (scipy's rtol 1e-5)."""
    from kcfd.fvm_operators import FVMSystem
    from kcfd.linear_solver import solve_pressure_correction
    A, b, _ = _diffusion_system(16, seed=9)
    tol = 1e-8 * np.linalg.norm(b)
    x = solve_pressure_correction(FVMSystem.from_csr(A, b), method="cg", tol=tol, maxiter=2000,
                                  preconditioner="jacobi")
    xs, info = spla.cg(A, b, x0=np.zeros(len(b)), atol=tol, maxiter=2000,
                       M=spla.LinearOperator(A.shape, matvec=lambda v: v / A.diagonal()))
    assert np.linalg.norm(b - A @ x) < 1.01 * max(tol, 1e-5 * np.linalg.norm(b))
    assert _rel(x, xs) < 1e-8
