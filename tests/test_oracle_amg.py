"""The oracle's smoothed-aggregation multigrid (oracle/amg.py), host only.

The reference's 'amg' preconditioner is pyamg's (core/preconditioner.py:63-74), which is
not installed, so the restatement is checked against the method's own properties and
at the solution level: aggregates partition the rows; P reproduces the constant on
zero-row-sum rows; the Galerkin operator of a symmetric matrix is symmetric; the dense
coarse solve inverts; the power-iteration omega matches a converged estimate; and
BiCGSTAB preconditioned by one V-cycle solves the reference's case-16 system and a
pressure-correction system to the direct solution in far fewer iterations than Jacobi.
"""
import numpy as np
from scipy import sparse
import scipy.sparse.linalg as spla

from conftest import load_golden
from oracle import amg, linsolve


def _c16():
    g = load_golden("solvers")
    A = sparse.csr_matrix((g["c16_20_data"], g["c16_20_indices"], g["c16_20_indptr"]))
    return A, g["c16_20_rhs"], g["c16_20_direct"]


def pp_system(N=12, iters=2):
    """The pressure-correction system of an N^3 jittered cavity after `iters` outer
    iterations of the oracle (pinned row 0, zero-gradient walls)."""
    from kcfd import meshgen
    from oracle import mesh as om, simple as osim
    nodes, cells, cf, bd = meshgen.hex_box_arrays(1.0, 1.0, 1.0, N, N, N, meshgen.CAVITY_3D_NAMES)
    nodes = meshgen.jitter_interior(nodes, (N, N, N), (1.0 / N,) * 3, 0.2, seed=0)
    o = osim.Simple(om.build_3d(nodes, cells, cf, bd), rho=1.0, mu=0.0025)
    osim.cavity_setup(o)
    for _ in range(iters):
        o.iterate()
    A, b, _ = o.pressure_system(o.face_mass_flux())
    A.sort_indices()
    return A, b


def test_aggregates_partition_rows():
    A, b = pp_system()
    agg, na = amg.aggregate(A)
    assert agg.min() == 0 and agg.max() == na - 1
    assert len(np.unique(agg)) == na
    assert na < A.shape[0] / 4      # 3D 7-point stencils: aggregates of about 8 rows


def test_prolongator_keeps_constants_on_zero_sum_rows():
    A, b = pp_system()
    H = amg.Hierarchy(A)
    L = H.levels[0]
    rs = np.asarray(A.sum(axis=1)).ravel()
    zero = np.abs(rs) < 1e-12 * np.asarray(abs(A).sum(axis=1)).ravel()
    prs = np.asarray(L.P.sum(axis=1)).ravel()
    np.testing.assert_allclose(prs[zero], 1.0, rtol=0, atol=1e-12)


def test_galerkin_of_symmetric_is_symmetric():
    A, b = pp_system()
    S = A.copy().tolil()
    S[0, :] = A[:, 0].T.toarray()       # undo the row-0 pin: symmetric Neumann operator + 1 on (0,0)
    S = S.tocsr()
    S = (S + S.T) * 0.5
    H = amg.Hierarchy(S.tocsr())
    for L in H.levels[1:]:
        d = L.A - L.A.T
        assert abs(d).max() <= 1e-12 * abs(L.A).max()


def test_dense_inverse():
    rng = np.random.default_rng(0)
    M = rng.normal(size=(40, 40)) + 40 * np.eye(40)
    np.testing.assert_allclose(amg.dense_inverse(M), np.linalg.inv(M), rtol=0, atol=1e-13)
    # a singular matrix: the dropped unknown gives a bounded result
    S = M.copy()
    S[:, 5] = 0.0
    inv = amg.dense_inverse(S)
    assert np.all(np.isfinite(inv))
    # one row pinned by a huge diagonal (the two-fluid pressure correction's pin) drops
    # nothing: the tolerance is per column
    P = M * 1e-4
    P[0, 0] += 1e10
    np.testing.assert_allclose(amg.dense_inverse(P) @ P, np.eye(40), rtol=0, atol=1e-9)


def test_power_omega_close_to_converged_estimate():
    A, b = pp_system()
    H = amg.Hierarchy(A)
    L = H.levels[1]
    lam_ref = np.max(np.abs(np.linalg.eigvals((sparse.diags(L.dinv) @ L.A).toarray())))
    lam = (4.0 / 3.0) / L.omega
    assert 0.8 * lam_ref <= lam <= 1.0001 * lam_ref


def test_amg_bicgstab_solves_case16_and_pressure_system():
    A, b, xd = _c16()
    H = amg.Hierarchy(A)
    x, info, its = linsolve.bicgstab_scipy(A, b, rtol=1e-10, atol=0.0, maxiter=500, M=H.operator())
    assert info == 0 and np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    _, _, its_j = linsolve.bicgstab_scipy(A, b, rtol=1e-10, atol=0.0, maxiter=500, M=linsolve.jacobi(A))
    assert its < its_j
    A, b = pp_system()
    xd = spla.spsolve(A.tocsc(), b)
    H = amg.Hierarchy(A)
    x, info, its = linsolve.bicgstab_scipy(A, b, rtol=1e-10, atol=0.0, maxiter=500, M=H.operator())
    assert info == 0 and np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    _, _, its_j = linsolve.bicgstab_scipy(A, b, rtol=1e-10, atol=0.0, maxiter=2000, M=linsolve.jacobi(A))
    assert its * 5 < its_j, (its, its_j)
