"""The algorithmic-byte formulas behind the bench's roofline fields, checked against
worked sizes of the 128^3 cavity (host only): one FP64 SpMV of the p' matrix is
nnz (8 + 4) + 4 (n + 1) + 2 n 8 = 216.9 MB; one BiCGSTAB + ILU(0) iteration is
2 SpMV + 2 ILU applies + 19 vectors = 1,270.3 MB; the whole outer iteration adds the
mass flux, gradient, MUSCL and assembly terms to the two solves."""

import bench

N = 128
n = N ** 3
Fi = 3 * N * N * (N - 1)          # internal faces of an N^3 hex box
Fb = 6 * N * N
nnz = n + 2 * Fi


def test_mesh_counts():
    assert nnz == 14_581_760 and Fi + Fb == 6_340_608


def test_spmv_and_iteration_bytes():
    spmv = nnz * 12 + 4 * (n + 1) + 16 * n
    assert spmv == 216_924_164
    ilu = nnz * 12 + 8 * (n + 1) + 4 * n * 8
    assert bench.solver_bytes(n, nnz, 1, "ilu0", 8) == 2 * spmv + 2 * ilu + 19 * n * 8 == 1_270_349_848
    assert bench.solver_bytes(n, nnz, 7, "ilu0", 8) == 7 * 1_270_349_848
    # Jacobi with 3 right-hand sides: the matrix once per SpMV, vectors per rhs
    spmv3 = nnz * 12 + 4 * (n + 1) + 2 * n * 8 * 3
    assert bench.solver_bytes(n, nnz, 1, "jacobi", 8, nrhs=3) == 2 * spmv3 + 21 * n * 8 * 3


def test_outer_step_is_solves_plus_face_and_cell_terms():
    its_m, its_p = 12, 470
    total = bench.outer_step_bytes(n, Fi, Fb, nnz, 3, its_m, its_p)
    solves = bench.solver_bytes(n, nnz, its_m, "jacobi", 8, nrhs=3) + bench.solver_bytes(n, nnz, its_p, "ilu0", 8)
    rest = total - solves
    assert 0 < rest < 0.05 * total          # assembly and gradients are a few percent of the step
    assert abs(total / 1e9 - 622.3) < 0.5   # GB per step at these Krylov counts
