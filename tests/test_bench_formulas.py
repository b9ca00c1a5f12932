"""The algorithmic-byte formulas behind the bench's roofline fields, checked against
worked sizes of the 128^3 cavity (host only): one FP64 SpMV of the p' matrix is
nnz (8 + 4) + 4 (n + 1) + 2 n 8 = 216.9 MB; one BiCGSTAB + ILU(0) iteration is
2 SpMV + 2 ILU applies + 19 vectors = 1,270.3 MB; one multigrid-preconditioned
iteration is 2 FP64 SpMV + 2 V-cycles + 17 FP64 vectors, a V-cycle summing its four
kernels per level and the dense coarse solve; the whole outer iteration adds the mass
flux, gradient, MUSCL and assembly terms to the two solves."""

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
    total = bench.outer_step_bytes(n, Fi, Fb, nnz, 3, its_m, its_p, "ilu0")
    solves = bench.solver_bytes(n, nnz, its_m, "jacobi", 8, nrhs=3) + bench.solver_bytes(n, nnz, its_p, "ilu0", 8)
    rest = total - solves
    assert 0 < rest < 0.05 * total          # assembly and gradients are a few percent of the step
    assert abs(total / 1e9 - 622.3) < 0.5   # GB per step at these Krylov counts


def test_vcycle_and_multigrid_iteration_bytes():
    levels = [{"rows": 1000, "nnz": 7000, "p_nnz": 3000}, {"rows": 120, "nnz": 3000, "p_nnz": 500},
              {"rows": 10, "nnz": 80, "p_nnz": 0}]
    w = 8
    l0 = (7000 * 12 + 1000 * (8 + 24)) + (3000 * 12 + 4 * 121 + 1000 * 8 + 120 * 8) + \
         (3000 * 12 + 4 * 1001 + 120 * 8 + 2 * 1000 * 8) + (7000 * 12 + 1000 * (16 + 16))
    l1 = (3000 * 12 + 120 * (8 + 24)) + (500 * 12 + 4 * 11 + 120 * 8 + 10 * 8) + \
         (500 * 12 + 4 * 121 + 10 * 8 + 2 * 120 * 8) + (3000 * 12 + 120 * (16 + 16))
    coarse = 100 * 8 + 2 * 10 * 8
    assert bench.vcycle_bytes(levels, w) == l0 + l1 + coarse
    # FP32 hierarchy: level-0 input and output stay the FP64 Krylov vectors
    l0_32 = (7000 * 8 + 1000 * (8 + 12)) + (3000 * 8 + 4 * 121 + 1000 * 4 + 120 * 4) + \
        (3000 * 8 + 4 * 1001 + 120 * 4 + 2 * 1000 * 4) + (7000 * 8 + 1000 * (8 + 16))
    l1_32 = (3000 * 8 + 120 * (4 + 12)) + (500 * 8 + 4 * 11 + 120 * 4 + 10 * 4) + \
        (500 * 8 + 4 * 121 + 10 * 4 + 2 * 120 * 4) + (3000 * 8 + 120 * (8 + 8))
    assert bench.vcycle_bytes(levels, 4) == l0_32 + l1_32 + 100 * 4 + 2 * 10 * 4
    spmv8 = 7000 * 12 + 4 * 1001 + 16 * 1000
    assert bench.solver_bytes(1000, 7000, 3, "amg", 8, amg=levels) == \
        3 * (2 * spmv8 + 2 * bench.vcycle_bytes(levels, 8) + 17 * 1000 * 8)
