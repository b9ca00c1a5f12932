"""The case-16 helper reproduces the reference's own case-16 matrix (golden)."""
import numpy as np

from conftest import load_golden
from case16 import channel_mesh, convdiff_system


def test_case16_matrix_matches_reference():
    g = load_golden("solvers")
    A, b = convdiff_system(channel_mesh(20, 20))
    A.sort_indices()
    np.testing.assert_array_equal(A.indptr, g["c16_20_indptr"])
    np.testing.assert_array_equal(A.indices, g["c16_20_indices"])
    np.testing.assert_allclose(A.data, g["c16_20_data"], rtol=1e-14)
    np.testing.assert_allclose(b, g["c16_20_rhs"], rtol=1e-14)


def test_case16_80_direct_solution_matches_reference():
    import scipy.sparse.linalg as spla
    g = load_golden("solvers")
    A, b = convdiff_system(channel_mesh(80, 80))
    np.testing.assert_allclose(spla.spsolve(A.tocsc(), b), g["c16_80_direct"], rtol=1e-10, atol=1e-14)
