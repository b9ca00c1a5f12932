"""Oracle FVM operators vs the reference's own outputs (golden fixtures)."""
import numpy as np
import pytest

from conftest import load_golden, golden_inputs
from oracle import fvm, mesh as om

NAMES = ["quad", "tri", "hex", "hybrid"]


def _mesh(name):
    d = load_golden("mesh_" + name)
    nodes, cells, bdict, cfl = golden_inputs(d)
    return om.build(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl)


def _patch_split(m, flat):
    out, k = {}, 0
    for nm, f in m.boundary_patches.items():
        out[nm] = flat[k:k + len(f)]
        k += len(f)
    return out


def _bc(m, d):
    out = {}
    for nm, kind, val in zip(m.boundary_patches, d["bc_kind"], d["bc_value"]):
        out[nm] = {"type": str(kind), "value": float(val)} if str(kind) == "neumann" else {"type": str(kind)}
    return out


def _check_system(s, d, p, rtol=1e-14):
    A = s.to_sparse()
    A.sort_indices()
    np.testing.assert_array_equal(A.indptr, d[p + "indptr"])
    np.testing.assert_array_equal(A.indices, d[p + "indices"])
    np.testing.assert_allclose(A.data, d[p + "data"], rtol=rtol, atol=1e-300)
    np.testing.assert_allclose(s.rhs, d[p + "rhs"], rtol=rtol, atol=1e-15)
    np.testing.assert_allclose(s.diag, d[p + "diag"], rtol=rtol, atol=1e-300)


@pytest.mark.parametrize("name", NAMES)
def test_operators_match_reference(name):
    m = _mesh(name)
    d = load_golden("ops_" + name)
    n = m.n_cells
    phib = _patch_split(m, d["phi_b"])
    bc = _bc(m, d)
    s = fvm.System(n); fvm.diffusion_operator(m, d["gamma"], s); _check_system(s, d, "diff_")
    s = fvm.System(n); fvm.convection_operator_upwind(m, d["mf"], s); _check_system(s, d, "conv_")
    s = fvm.System(n); fvm.temporal_operator(m, 1.3, 0.01, d["phi_old"], s); _check_system(s, d, "temp_")
    s = fvm.System(n); fvm.source_term(m, d["S"], s)
    np.testing.assert_allclose(s.rhs, d["src_rhs"], rtol=1e-14)
    s = fvm.System(n); fvm.linearized_source(m, d["Sp"], d["Su"], s); _check_system(s, d, "lin_")
    s = fvm.System(n); fvm.apply_boundary_conditions(m, phib, d["gamma"], d["mf"], s, bc); _check_system(s, d, "bc_")
    s = fvm.System(n)
    fvm.diffusion_operator(m, d["gamma"], s)
    fvm.convection_operator_upwind(m, d["mf"], s)
    fvm.temporal_operator(m, 1.3, 0.01, d["phi_old"], s)
    fvm.apply_boundary_conditions(m, phib, d["gamma"], d["mf"], s, bc)
    fvm.under_relax(s, d["phi"], 0.7)
    _check_system(s, d, "full_")


@pytest.mark.parametrize("name", NAMES)
def test_gradient_flux_muscl_match_reference(name):
    m = _mesh(name)
    d = load_golden("ops_" + name)
    phib = _patch_split(m, d["phi_b"])
    fb = fvm.face_patch_values(m, phib, d["phi"])
    g = fvm.green_gauss_gradient(m, d["phi"], fb)
    np.testing.assert_allclose(g, d["gg"], rtol=1e-13, atol=1e-13)
    gl = fvm.least_squares_gradient(m, d["phi"], fb)
    np.testing.assert_allclose(gl, d["lsq"], rtol=1e-12, atol=1e-12)
    ub = _patch_split(m, d["U_b"])
    ufb = fvm.face_patch_values(m, ub, d["U"])
    mf = fvm.compute_mass_flux(m, d["U"], ufb, 1.7)
    np.testing.assert_allclose(mf, d["mflux"], rtol=1e-14, atol=1e-15)
    for lim in fvm.LIMITERS:
        c = fvm.muscl_deferred_correction(m, d["phi"], d["mf"], d["gg"], lim)
        np.testing.assert_allclose(c, d["muscl_" + lim], rtol=1e-13, atol=1e-14)


def test_csr_pattern_is_canonical_with_explicit_zeros():
    """F10: the pattern is diag + both sides of every internal face, values aside."""
    for name in NAMES:
        m = _mesh(name)
        d = load_golden("ops_" + name)
        ip, ix = om.csr_pattern(m)
        np.testing.assert_array_equal(ip, d["full_indptr"])
        np.testing.assert_array_equal(ix, d["full_indices"])
        assert ip[-1] == m.n_cells + 2 * m.n_internal_faces
