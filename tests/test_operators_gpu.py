"""Generic device operators vs the reference's own outputs (golden fixtures).

Sums are accumulated colour by colour instead of in face-id order, so values agree
with the reference to 1e-12 (scaled by the largest entry); the CSR pattern is the
reference's by construction.
"""
import numpy as np
import pytest

from conftest import load_golden, golden_inputs

pytestmark = pytest.mark.gpu
NAMES = ["quad", "tri", "hex", "hybrid"]


def _close(a, b, tol=1e-12):
    scale = max(np.abs(b).max(), 1e-300)
    assert np.abs(a - b).max() / scale < tol, np.abs(a - b).max() / scale


def _setup(name):
    import torch
    from kcfd import mesh as km
    from kcfd.device_mesh import DeviceMesh
    d = load_golden("mesh_" + name)
    nodes, cells, bdict, cfl = golden_inputs(d)
    m = km.build_mesh(nodes, cells, bdict, ndim=int(d["ndim"]), cell_face_node_list=cfl)
    dm = DeviceMesh(m)
    g = load_golden("ops_" + name)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    f = {k: T(g[k]) for k in ("gamma", "phi", "phi_old", "S", "Sp", "Su")}
    f["mf"] = T(g["mf"][dm.face_ref])
    return m, dm, g, f, T


def _check(sysm, g, p):
    """Operators whose reference COO covers every internal face (diffusion, upwind,
    the full system) must give the reference's CSR pattern exactly; cell-only and
    boundary operators are compared by value (the device system always carries the
    mesh pattern, with explicit zeros where the reference has no entry)."""
    from scipy import sparse
    sysm_csr = sysm.to_sparse()
    sysm_csr.sort_indices()
    ref = sparse.csr_matrix((g[p + "data"], g[p + "indices"], g[p + "indptr"]), shape=sysm_csr.shape)
    if p in ("diff_", "conv_", "full_"):
        np.testing.assert_array_equal(sysm_csr.indptr, g[p + "indptr"])
        np.testing.assert_array_equal(sysm_csr.indices, g[p + "indices"])
        _close(sysm_csr.data, g[p + "data"])
    else:
        diff = (sysm_csr - ref).tocsr()
        scale = max(abs(ref).max(), 1e-300)
        assert (abs(diff).max() if diff.nnz else 0.0) / scale < 1e-12
    _close(sysm.rhs.cpu().numpy(), g[p + "rhs"]) if np.abs(g[p + "rhs"]).max() > 0 else None
    _close(sysm.diag.cpu().numpy(), g[p + "diag"]) if np.abs(g[p + "diag"]).max() > 0 else None


@pytest.mark.parametrize("name", NAMES)
def test_operators_match_reference(name):
    from kcfd.assembly import DeviceSystem, boundary_arrays
    m, dm, g, f, T = _setup(name)
    s = DeviceSystem(dm); s.diffusion_operator(f["gamma"]); _check(s, g, "diff_")
    s = DeviceSystem(dm); s.convection_operator_upwind(f["mf"]); _check(s, g, "conv_")
    s = DeviceSystem(dm); s.temporal_operator(1.3, 0.01, f["phi_old"]); _check(s, g, "temp_")
    s = DeviceSystem(dm); s.source_term(f["S"]); _close(s.rhs.cpu().numpy(), g["src_rhs"])
    s = DeviceSystem(dm); s.linearized_source(f["Sp"], f["Su"]); _check(s, g, "lin_")
    names = list(m.boundary_patches)
    bc = {}
    for nm, kind, val in zip(names, g["bc_kind"], g["bc_value"]):
        bc[nm] = {"type": str(kind), "value": float(val)} if str(kind) == "neumann" else {"type": str(kind)}
    phib, k = {}, 0
    for nm in names:
        nf = len(m.boundary_patches[nm])
        phib[nm] = g["phi_b"][k:k + nf]
        k += nf
    bt, bv, bg = boundary_arrays(dm, bc, phib)
    s = DeviceSystem(dm); s.apply_boundary_conditions(bt, bv, bg, f["gamma"], f["mf"]); _check(s, g, "bc_")
    s = DeviceSystem(dm)
    s.diffusion_operator(f["gamma"])
    s.convection_operator_upwind(f["mf"])
    s.temporal_operator(1.3, 0.01, f["phi_old"])
    s.apply_boundary_conditions(bt, bv, bg, f["gamma"], f["mf"])
    s.under_relax(f["phi"], 0.7)
    _check(s, g, "full_")


@pytest.mark.parametrize("name", NAMES)
def test_muscl_matches_reference(name):
    from kcfd.assembly import muscl_deferred_correction
    m, dm, g, f, T = _setup(name)
    grad = T(g["gg"])
    for lim in ("minmod", "superbee", "van_albada", "van_leer"):
        c = muscl_deferred_correction(dm, f["phi"], f["mf"], grad, lim)
        _close(c.cpu().numpy(), g["muscl_" + lim])


def test_device_system_solves_through_linear_solver():
    """A device-assembled system goes straight into solve_linear_system(backend='b200')."""
    import scipy.sparse.linalg as spla
    from kcfd.assembly import DeviceSystem
    from kcfd.linear_solver import solve_linear_system
    m, dm, g, f, T = _setup("hex")
    s = DeviceSystem(dm)
    s.diffusion_operator(f["gamma"])
    s.temporal_operator(1.3, 0.01, f["phi_old"])
    x = solve_linear_system(s, None, "bicgstab", 1e-12, 2000, "b200", "ilu0", rtol=0.0)
    A = s.to_sparse()
    b = s.rhs.cpu().numpy()
    xd = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-9


@pytest.mark.parametrize("name", NAMES)
def test_reference_signature_operators(name):
    """The module-level operators of kcfd.fvm_operators (the reference's signatures:
    op(mesh, ..., system), host arrays, mass flux in reference face order, a
    ScalarField-like phi with per-patch boundary values) give the reference's full
    system on the host FVMSystem mirror and on a DeviceSystem."""
    from types import SimpleNamespace
    from scipy import sparse
    from kcfd import fvm_operators as kf
    from kcfd.assembly import DeviceSystem
    m, dm, g, f, T = _setup(name)
    names = list(m.boundary_patches)
    bc = {}
    for nm, kind, val in zip(names, g["bc_kind"], g["bc_value"]):
        bc[nm] = {"type": str(kind), "value": float(val)} if str(kind) == "neumann" else {"type": str(kind)}
    phib, k = {}, 0
    for nm in names:
        nf = len(m.boundary_patches[nm])
        phib[nm] = g["phi_b"][k:k + nf]
        k += nf
    phi = SimpleNamespace(values=g["phi"], boundary_values=phib)
    gamma = SimpleNamespace(values=g["gamma"])
    ref = sparse.csr_matrix((g["full_data"], g["full_indices"], g["full_indptr"]))
    for system in (kf.FVMSystem(m.n_cells), DeviceSystem(dm)):
        kf.diffusion_operator(m, gamma, system)
        kf.convection_operator_upwind(m, g["mf"], system)
        kf.temporal_operator(m, 1.3, 0.01, g["phi_old"], system)
        kf.apply_boundary_conditions(m, phi, gamma, g["mf"], system, bc)
        kf.under_relax(system, phi, 0.7)
        A = system.to_sparse()
        A.sort_indices()
        np.testing.assert_array_equal(A.indptr, g["full_indptr"])
        np.testing.assert_array_equal(A.indices, g["full_indices"])
        _close(A.data, ref.data)
        rhs = system.rhs.cpu().numpy() if hasattr(system.rhs, "cpu") else system.rhs
        diag = system.diag.cpu().numpy() if hasattr(system.diag, "cpu") else system.diag
        _close(rhs, g["full_rhs"])
        _close(diag, g["full_diag"])
    s = kf.FVMSystem(m.n_cells)
    kf.source_term(m, g["S"], s)
    _close(s.rhs, g["src_rhs"])
    s = kf.FVMSystem(m.n_cells)
    kf.linearized_source(m, g["Sp"], g["Su"], s)
    _close(s.rhs, g["lin_rhs"]) if np.abs(g["lin_rhs"]).max() > 0 else None
    _close(s.diag, g["lin_diag"]) if np.abs(g["lin_diag"]).max() > 0 else None


@pytest.mark.parametrize("name", NAMES)
def test_reference_signature_muscl(name):
    """kcfd.interpolation.muscl_deferred_correction with the reference's signature
    (host arrays, mass flux in reference face order) equals the reference's output."""
    from types import SimpleNamespace
    from kcfd.interpolation import muscl_deferred_correction
    m, dm, g, f, T = _setup(name)
    phi = SimpleNamespace(values=g["phi"])
    for lim in ("minmod", "superbee", "van_albada", "van_leer"):
        c = muscl_deferred_correction(m, phi, g["mf"], g["gg"], lim)
        _close(c, g["muscl_" + lim])
