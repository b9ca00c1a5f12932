"""Device assembly kernels vs the oracle (and through it the reference).

The device accumulates face contributions colour by colour instead of in face-id
order, so sums differ from the oracle's by rounding only: values agree to 1e-12
relative (scaled by the largest entry); the CSR pattern is identical by construction.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden, golden_inputs

pytestmark = pytest.mark.gpu

MESHES = ["quad", "tri", "hex", "hybrid"]


def _close(a, b, tol=1e-12):
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale
    assert err < tol, err


def _setup(name, seed=0, muscl=None, nonorth=False):
    from kcfd import mesh as km
    from kcfd.simple import SIMPLESolver
    from oracle import mesh as om, simple as osim
    d = load_golden("mesh_" + name)
    nodes, cells, bdict, cfl = golden_inputs(d)
    ndim = int(d["ndim"])
    m = km.build_mesh(nodes, cells, bdict, ndim=ndim, cell_face_node_list=cfl)
    ref = om.build(nodes, cells, bdict, ndim=ndim, cell_face_node_list=cfl)
    rng = np.random.default_rng(seed)
    dev = SIMPLESolver(m, rho=1.3, mu=0.02, muscl=muscl, nonorth=nonorth)
    ora = osim.Simple(ref, rho=1.3, mu=0.02)
    ora.muscl, ora.nonorth = muscl, nonorth
    names = list(m.boundary_patches)
    for i, nm in enumerate(names):
        kind = "dirichlet" if i % 2 == 0 else "zero_gradient"
        val = rng.normal(size=ndim)
        for s in (dev, ora):
            s.set_velocity_bc(nm, kind, val)
            s.set_pressure_bc(nm, "dirichlet" if i == 1 else "zero_gradient", 0.3)
    U = rng.normal(size=(m.n_cells, ndim))
    p = rng.normal(size=m.n_cells)
    dev.U.values = U
    dev.p.values = p
    ora.U = U.copy()
    ora.p = p.copy()
    return dev, ora


def _call(dev, fn, *args):
    from kcfd import _lib
    _lib.check(getattr(_lib.lib(), fn)(*args), fn)


@pytest.mark.parametrize("name", MESHES)
def test_mass_flux(name):
    from kcfd import _lib
    dev, ora = _setup(name)
    dev.bcs.upload()
    P = _lib.ptr
    _call(dev, "kcfd_mass_flux", C.byref(dev.dm.desc), C.byref(dev.bcs.desc), P(dev.U_t), dev.rho, P(dev.mf_t),
          _lib.stream_handle())
    _close(dev.face_mass_flux(), ora.face_mass_flux(), 1e-13)


@pytest.mark.parametrize("name", MESHES)
@pytest.mark.parametrize("variant", ["upwind", "muscl", "nonorth", "both"])
def test_momentum_and_pressure_assembly(name, variant):
    import torch
    from kcfd import _lib
    muscl = "van_leer" if variant in ("muscl", "both") else None
    nonorth = variant in ("nonorth", "both")
    dev, ora = _setup(name, seed=1, muscl=muscl, nonorth=nonorth)
    dev.bcs.upload()
    mf = ora.face_mass_flux()
    dev.mf_t.copy_(torch.from_numpy(mf[dev.dm.face_ref]))
    P = _lib.ptr
    st = _lib.stream_handle()
    dm, bc = C.byref(dev.dm.desc), C.byref(dev.bcs.desc)
    prm = _lib.MomParams(dev.rho, dev.mu, 0.7, 0.0, _lib.LIMITERS[muscl], 1 if nonorth else 0)
    if dev.gU_t is not None:
        _call(dev, "kcfd_gg_gradient", dm, dev.ndim, P(dev.U_t), P(dev.bcs.tensor("u_type")),
              P(dev.bcs.tensor("u_val")), P(dev.gU_t), st)
    _call(dev, "kcfd_momentum_assemble", dm, bc, C.byref(prm), P(dev.U_t), None, P(dev.p_t), P(dev.mf_t),
          P(dev.gU_t), P(dev.aP_t), P(dev.A_m.vals64), None, P(dev.b_m), P(dev.dP_t), st)
    torch.cuda.synchronize()
    vals = dev.A_m.vals64.cpu().numpy()
    bm = dev.b_m.cpu().numpy()
    for comp in range(dev.ndim):
        A, b, aP = ora.momentum_system(comp, mf)
        A.sort_indices()
        np.testing.assert_array_equal(A.indptr, dev.mesh.indptr)
        np.testing.assert_array_equal(A.indices, dev.mesh.indices)
        _close(vals, A.data)
        _close(bm[:, comp], b)
        ora._aP[comp] = aP * ora.alpha_u
    # p' system from the same state
    _call(dev, "kcfd_pressure_assemble", dm, bc, dev.rho, P(dev.dP_t), P(dev.mf_t), P(dev.aP_t),
          P(dev.A_p.vals64), None, P(dev.b_p), st)
    torch.cuda.synchronize()
    Ap, bp, dP = ora.pressure_system(mf)
    Ap.sort_indices()
    _close(dev.dP_t.cpu().numpy(), dP)
    _close(dev.A_p.vals64.cpu().numpy(), Ap.data)
    _close(dev.b_p.cpu().numpy(), bp)


@pytest.mark.parametrize("name", MESHES)
def test_green_gauss(name):
    import torch
    from kcfd import _lib
    from oracle import fvm
    dev, ora = _setup(name, seed=2)
    dev.bcs.upload()
    P = _lib.ptr
    st = _lib.stream_handle()
    phi = np.random.default_rng(5).normal(size=dev.mesh.n_cells)
    dev.pp_t.copy_(torch.from_numpy(phi))
    _call(dev, "kcfd_gg_gradient", C.byref(dev.dm.desc), 1, P(dev.pp_t), P(dev.bcs.tensor("pp_type")),
          P(dev.bcs.tensor("pp_val")), P(dev.gpp_t), st)
    g = fvm.green_gauss_gradient(ora.mesh, phi, ora.pp_face_values(phi))
    _close(dev.gpp_t.cpu().numpy(), g)
    # vector field with dirichlet values on velocity patches
    _call(dev, "kcfd_gg_gradient", C.byref(dev.dm.desc), dev.ndim, P(dev.U_t), P(dev.bcs.tensor("u_type")),
          P(dev.bcs.tensor("u_val")), P(torch.zeros(dev.mesh.n_cells, dev.ndim, dev.ndim, dtype=torch.float64,
                                                     device="cuda")), st)
    gU = torch.zeros(dev.mesh.n_cells, dev.ndim, dev.ndim, dtype=torch.float64, device="cuda")
    _call(dev, "kcfd_gg_gradient", C.byref(dev.dm.desc), dev.ndim, P(dev.U_t), P(dev.bcs.tensor("u_type")),
          P(dev.bcs.tensor("u_val")), P(gU), st)
    gu = gU.cpu().numpy()
    for c in range(dev.ndim):
        _close(gu[:, c, :], ora._grad_U(c))
