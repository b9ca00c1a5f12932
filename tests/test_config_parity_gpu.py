"""Device SIMPLE at the benchmark configurations' own settings, against the reference
and the oracle.

- C1 exactly as benchmarked: the 64^2 quad cavity (4,096 cells), rho 1, mu 0.01,
  upwind, alpha_u 0.7 / alpha_p 0.3, BiCGSTAB + Jacobi for momentum and p', 500
  outer iterations. Compared with the reference's own SIMPLESolver run of the same
  500 iterations (spsolve for every system; tests/golden/c1_cavity64.npz) and with
  the oracle run with the device's solver settings. At a solve tolerance of 1e-12
  every field (u, v, p) agrees to 1e-10 relative L2.
- C2-shaped: the jittered lid-driven cavity at 24^3 (13,824 cells, the 128^3
  workload's generator, seed and physics: Re 400, MUSCL van Leer deferred correction,
  over-relaxed non-orthogonal correction, Green-Gauss gradients, Jacobi for u, v, w
  and ILU(0) or multigrid for p'), 20 outer iterations, on the graph engine (the 128^3
  solve path) and on the automatic team, against the oracle (scipy BiCGSTAB, the
  reference's spilu for p') at a solve tolerance of 1e-12: u, v, w, p each within
  1e-10. MUSCL inside SIMPLE and the non-orthogonal correction have no reference
  counterpart, so this pin is the oracle restatement.
- The reference's channel boundary conditions (verification/case1_poiseuille.py:67-99,
  case5_3d_duct.py:75-112): per-face parabolic inlet, zero-gradient outlet velocity,
  outlet p = 0 and no-slip walls, on 20 x 8 quads, 8 x 4 split-quad triangles and an
  8 x 4 x 4 duct, against the reference's own runs (tests/golden/channel.npz) at 1e-10.
- The mixed form against FP64 on the C2-shaped case, each field within 1e-6.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _device_cavity(m, mu, **kw):
    from kcfd.simple import SIMPLESolver
    s = SIMPLESolver(m, rho=1.0, mu=mu, **kw)
    for nm in m.boundary_patches:
        s.set_velocity_bc(nm, "dirichlet", [1.0] + [0.0] * (m.ndim - 1) if nm == "lid" else [0.0] * m.ndim)
        s.set_pressure_bc(nm, "zero_gradient")
    s.alpha_u, s.alpha_p, s.tol = 0.7, 0.3, 0.0
    return s


@pytest.fixture(scope="module")
def c1_oracle():
    from kcfd import meshgen
    from oracle import mesh as om, simple as osim
    nodes, cells, bd = meshgen.quad_box_arrays(0, 0, 1, 1, 64, 64, meshgen.CAVITY_2D_NAMES)
    o = osim.Simple(om.build_2d(nodes, cells, bd), rho=1.0, mu=0.01)
    osim.cavity_setup(o)
    o.solver, o.rtol, o.precond_u, o.precond_p = "bicgstab", 1e-12, "jacobi", "jacobi"
    o.alpha_u, o.alpha_p, o.max_outer_iter, o.tol = 0.7, 0.3, 500, 0.0
    r = o.solve_steady()
    return (nodes, cells, bd), o, r


def test_c1_500_iterations_match_reference_and_oracle(c1_oracle):
    from kcfd import mesh as km
    (nodes, cells, bd), o, ro = c1_oracle
    g = load_golden("c1_cavity64")
    m = km.build_mesh(nodes, cells, bd)
    s = _device_cavity(m, 0.01, precond_p="jacobi", rtol=1e-12, maxiter=20000, graph=True)
    s.max_outer_iter = int(g["iters"])
    r = s.solve_steady()
    U, p = s.U.values, s.p.values
    for k, name in enumerate("uv"):
        assert _rel(U[:, k], g["U"][:, k]) < 1e-10, name
        assert _rel(U[:, k], o.U[:, k]) < 1e-10, name
    assert _rel(p, g["p"]) < 1e-10
    assert _rel(p, o.p) < 1e-10
    # the residual history of all 500 iterations follows the reference's
    np.testing.assert_allclose(r["residuals"], g["res"], rtol=1e-6)
    np.testing.assert_allclose(r["residuals"], ro["residuals"], rtol=1e-6)


def _c2_case(N=24):
    from kcfd import meshgen
    nodes, cells, cf, bd = meshgen.hex_box_arrays(1.0, 1.0, 1.0, N, N, N, meshgen.CAVITY_3D_NAMES)
    nodes = meshgen.jitter_interior(nodes, (N, N, N), (1.0 / N,) * 3, 0.2, seed=0)
    return nodes, cells, cf, bd


@pytest.fixture(scope="module")
def c2_oracle():
    from oracle import mesh as om, simple as osim
    nodes, cells, cf, bd = _c2_case()
    o = osim.Simple(om.build_3d(nodes, cells, cf, bd), rho=1.0, mu=0.0025)
    osim.cavity_setup(o)
    o.muscl, o.nonorth = "van_leer", True
    o.solver, o.rtol, o.precond_u, o.precond_p = "bicgstab", 1e-12, "jacobi", "spilu"
    o.alpha_u, o.alpha_p, o.max_outer_iter, o.tol = 0.7, 0.3, 20, 0.0
    r = o.solve_steady()
    return (nodes, cells, cf, bd), o, r


@pytest.mark.parametrize("team,pc", [(3, "ilu0"), (0, "ilu0"), (3, "amg")])
def test_c2_shaped_matches_oracle(c2_oracle, team, pc):
    from kcfd import mesh as km
    (nodes, cells, cf, bd), o, ro = c2_oracle
    m = km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
    s = _device_cavity(m, 0.0025, precond_p=pc, ilu_order="color", rtol=1e-12, maxiter=20000,
                       muscl="van_leer", nonorth=True, graph=True, team=team)
    if team == 3:
        assert s.s_p.graph_engine and s.s_m.graph_engine
    s.max_outer_iter = 20
    r = s.solve_steady()
    U, p = s.U.values, s.p.values
    for k, name in enumerate("uvw"):
        assert _rel(U[:, k], o.U[:, k]) < 1e-10, name
    assert _rel(p, o.p) < 1e-10
    np.testing.assert_allclose(r["residuals"], ro["residuals"], rtol=1e-6)


def test_c2_shaped_mixed_field_errors():
    """Mixed form (FP32 inner iterations, FP64 residuals and refinement) against the
    FP64 form on the C2-shaped case at the benchmark's 1e-8: u, v, w, p each <= 1e-6."""
    from kcfd import mesh as km
    nodes, cells, cf, bd = _c2_case()
    m = km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
    out = {}
    for prec in ("fp64", "mixed"):
        s = _device_cavity(m, 0.0025, precision=prec, precond_p="ilu0", rtol=1e-8, maxiter=20000,
                           muscl="van_leer", nonorth=True, graph=True)
        s.max_outer_iter = 20
        s.solve_steady()
        out[prec] = (s.U.values, s.p.values)
    (Ua, pa), (Ub, pb) = out["fp64"], out["mixed"]
    for k, name in enumerate("uvw"):
        assert _rel(Ub[:, k], Ua[:, k]) < 1e-6, name
    assert _rel(pb, pa) < 1e-6


CH_MU, CH_DPDX = 0.01, -1.0


def _channel_device(m, H, alpha_u, alpha_p, inlet_u):
    from kcfd.simple import SIMPLESolver
    D = m.ndim
    s = SIMPLESolver(m, rho=1.0, mu=CH_MU, precond_p="jacobi", rtol=1e-12, maxiter=20000)
    z = np.zeros((len(inlet_u), D))
    z[:, 0] = inlet_u
    s.set_velocity_bc("inlet", "dirichlet", z)
    s.set_velocity_bc("outlet", "zero_gradient")
    walls = [nm for nm in m.boundary_patches if nm.startswith("wall")]
    for w in walls:
        s.set_velocity_bc(w, "dirichlet", [0.0] * D)
        s.set_pressure_bc(w, "zero_gradient")
    s.set_pressure_bc("inlet", "zero_gradient")
    s.set_pressure_bc("outlet", "dirichlet", 0.0)
    s.alpha_u, s.alpha_p, s.tol = alpha_u, alpha_p, 0.0
    return s


@pytest.mark.parametrize("tag", ["quad", "tri"])
def test_channel_bcs_match_reference(tag):
    from kcfd import mesh as km, meshgen
    g = load_golden("channel")
    H = 0.1
    if tag == "quad":
        arrays, au, ap = meshgen.quad_box_arrays(0.0, 0.0, 1.0, H, 20, 8, meshgen.CHANNEL_2D_NAMES), 0.7, 0.3
    else:
        arrays, au, ap = meshgen.tri_channel_arrays(0.2, H, 8, 4), 0.2, 0.05
    m = km.build_mesh(*arrays)
    y = np.asarray(m.fcenter)[m.boundary_patches["inlet"], 1]
    s = _channel_device(m, H, au, ap, -CH_DPDX / (2.0 * CH_MU) * y * (H - y))
    U0 = np.zeros((m.n_cells, 2))
    U0[:, 0] = -CH_DPDX * H ** 2 / (8.0 * CH_MU) * 0.5
    s.U.values = U0
    s.max_outer_iter = int(g[tag + "_iters"])
    r = s.solve_steady()
    assert _rel(s.U.values, g[tag + "_U"]) < 1e-10
    assert _rel(s.p.values, g[tag + "_p"]) < 1e-10
    np.testing.assert_allclose(r["residuals"], g[tag + "_res"], rtol=1e-6)


def test_duct_bcs_match_reference():
    from kcfd import mesh as km, meshgen
    g = load_golden("channel")
    nodes, cells, cf, bd = meshgen.hex_box_arrays(2.0, 0.1, 0.1, 8, 4, 4, meshgen.CHANNEL_3D_NAMES)
    m = km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
    s = _channel_device(m, 0.1, 0.7, 0.3, g["duct_inlet_u"])
    U0 = np.zeros((m.n_cells, 3))
    U0[:, 0] = -CH_DPDX * 0.1 ** 2 / (8.0 * CH_MU) * 0.3
    s.U.values = U0
    s.max_outer_iter = int(g["duct_iters"])
    r = s.solve_steady()
    assert _rel(s.U.values, g["duct_U"]) < 1e-10
    assert _rel(s.p.values, g["duct_p"]) < 1e-10
    np.testing.assert_allclose(r["residuals"], g["duct_res"], rtol=1e-6)
