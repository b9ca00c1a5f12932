"""Device SIMPLE vs the reference's SIMPLESolver (golden) and the oracle.

The reference solves each linear system with spsolve; the device runs BiCGSTAB. At
rtol 1e-12 the device fields after 20 (2D) / 6 (3D) outer iterations match the
reference's to 1e-10 relative L2 (the plain-form bar). At the configs' rtol 1e-8
the agreement is 1e-6. The mixed form (FP32 inner, FP64 refinement) is checked
against the FP64 form with the same 1e-6 bar.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _cavity(tag, **kw):
    from kcfd import mesh as km, meshgen
    from kcfd.simple import SIMPLESolver
    if tag == "2d":
        nodes, cells, bd = meshgen.quad_box_arrays(0, 0, 1, 1, 8, 8, meshgen.CAVITY_2D_NAMES)
        m = km.build_mesh(nodes, cells, bd)
    else:
        nodes, cells, cf, bd = meshgen.hex_box_arrays(1, 1, 1, 3, 3, 3, meshgen.CAVITY_3D_NAMES)
        m = km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
    s = SIMPLESolver(m, rho=1.0, mu=0.01, **kw)
    for nm in m.boundary_patches:
        s.set_velocity_bc(nm, "dirichlet", [1.0] + [0.0] * (m.ndim - 1) if nm == "lid" else [0.0] * m.ndim)
        s.set_pressure_bc(nm, "zero_gradient")
    s.alpha_u, s.alpha_p, s.tol = 0.7, 0.3, 0.0
    return s


@pytest.mark.parametrize("tag", ["2d", "3d"])
@pytest.mark.parametrize("pc", ["jacobi", "ilu0"])
def test_simple_matches_reference(tag, pc):
    g = load_golden("simple")
    s = _cavity(tag, rtol=1e-12, precond_p=pc)
    s.max_outer_iter = int(g[tag + "_iters"])
    r = s.solve_steady()
    assert _rel(s.U.values, g[tag + "_U"]) < 1e-10
    assert _rel(s.p.values, g[tag + "_p"]) < 1e-10
    np.testing.assert_allclose(r["residuals"], g[tag + "_res"], rtol=1e-6)


@pytest.mark.parametrize("tag", ["2d", "3d"])
def test_simple_rtol_1e8(tag):
    g = load_golden("simple")
    s = _cavity(tag, rtol=1e-8)
    s.max_outer_iter = int(g[tag + "_iters"])
    s.solve_steady()
    assert _rel(s.U.values, g[tag + "_U"]) < 1e-6
    assert _rel(s.p.values, g[tag + "_p"]) < 1e-6


def test_graph_replay_equals_eager():
    a = _cavity("2d", rtol=1e-10)
    b = _cavity("2d", rtol=1e-10, graph=True)
    for s in (a, b):
        s.max_outer_iter = 15
        s.solve_steady()
    np.testing.assert_array_equal(a.U.values, b.U.values)
    np.testing.assert_array_equal(a.p.values, b.p.values)


@pytest.mark.parametrize("tag", ["2d", "3d"])
def test_mixed_matches_fp64(tag):
    a = _cavity(tag, rtol=1e-8)
    b = _cavity(tag, rtol=1e-8, precision="mixed")
    for s in (a, b):
        s.max_outer_iter = 20
        s.solve_steady()
    assert _rel(b.U.values, a.U.values) < 1e-6
    assert _rel(b.p.values, a.p.values) < 1e-6


def test_extensions_match_oracle():
    """MUSCL + over-relaxed non-orthogonal correction on a jittered hex cavity
    (no reference counterpart: parity with the oracle restatement)."""
    from kcfd import mesh as km, meshgen
    from kcfd.simple import SIMPLESolver
    from oracle import mesh as om, simple as osim
    nodes, cells, cf, bd = meshgen.hex_box_arrays(1, 1, 1, 5, 5, 5, meshgen.CAVITY_3D_NAMES)
    nodes = meshgen.jitter_interior(nodes, (5, 5, 5), (0.2, 0.2, 0.2), 0.2, seed=0)
    m = km.build_mesh(nodes, cells, bd, ndim=3, cell_face_node_list=cf)
    ref = om.build_3d(nodes, cells, cf, bd)
    s = SIMPLESolver(m, rho=1.0, mu=0.0025, muscl="van_leer", nonorth=True, rtol=1e-12)
    o = osim.Simple(ref, rho=1.0, mu=0.0025)
    o.muscl, o.nonorth = "van_leer", True
    for x in (s, o):
        osim.cavity_setup(x) if x is o else None
    for nm in m.boundary_patches:
        s.set_velocity_bc(nm, "dirichlet", [1.0, 0, 0] if nm == "lid" else [0.0, 0, 0])
        s.set_pressure_bc(nm, "zero_gradient")
    s.tol = o.tol = 0.0
    s.max_outer_iter = o.max_outer_iter = 5
    s.solve_steady()
    o.solve_steady()
    assert _rel(s.U.values, o.U) < 1e-10
    assert _rel(s.p.values, o.p) < 1e-10
