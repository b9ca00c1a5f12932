"""The oracle's SIMPLE restatement against the reference's own verification criteria.
Host only.

Poiseuille flow between plates, u(y) = -dpdx / (2 mu) y (H - y), with a parabolic inlet,
outlet p = 0, no-slip walls, started from u = u_max / 2:

- case 1 (verification/case1_poiseuille.py:47-99,119): 50 x 20 quads, L = 1, H = 0.1,
  alpha_u 0.7, alpha_p 0.3, at most 500 outer iterations to 1e-5. The profile is
  SIMPLESolver.get_velocity_at_y(0.8) (models/single_phase.py:390-405). Passes when
  the relative L2 error is below 1 %.
- case 7 (verification/case7_unstructured.py:38-112): 20 x 10 split quads (400
  triangles), Lx = 0.2, Ly = 0.1, alpha_u 0.2, alpha_p 0.05, at most 3000 iterations
  to 1e-4. The profile is every cell within 2 dx of x = 0.8 Lx. Passes below 10 %.

- case 22 (verification/case22_hybrid_mesh.py:64-131): the same duct on 16 x 4 x 4
  columns, hexes on the low-x half and 12 tets per column cell on the high-x half,
  at most 300 iterations to 1e-3. Passes below 10 %.
- case 14 (verification/case14_3d_cavity.py:38-110,180-186): the 12^3 lid-driven
  cavity at Re 100, alpha_u 0.5, alpha_p 0.2, at most 500 iterations to 1e-3. The
  vertical centreline (cells within 1.5 dx of x = z = 0.5) must recirculate: mean u
  above y = 0.7 positive, between y = 0.3 and 0.6 negative.
- case 5 (verification/case5_3d_duct.py:21-63,75-131): a 2 x 0.1 x 0.1 duct of 20 x 8 x 8
  hexes with the case's series profile at the inlet, alpha_u 0.7, alpha_p 0.3, at most
  500 iterations to 1e-4, cells within 1.5 dx of x = 0.8 Lx. Passes below 5 %.

The relative L2 is sqrt(mean((u - u_exact)^2)) / max|u_exact|, as in every case."""
import numpy as np

from kcfd import meshgen
from oracle import mesh as om, simple as osim

MU, DPDX = 0.01, -1.0


def exact(y, H):
    return -DPDX / (2.0 * MU) * y * (H - y)


def poiseuille(nodes, cells, bd, H, alpha_u, alpha_p, max_iter, tol):
    m = om.build_2d(nodes, cells, bd)
    o = osim.Simple(m, rho=1.0, mu=MU)
    y_in = m.fcenter[m.boundary_patches["inlet"], 1]
    o.set_velocity_bc("inlet", "dirichlet", np.c_[exact(y_in, H), np.zeros_like(y_in)])
    o.set_velocity_bc("outlet", "zero_gradient")
    for w in ("wall_bottom", "wall_top"):
        o.set_velocity_bc(w, "dirichlet", [0.0, 0.0])
        o.set_pressure_bc(w, "zero_gradient")
    o.set_pressure_bc("inlet", "zero_gradient")
    o.set_pressure_bc("outlet", "dirichlet", 0.0)
    o.U[:, 0] = -DPDX * H ** 2 / (8.0 * MU) * 0.5
    o.U[:, 1] = 0.0
    o.alpha_u, o.alpha_p, o.max_outer_iter, o.tol = alpha_u, alpha_p, max_iter, tol
    return m, o, o.solve_steady()


def duct_exact(y, z, H, W, terms=20):
    """The series profile of verification/case5_3d_duct.py:21-63 on [0, H] x [0, W]: the
    rectangular-duct Poiseuille series in the centred coordinates, scaled as that case
    scales it (4 G a^2 / (mu pi^3), a = H / 2) and floored at 0."""
    a, b = H / 2.0, W / 2.0
    yc, zc = y - a, z - b
    s = np.zeros_like(y)
    for k in range(terms):
        m = 2 * k + 1
        lam = m * np.pi / (2 * a)
        den = np.cosh(lam * b)
        ratio = np.where(den > 1e200, 0.0, np.cosh(lam * zc) / np.maximum(den, 1e-30))
        s += (-1) ** k / m ** 3 * (1.0 - ratio) * np.cos(m * np.pi * yc / (2 * a))
    return np.maximum(s * 4.0 * (-DPDX) * a ** 2 / (MU * np.pi ** 3), 0.0)


def duct(nx, ny, nz, max_iter, tol, Lx=2.0, H=0.1, W=0.1, arrays=None):
    nodes, cells, cf, bd = arrays or meshgen.hex_box_arrays(Lx, H, W, nx, ny, nz, meshgen.CHANNEL_3D_NAMES)
    m = om.build_3d(nodes, cells, cf, bd)
    o = osim.Simple(m, rho=1.0, mu=MU)
    fi = m.boundary_patches["inlet"]
    u_in = duct_exact(m.fcenter[fi, 1], m.fcenter[fi, 2], H, W)
    z = np.zeros_like(u_in)
    o.set_velocity_bc("inlet", "dirichlet", np.c_[u_in, z, z])
    o.set_velocity_bc("outlet", "zero_gradient")
    for w in ("wall_bottom", "wall_top", "wall_front", "wall_back"):
        o.set_velocity_bc(w, "dirichlet", [0.0, 0.0, 0.0])
        o.set_pressure_bc(w, "zero_gradient")
    o.set_pressure_bc("inlet", "zero_gradient")
    o.set_pressure_bc("outlet", "dirichlet", 0.0)
    o.U[:, 0] = -DPDX * H ** 2 / (8.0 * MU) * 0.3
    o.alpha_u, o.alpha_p, o.max_outer_iter, o.tol = 0.7, 0.3, max_iter, tol
    return m, o, u_in, o.solve_steady()


def rel_l2(u, y, H):
    ue = exact(y, H)
    return np.sqrt(np.mean((u - ue) ** 2)) / max(np.max(np.abs(ue)), 1e-15)


def test_case1_poiseuille_quads():
    H = 0.1
    nodes, cells, bd = meshgen.quad_box_arrays(0.0, 0.0, 1.0, H, 50, 20, meshgen.CHANNEL_2D_NAMES)
    m, o, res = poiseuille(nodes, cells, bd, H, 0.7, 0.3, 500, 1e-5)
    # get_velocity_at_y(0.8): dx from the first internal face with a nonzero x offset
    it = np.nonzero(m.neighbour >= 0)[0]
    dxs = np.abs(m.ccenter[m.owner[it], 0] - m.ccenter[m.neighbour[it], 0])
    dx = dxs[np.nonzero(dxs > 1e-10)[0][0]]
    sel = np.abs(m.ccenter[:, 0] - 0.8) < 1.5 * dx
    assert sel.sum() == 40  # the two columns either side of x = 0.8
    err = rel_l2(o.U[sel, 0], m.ccenter[sel, 1], H)
    assert err < 0.01, (err, res["iterations"])


def test_case7_poiseuille_triangles():
    Lx, Ly, nx = 0.2, 0.1, 20
    nodes, cells, bd = meshgen.tri_channel_arrays(Lx, Ly, nx, 10)
    m, o, res = poiseuille(nodes, cells, bd, Ly, 0.2, 0.05, 3000, 1e-4)
    sel = np.abs(m.ccenter[:, 0] - 0.8 * Lx) < Lx / nx * 2.0
    assert sel.sum() > 0
    err = rel_l2(o.U[sel, 0], m.ccenter[sel, 1], Ly)
    assert err < 0.10, (err, res["iterations"])


def test_channel_matches_reference_run():
    """The same channel set-up against the reference's own SIMPLESolver run
    (tests/golden/channel.npz, written by tests/golden/make_golden.py --only channel):
    outlet p = 0, zero-gradient outlet velocity and a per-face inlet profile, paths the
    cavity fixtures do not reach."""
    from conftest import load_golden
    g = load_golden("channel")
    for tag, arrays, H, au, ap in (("quad", meshgen.quad_box_arrays(0.0, 0.0, 1.0, 0.1, 20, 8, meshgen.CHANNEL_2D_NAMES),
                                    0.1, 0.7, 0.3),
                                   ("tri", meshgen.tri_channel_arrays(0.2, 0.1, 8, 4), 0.1, 0.2, 0.05)):
        m, o, res = poiseuille(*arrays, H, au, ap, int(g[tag + "_iters"]), 0.0)
        for mine, ref in ((o.U, g[tag + "_U"]), (o.p, g[tag + "_p"])):
            assert np.linalg.norm(mine - ref) <= 1e-10 * np.linalg.norm(ref), tag
        np.testing.assert_allclose(res["residuals"], g[tag + "_res"], rtol=1e-8)


def test_case6_muscl_step_advection():
    """verification/case6_muscl.py:136-223 on the oracle's operators: a step phi = [x < 0.3]
    advected at u = 1 on a 100 x 1 channel to T = 0.4 (CFL 0.4), backward Euler with upwind,
    and with the van Leer deferred correction (2 inner passes per step), each step clipped
    to [0, 1]. Both final fields equal the reference's own run (tests/golden/muscl_case.npz),
    and MUSCL's 10-90 % front is no wider than upwind's, the case's pass criterion."""
    import scipy.sparse.linalg as spla
    from conftest import load_golden
    from oracle import fvm as of
    g = load_golden("muscl_case")
    nodes, cells, bd = meshgen.quad_box_arrays(0.0, 0.0, 1.0, 0.02, 100, 1, meshgen.CHANNEL_2D_NAMES)
    m = om.build_2d(nodes, cells, bd)
    n = m.n_cells
    U = np.c_[np.ones(n), np.zeros(n)]
    Ub = np.zeros((m.n_faces, 2))
    Ub[:, 0] = 1.0
    mf = of.compute_mass_flux(m, U, Ub, 1.0)
    phi0 = np.where(m.ccenter[:, 0] < 0.3, 1.0, 0.0)
    dt, n_steps = float(g["dt"]), int(g["n_steps"])
    inlet = m.boundary_patches["inlet"]
    phi_b = {nm: (1.0 if nm == "inlet" else 0.0) for nm in m.boundary_patches}

    def system_for(phi_old):
        s = of.System(n)
        of.temporal_operator(m, 1.0, dt, phi_old, s)
        of.convection_operator_upwind(m, mf, s)
        F = mf[inlet]
        neg = F < 0  # inflow through the inlet: the case adds -F phi_b to the rhs
        s.add_source(m.owner[inlet][neg], -F[neg] * 1.0)
        return s

    def solve(s):
        return np.clip(spla.spsolve(s.to_sparse(), s.rhs), 0.0, 1.0)

    uw, mu = phi0.copy(), phi0.copy()
    for _ in range(n_steps):
        uw = solve(system_for(uw))
        cur = mu.copy()
        for _ in range(2):
            grad = of.green_gauss_gradient(m, cur, of.face_patch_values(m, phi_b, cur))
            s = system_for(mu)
            s.rhs += of.muscl_deferred_correction(m, cur, mf, grad, "van_leer")
            cur = solve(s)
        mu = cur
    np.testing.assert_allclose(uw, g["phi_upwind"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(mu, g["phi_muscl"], rtol=0, atol=1e-12)

    def width(phi):
        x = m.ccenter[(phi >= 0.1) & (phi <= 0.9), 0]
        return float(x[-1] - x[0]) if len(x) > 1 else 0.0

    assert width(mu) <= width(uw)
    assert abs(width(uw) - float(g["width_upwind"])) < 1e-12 and abs(width(mu) - float(g["width_muscl"])) < 1e-12


def test_case5_duct():
    Lx, H, W = 2.0, 0.1, 0.1
    m, o, _, res = duct(20, 8, 8, 500, 1e-4)
    sel = np.abs(m.ccenter[:, 0] - 0.8 * Lx) < Lx / 20 * 1.5
    ue = duct_exact(m.ccenter[sel, 1], m.ccenter[sel, 2], H, W)
    err = np.sqrt(np.mean((o.U[sel, 0] - ue) ** 2)) / max(np.max(np.abs(ue)), 1e-15)
    assert err < 0.05, (err, res["iterations"])


def test_duct_matches_reference_run():
    """8 x 4 x 4 duct, 10 outer iterations, against the reference's own run
    (tests/golden/channel.npz): the inlet series equals the case's function and the
    fields agree to 1e-10 (3D outlet p = 0 and zero-gradient velocity)."""
    from conftest import load_golden
    g = load_golden("channel")
    m, o, u_in, res = duct(8, 4, 4, int(g["duct_iters"]), 0.0)
    np.testing.assert_allclose(u_in, g["duct_inlet_u"], rtol=1e-13, atol=1e-16)
    for mine, ref in ((o.U, g["duct_U"]), (o.p, g["duct_p"])):
        assert np.linalg.norm(mine - ref) <= 1e-10 * np.linalg.norm(ref)
    np.testing.assert_allclose(res["residuals"], g["duct_res"], rtol=1e-8)


def test_case22_hybrid_duct():
    Lx, H, W = 2.0, 0.1, 0.1
    arrays = meshgen.hybrid_hex_tet_arrays(Lx, H, W, 16, 4, 4, tet_fraction=0.5)
    m, o, _, res = duct(16, 4, 4, 300, 1e-3, arrays=arrays)
    sel = np.abs(m.ccenter[:, 0] - 0.8 * Lx) < Lx / 16 * 1.5
    ue = duct_exact(m.ccenter[sel, 1], m.ccenter[sel, 2], H, W)
    err = np.sqrt(np.mean((o.U[sel, 0] - ue) ** 2)) / np.max(np.abs(ue))
    assert err < 0.10, (err, res["iterations"])


def test_case14_cavity_recirculates():
    nodes, cells, cf, bd = meshgen.hex_box_arrays(1.0, 1.0, 1.0, 12, 12, 12, meshgen.CAVITY_3D_NAMES)
    m = om.build_3d(nodes, cells, cf, bd)
    o = osim.Simple(m, rho=1.0, mu=0.01)
    osim.cavity_setup(o)
    o.alpha_u, o.alpha_p, o.max_outer_iter, o.tol = 0.5, 0.2, 500, 1e-3
    o.solve_steady()
    c = m.ccenter
    sel = (np.abs(c[:, 0] - 0.5) < 1.5 / 12) & (np.abs(c[:, 2] - 0.5) < 1.5 / 12)
    y, u = c[sel, 1], o.U[sel, 0]
    assert np.mean(u[y > 0.7]) > 0 and np.mean(u[(y > 0.3) & (y < 0.6)]) < 0


def test_case4_bubble_column_matches_reference_run():
    """verification/case4_bubble_column.py:40-114 on the oracle's two-fluid model: the
    8 x 20 bubble column (inlet alpha_g 0.04 at 0.1 m/s through the middle third of the
    bottom, outlet p = 0, walls), its first 5 steps of dt = 0.02 against the reference's
    own run (tests/golden/bubble.npz, one solve_transient(dt, dt) per step) to 1e-10, and
    the case's physical-validity check on the result (alpha_g <= 1, mean alpha_g < 0.5)."""
    from conftest import load_golden
    from oracle.two_fluid import TwoFluid
    g = load_golden("bubble")
    nodes, cells, bd = meshgen.bubble_column_arrays(0.15, 0.45, 8, 20)
    o = TwoFluid(om.build_2d(nodes, cells, bd))
    o.rho_l, o.rho_g, o.mu_l, o.mu_g, o.d_b = 998.2, 1.225, 1.003e-3, 1.789e-5, 0.005
    o.g = np.array([0.0, -9.81])
    o.initialize(alpha_g_init=0.001)
    o.set_inlet_bc("inlet_gas", 0.04, U_l=[0.0, 0.0], U_g=[0.0, 0.1])
    o.set_outlet_bc("outlet", p_val=0.0)
    for w in ("wall_bottom", "wall_left", "wall_right"):
        o.set_wall_bc(w)
    o.alpha_u, o.alpha_p, o.alpha_alpha = 0.3, 0.2, 0.3
    o._set_uniform("T_l", 300.0)
    o._set_uniform("T_g", 300.0)
    for step in range(5):
        res = o.step(0.02)
        assert abs(res - g[f"{step}_res"][0]) <= 1e-6 * abs(g[f"{step}_res"][0])
        for f in ("alpha_g", "U_l", "U_g", "p"):
            ref = g[f"{step}_{f}"]
            assert np.linalg.norm(o.v[f] - ref) <= 1e-10 * max(np.linalg.norm(ref), 1e-300), (step, f)
    a = o.v["alpha_g"]
    assert a.max() <= 1.0 and a.mean() < 0.5
