"""Generate the golden fixtures in tests/golden/ by running the K-CFD reference itself.

Run in a container that holds the reference checkout (it is read, never modified):

    python tests/golden/make_golden.py --ref <reference checkout>   (or KCFD_REFERENCE=<checkout>)

The reference is pure Python. Its mesh package imports ``gmsh`` at module level
without using it (mesh/mesh_generator.py:8), and its verification cases import
matplotlib for plotting only, so both are replaced by empty stub modules before
the import. Every fixture is small (kilobytes) and is written with
numpy.savez_compressed; the tests/test_oracle_*.py files check the oracle against
them and the GPU tests compare the device path with them and reuse the generator
inputs recorded here.
"""
from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _install_stubs():
    sys.modules.setdefault("gmsh", types.ModuleType("gmsh"))
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt
    pc = types.ModuleType("verification.plot_config")
    pc._FONT_NAME = None
    sys.modules["verification.plot_config"] = pc


def _mesh_arrays(mesh, prefix=""):
    F = mesh.n_faces
    ndim = mesh.ndim
    names = list(mesh.boundary_patches.keys())
    ptr = [0]
    fids = []
    for nm in names:
        fids.extend(mesh.boundary_patches[nm])
        ptr.append(len(fids))
    kmax = max(len(c.faces) for c in mesh.cells)
    cf = -np.ones((mesh.n_cells, kmax), dtype=np.int64)
    for ci, c in enumerate(mesh.cells):
        cf[ci, :len(c.faces)] = c.faces
    return {
        prefix + "ndim": np.int64(ndim),
        prefix + "owner": np.array([f.owner for f in mesh.faces], dtype=np.int64),
        prefix + "neighbour": np.array([f.neighbour for f in mesh.faces], dtype=np.int64),
        prefix + "area": np.array([f.area for f in mesh.faces]),
        prefix + "normal": np.array([np.asarray(f.normal)[:ndim] for f in mesh.faces]).reshape(F, ndim),
        prefix + "fcenter": np.array([np.asarray(f.center)[:ndim] for f in mesh.faces]).reshape(F, ndim),
        prefix + "ccenter": np.array([np.asarray(c.center)[:ndim] for c in mesh.cells]),
        prefix + "volume": np.array([c.volume for c in mesh.cells]),
        prefix + "cell_faces": cf,
        prefix + "patch_names": np.array(names),
        prefix + "patch_ptr": np.array(ptr, dtype=np.int64),
        prefix + "patch_fids": np.array(fids, dtype=np.int64),
    }


class _Recorder:
    """Wraps build_fvmesh_from_arrays to record the generator's inputs."""

    def __init__(self, real):
        self.real = real
        self.calls = []

    def __call__(self, node_coords, cell_node_list, boundary_faces_dict, cell_zone_map=None,
                 ndim=2, cell_face_node_list=None):
        self.calls.append((np.array(node_coords), [np.asarray(c) for c in cell_node_list],
                           {k: [np.asarray(f) for f in v] for k, v in boundary_faces_dict.items()},
                           ndim, None if cell_face_node_list is None else
                           [[np.asarray(f) for f in fl] for fl in cell_face_node_list]))
        return self.real(node_coords, cell_node_list, boundary_faces_dict, cell_zone_map=cell_zone_map,
                         ndim=ndim, cell_face_node_list=cell_face_node_list)


def _inputs_arrays(call, prefix="in_"):
    nodes, cells, bdict, ndim, cfl = call
    out = {prefix + "nodes": nodes}
    lens = np.array([len(c) for c in cells], dtype=np.int64)
    out[prefix + "cell_ptr"] = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    out[prefix + "cell_nodes"] = np.concatenate(cells).astype(np.int64)
    names = list(bdict.keys())
    out[prefix + "bnames"] = np.array(names)
    bl = [len(bdict[k]) for k in names]
    out[prefix + "bptr"] = np.concatenate([[0], np.cumsum(bl)]).astype(np.int64)
    bf = [f for k in names for f in bdict[k]]
    out[prefix + "bface_len"] = np.array([len(f) for f in bf], dtype=np.int64)
    out[prefix + "bface_nodes"] = np.concatenate(bf).astype(np.int64) if bf else np.zeros(0, np.int64)
    if cfl is not None:
        nf = np.array([len(fl) for fl in cfl], dtype=np.int64)
        out[prefix + "cface_ptr"] = np.concatenate([[0], np.cumsum(nf)]).astype(np.int64)
        flat = [f for fl in cfl for f in fl]
        out[prefix + "face_len"] = np.array([len(f) for f in flat], dtype=np.int64)
        out[prefix + "face_nodes"] = np.concatenate(flat).astype(np.int64)
    return out


def _system_arrays(system, prefix):
    A = system.to_sparse()
    A.sort_indices()
    return {prefix + "indptr": A.indptr.astype(np.int64), prefix + "indices": A.indices.astype(np.int64),
            prefix + "data": A.data.copy(), prefix + "rhs": system.rhs.copy(), prefix + "diag": system.diag.copy()}


def make_meshes(out):
    import mesh.mesh_generator as mg
    import mesh.mesh_generator_3d as mg3
    import mesh.hybrid_mesh_generator as mgh
    rec = _Recorder(mg.build_fvmesh_from_arrays)
    mg.build_fvmesh_from_arrays = rec
    mg3.build_fvmesh_from_arrays = rec
    mgh.build_fvmesh_from_arrays = rec
    cases = {
        "quad": lambda: mg.generate_channel_mesh(1.0, 0.6, 6, 5),
        "cavity": lambda: mg.generate_cavity_mesh(1.0, 8),
        "tri": lambda: mg.generate_triangle_channel_mesh(1.0, 0.5, 5, 3),
        "hex": lambda: mg3.generate_3d_cavity_mesh(1.0, 0.9, 0.8, 4, 3, 2),
        "hybrid": lambda: mgh.generate_hybrid_hex_tet_mesh(1.0, 0.5, 0.5, 4, 2, 2, 0.5),
    }
    meshes = {}
    for name, fn in cases.items():
        rec.calls.clear()
        m = fn()
        meshes[name] = m
        d = _mesh_arrays(m)
        d.update(_inputs_arrays(rec.calls[0]))
        np.savez_compressed(os.path.join(out, f"mesh_{name}.npz"), **d)
    return meshes


def make_operators(out, meshes):
    from core.fields import ScalarField, VectorField
    from core.fvm_operators import (FVMSystem, diffusion_operator, convection_operator_upwind,
                                    temporal_operator, source_term, linearized_source,
                                    apply_boundary_conditions, under_relax)
    from core.gradient import green_gauss_gradient, least_squares_gradient
    from core.interpolation import compute_mass_flux, muscl_deferred_correction
    for name in ("quad", "tri", "hex", "hybrid"):
        m = meshes[name]
        rng = np.random.default_rng(1234)
        n, F, ndim = m.n_cells, m.n_faces, m.ndim
        d = {}
        gamma = ScalarField(m, "gamma")
        gamma.values = rng.uniform(0.1, 2.0, n)
        phi = ScalarField(m, "phi")
        phi.values = rng.normal(size=n)
        for bn in phi.boundary_values:
            phi.boundary_values[bn] = rng.normal(size=len(phi.boundary_values[bn]))
        U = VectorField(m, "U")
        U.values = rng.normal(size=(n, ndim))
        for bn in U.boundary_values:
            U.boundary_values[bn] = rng.normal(size=U.boundary_values[bn].shape)
        mf = rng.normal(size=F)
        phi_old = rng.normal(size=n)
        S = rng.normal(size=n)
        Sp = -rng.uniform(0.0, 1.0, n)
        Su = rng.normal(size=n)
        d["gamma"], d["phi"], d["U"], d["mf"] = gamma.values, phi.values, U.values, mf
        d["phi_old"], d["S"], d["Sp"], d["Su"] = phi_old, S, Sp, Su
        names = list(m.boundary_patches.keys())
        d["phi_b"] = np.concatenate([phi.boundary_values[k] for k in names])
        d["U_b"] = np.concatenate([U.boundary_values[k] for k in names])
        # boundary condition mix: patch i -> dirichlet / zero_gradient / neumann cyclically
        kinds = ["dirichlet", "zero_gradient", "neumann"]
        bc = {}
        for i, k in enumerate(names):
            t = kinds[i % 3]
            bc[k] = {"type": t, "value": 0.37 * (i + 1)} if t == "neumann" else {"type": t}
        d["bc_kind"] = np.array([bc[k]["type"] for k in names])
        d["bc_value"] = np.array([bc[k].get("value", 0.0) for k in names])
        s = FVMSystem(n); diffusion_operator(m, gamma, s); d.update(_system_arrays(s, "diff_"))
        s = FVMSystem(n); convection_operator_upwind(m, mf, s); d.update(_system_arrays(s, "conv_"))
        s = FVMSystem(n); temporal_operator(m, 1.3, 0.01, phi_old, s); d.update(_system_arrays(s, "temp_"))
        s = FVMSystem(n); source_term(m, S, s); d["src_rhs"] = s.rhs.copy()
        s = FVMSystem(n); linearized_source(m, Sp, Su, s); d.update(_system_arrays(s, "lin_"))
        s = FVMSystem(n); apply_boundary_conditions(m, phi, gamma, mf, s, bc); d.update(_system_arrays(s, "bc_"))
        # a full transport system in the two-fluid order, then under-relaxation
        s = FVMSystem(n)
        diffusion_operator(m, gamma, s)
        convection_operator_upwind(m, mf, s)
        temporal_operator(m, 1.3, 0.01, phi_old, s)
        apply_boundary_conditions(m, phi, gamma, mf, s, bc)
        under_relax(s, phi, 0.7)
        d.update(_system_arrays(s, "full_"))
        d["gg"] = green_gauss_gradient(phi)
        d["lsq"] = least_squares_gradient(phi)
        d["mflux"] = compute_mass_flux(U, 1.7, m)
        for lim in ("minmod", "superbee", "van_albada", "van_leer"):
            d["muscl_" + lim] = muscl_deferred_correction(m, phi, mf, d["gg"], lim)
        np.savez_compressed(os.path.join(out, f"ops_{name}.npz"), **d)


def make_solvers(out):
    import scipy.sparse.linalg as spla
    from core.gpu_solver import _cpu_bicgstab
    from core.preconditioner import create_preconditioner
    from verification.case16_preconditioner import _build_convdiff_system
    from mesh.mesh_generator import generate_channel_mesh
    d = {}
    for nx in (20, 80):
        m = generate_channel_mesh(1.0, 1.0, nx, nx)
        s = _build_convdiff_system(m, gamma_val=0.01, u_conv=1.0)
        A = s.to_sparse()
        b = s.rhs.copy()
        p = f"c16_{nx}_"
        if nx == 20:
            A.sort_indices()
            d[p + "indptr"], d[p + "indices"], d[p + "data"], d[p + "rhs"] = A.indptr, A.indices, A.data, b
        d[p + "direct"] = spla.spsolve(A.tocsc(), b)
        # the reference's case 16 call: bicgstab(atol=1e-10, rtol=0) per preconditioner
        # (verification/case16_preconditioner.py:170-173)
        for pc in ("none", "jacobi", "ilu0"):
            M, _ = create_preconditioner(A, pc)
            cnt = [0]

            def cb(xk):
                cnt[0] += 1

            x, info = spla.bicgstab(A, b, x0=np.zeros(len(b)), atol=1e-10, rtol=0.0, maxiter=2000, M=M,
                                    callback=cb)
            d[p + pc + "_iters"] = np.int64(cnt[0])
            d[p + pc + "_info"] = np.int64(info)
            d[p + pc + "_x"] = x
    # the incumbent GPU path's algorithm (core/gpu_solver.py:158-199) on the 20x20 system
    m = generate_channel_mesh(1.0, 1.0, 20, 20)
    s = _build_convdiff_system(m, gamma_val=0.01, u_conv=1.0)
    A = s.to_sparse()

    class Counting:
        def __init__(self, A):
            self.A, self.n = A, 0

        def __matmul__(self, x):
            self.n += 1
            return self.A @ x

    for tol in (1e-6, 1e-10):
        C = Counting(A)
        x = _cpu_bicgstab(C, s.rhs.copy(), None, tol, 1000)
        d[f"gpu_{tol:.0e}_x"] = x
        d[f"gpu_{tol:.0e}_matvecs"] = np.int64(C.n)
    np.savez_compressed(os.path.join(out, "solvers.npz"), **d)


def make_simple(out):
    from mesh.mesh_generator import generate_cavity_mesh
    from mesh.mesh_generator_3d import generate_3d_cavity_mesh
    from models.single_phase import SIMPLESolver
    import contextlib
    import io
    d = {}
    for tag, mk, mu, iters in (("2d", lambda: generate_cavity_mesh(1.0, 8), 0.01, 20),
                               ("3d", lambda: generate_3d_cavity_mesh(1, 1, 1, 3, 3, 3), 0.01, 6)):
        m = mk()
        sv = SIMPLESolver(m, rho=1.0, mu=mu)
        ndim = m.ndim
        for pname in m.boundary_patches:
            if pname == "lid":
                sv.set_velocity_bc(pname, "dirichlet", [1.0] + [0.0] * (ndim - 1))
            else:
                sv.set_velocity_bc(pname, "dirichlet", [0.0] * ndim)
            sv.set_pressure_bc(pname, "zero_gradient")
        sv.alpha_u, sv.alpha_p, sv.max_outer_iter, sv.tol = 0.7, 0.3, iters, 0.0
        with contextlib.redirect_stdout(io.StringIO()):
            r = sv.solve_steady()
        d[tag + "_U"] = sv.U.values.copy()
        d[tag + "_p"] = sv.p.values.copy()
        d[tag + "_res"] = np.array(r["residuals"])
        d[tag + "_iters"] = np.int64(iters)
    np.savez_compressed(os.path.join(out, "simple.npz"), **d)


def make_c1(out):
    """The reference's own CPU-runnable configuration, exactly: SIMPLESolver on
    generate_cavity_mesh(1.0, 64) (4,096 quads), rho 1, mu 0.01, lid u = 1, no-slip
    walls, zero-gradient pressure, upwind, alpha_u 0.7, alpha_p 0.3, 500 outer
    iterations (tol 0), every system solved by the reference's spsolve
    (models/single_phase.py:265,351). About 3 minutes on one host core."""
    from mesh.mesh_generator import generate_cavity_mesh
    from models.single_phase import SIMPLESolver
    import contextlib
    import io
    m = generate_cavity_mesh(1.0, 64)
    sv = SIMPLESolver(m, rho=1.0, mu=0.01)
    for pname in m.boundary_patches:
        sv.set_velocity_bc(pname, "dirichlet", [1.0, 0.0] if pname == "lid" else [0.0, 0.0])
        sv.set_pressure_bc(pname, "zero_gradient")
    sv.alpha_u, sv.alpha_p, sv.max_outer_iter, sv.tol = 0.7, 0.3, 500, 0.0
    with contextlib.redirect_stdout(io.StringIO()):
        r = sv.solve_steady()
    np.savez_compressed(os.path.join(out, "c1_cavity64.npz"), U=sv.U.values.copy(), p=sv.p.values.copy(),
                        res=np.array(r["residuals"]), iters=np.int64(500))


CHANNEL_MU, CHANNEL_DPDX = 0.01, -1.0


def channel_setup(sv, mesh, H):
    """Poiseuille channel of verification/case1_poiseuille.py:67-99 (and case7): parabolic
    inlet profile per inlet face, zero-gradient velocity and p = 0 at the outlet, no-slip
    walls, u started at half the analytical maximum."""
    ndim = mesh.ndim
    fids = mesh.boundary_patches["inlet"]
    y = np.array([mesh.faces[f].center[1] for f in fids])
    u = np.zeros((len(fids), ndim))
    u[:, 0] = -CHANNEL_DPDX / (2.0 * CHANNEL_MU) * y * (H - y)
    sv.U.boundary_values["inlet"] = u
    sv.set_velocity_bc("inlet", "dirichlet")
    sv.set_velocity_bc("outlet", "zero_gradient")
    for w in ("wall_bottom", "wall_top"):
        sv.set_velocity_bc(w, "dirichlet", [0.0] * ndim)
        sv.set_pressure_bc(w, "zero_gradient")
    sv.set_pressure_bc("inlet", "zero_gradient")
    sv.set_pressure_bc("outlet", "dirichlet", 0.0)
    sv.U.values[:, 0] = -CHANNEL_DPDX * H ** 2 / (8.0 * CHANNEL_MU) * 0.5
    sv.U.values[:, 1] = 0.0


def make_channel(out):
    """SIMPLESolver on the channel set-up of the reference's Poiseuille cases: quads
    (generate_channel_mesh(1.0, 0.1, 20, 8), alpha 0.7 / 0.3) and split-quad triangles
    (generate_triangle_channel_mesh(0.2, 0.1, 8, 4), alpha 0.2 / 0.05), a fixed number of
    outer iterations each (tol 0)."""
    from mesh.mesh_generator import generate_channel_mesh, generate_triangle_channel_mesh
    from models.single_phase import SIMPLESolver
    import contextlib
    import io
    d = {}
    for tag, mk, H, au, ap, iters in (("quad", lambda: generate_channel_mesh(1.0, 0.1, 20, 8), 0.1, 0.7, 0.3, 15),
                                      ("tri", lambda: generate_triangle_channel_mesh(0.2, 0.1, 8, 4), 0.1, 0.2, 0.05,
                                       15)):
        m = mk()
        sv = SIMPLESolver(m, rho=1.0, mu=CHANNEL_MU)
        channel_setup(sv, m, H)
        sv.alpha_u, sv.alpha_p, sv.max_outer_iter, sv.tol = au, ap, iters, 0.0
        with contextlib.redirect_stdout(io.StringIO()):
            r = sv.solve_steady()
        d[tag + "_U"] = sv.U.values.copy()
        d[tag + "_p"] = sv.p.values.copy()
        d[tag + "_res"] = np.array(r["residuals"])
        d[tag + "_iters"] = np.int64(iters)
    # the 3D duct of verification/case5_3d_duct.py:75-112 at 8 x 4 x 4, inlet from the
    # case's own series profile
    from mesh.mesh_generator_3d import generate_3d_duct_mesh
    from verification.case5_3d_duct import analytical_3d_duct
    m = generate_3d_duct_mesh(2.0, 0.1, 0.1, 8, 4, 4)
    sv = SIMPLESolver(m, rho=1.0, mu=CHANNEL_MU)
    fids = m.boundary_patches["inlet"]
    yz = np.array([m.faces[f].center for f in fids])
    u = np.zeros((len(fids), 3))
    u[:, 0] = analytical_3d_duct(yz[:, 1], yz[:, 2], 0.1, 0.1, CHANNEL_DPDX, CHANNEL_MU)
    sv.U.boundary_values["inlet"] = u
    sv.set_velocity_bc("inlet", "dirichlet")
    sv.set_velocity_bc("outlet", "zero_gradient")
    for w in ("wall_bottom", "wall_top", "wall_front", "wall_back"):
        sv.set_velocity_bc(w, "dirichlet", [0.0, 0.0, 0.0])
        sv.set_pressure_bc(w, "zero_gradient")
    sv.set_pressure_bc("inlet", "zero_gradient")
    sv.set_pressure_bc("outlet", "dirichlet", 0.0)
    sv.U.values[:, 0] = -CHANNEL_DPDX * 0.1 ** 2 / (8.0 * CHANNEL_MU) * 0.3
    sv.U.values[:, 1] = 0.0
    sv.U.values[:, 2] = 0.0
    sv.alpha_u, sv.alpha_p, sv.max_outer_iter, sv.tol = 0.7, 0.3, 10, 0.0
    with contextlib.redirect_stdout(io.StringIO()):
        r = sv.solve_steady()
    d["duct_inlet_u"] = u[:, 0].copy()
    d["duct_U"] = sv.U.values.copy()
    d["duct_p"] = sv.p.values.copy()
    d["duct_res"] = np.array(r["residuals"])
    d["duct_iters"] = np.int64(10)
    np.savez_compressed(os.path.join(out, "channel.npz"), **d)


def make_muscl_case(out):
    """The reference's MUSCL verification (verification/case6_muscl.py:136-205): a step
    phi = [x < 0.3] advected at u = 1 on generate_channel_mesh(1.0, 0.02, 100, 1) to
    T = 0.4 at CFL 0.4, once with backward-Euler upwind and once with the van Leer
    deferred correction (2 inner passes per step), each step clipped to [0, 1], by the
    case's own step functions. Stores both final fields and the step count."""
    import contextlib
    import io
    import verification.case6_muscl as c6
    from core.fields import VectorField
    from core.interpolation import compute_mass_flux
    from mesh.mesh_generator import generate_channel_mesh
    mesh = generate_channel_mesh(1.0, 0.02, 100, 1)
    U = VectorField(mesh, name="U")
    U.values[:, 0], U.values[:, 1] = 1.0, 0.0
    for bname, fids in mesh.boundary_patches.items():
        U.boundary_values[bname] = np.zeros((len(fids), 2))
        U.boundary_values[bname][:, 0] = 1.0
    mf = compute_mass_flux(U, 1.0, mesh)
    xc = np.array([c.center[0] for c in mesh.cells])
    phi0 = np.where(xc < 0.3, 1.0, 0.0).astype(np.float64)
    dt = 0.4 * (1.0 / 100) / 1.0
    n_steps = int(np.ceil(0.4 / dt))
    dt = 0.4 / n_steps
    uw, mu = phi0.copy(), phi0.copy()
    with contextlib.redirect_stdout(io.StringIO()):
        for _ in range(n_steps):
            uw = np.clip(c6._solve_upwind_step(mesh, uw, mf, 1.0, dt, 1.0), 0.0, 1.0)
            mu = np.clip(c6._solve_muscl_step(mesh, mu, mf, 1.0, dt, 1.0, n_inner=2), 0.0, 1.0)
    np.savez_compressed(os.path.join(out, "muscl_case.npz"), phi_upwind=uw, phi_muscl=mu, n_steps=np.int64(n_steps),
                        dt=np.float64(dt), width_upwind=np.float64(c6._compute_diffusion_width(xc, uw)),
                        width_muscl=np.float64(c6._compute_diffusion_width(xc, mu)))


def bubble_setup(sv):
    """verification/case4_bubble_column.py:40-69: water-air properties, d_b 5 mm, gravity
    -9.81 along y, alpha_g 0.001 at rest, 300 K, inlet alpha_g 0.04 at U_g = 0.1 m/s up,
    outlet p = 0, walls; relaxation 0.3 / 0.2 / 0.3."""
    sv.rho_l, sv.rho_g, sv.mu_l, sv.mu_g, sv.d_b = 998.2, 1.225, 1.003e-3, 1.789e-5, 0.005
    sv.g = np.array([0.0, -9.81])
    sv.initialize(alpha_g_init=0.001)
    sv.set_inlet_bc("inlet_gas", 0.04, U_l=[0.0, 0.0], U_g=[0.0, 0.1])
    sv.set_outlet_bc("outlet", p_val=0.0)
    for w in ("wall_bottom", "wall_left", "wall_right"):
        sv.set_wall_bc(w)
    sv.alpha_u, sv.alpha_p, sv.alpha_alpha = 0.3, 0.2, 0.3


def make_bubble(out):
    """The bubble column of verification/case4_bubble_column.py on its 8 x 20 mesh: the
    first 5 steps of dt = 0.02 of its solve_transient run, one solve_transient(dt, dt)
    call per step, fields after every step."""
    import contextlib
    import io
    from mesh.mesh_generator import generate_bubble_column_mesh
    from models.two_fluid import TwoFluidSolver
    mesh = generate_bubble_column_mesh(0.15, 0.45, 8, 20)
    sv = TwoFluidSolver(mesh)
    bubble_setup(sv)
    sv.T_l.set_uniform(300.0)
    sv.T_g.set_uniform(300.0)
    sv.dt = 0.02
    d = {}
    for step in range(5):
        with contextlib.redirect_stdout(io.StringIO()):
            r = sv.solve_transient(sv.dt, sv.dt)
        assert r["time_steps"] == 1
        for f in ("alpha_g", "U_l", "U_g", "p"):
            d[f"{step}_{f}"] = getattr(sv, f).values.copy()
        d[f"{step}_res"] = np.array(r["residuals"])
    np.savez_compressed(os.path.join(out, "bubble.npz"), **d)


def two_fluid_setup(sv, mesh, seed):
    """Shared set-up of the two-fluid fixtures (also restated by the oracle and the
    device tests): inlet / outlet / heated bottom wall / adiabatic walls, seeded
    alpha_g in [0.02, 0.08], T_l in [370, 376] K, T_g in [371.15, 375.15] K (both
    sides of T_sat, so evaporation and condensation are active), 6-equation energy."""
    ndim = mesh.ndim
    rng = np.random.default_rng(seed)
    n = mesh.n_cells
    sv.d_b = 0.003
    sv.solve_energy = True
    sv.max_outer_iter = 4
    sv.tol = 1e-12
    sv.dt = 1e-3
    sv.initialize(0.05)
    ul = [0.1] + [0.0] * (ndim - 1)
    ug = [0.2] + [0.0] * (ndim - 1)
    sv.set_inlet_bc("inlet", 0.05, U_l=ul, U_g=ug, T_l=372.0, T_g=373.0)
    sv.set_outlet_bc("outlet", 0.0)
    for nm in mesh.boundary_patches:
        if nm.startswith("wall"):
            sv.set_wall_bc(nm, q_wall=2.0e4 if nm == "wall_bottom" else None)
    ag = rng.uniform(0.02, 0.08, n)
    sv.alpha_g.values = ag.copy()
    sv.alpha_l.values = 1.0 - ag
    sv.T_l.values = 370.0 + rng.uniform(0.0, 6.0, n)
    sv.T_g.values = 373.15 + rng.uniform(-2.0, 2.0, n)
    sv.U_l.values = np.tile(np.array(ul), (n, 1)) * rng.uniform(0.5, 1.5, (n, 1))
    sv.U_g.values = np.tile(np.array(ug), (n, 1)) * rng.uniform(0.5, 1.5, (n, 1))


def make_two_fluid(out, meshes):
    """TwoFluidSolver (models/two_fluid.py) on the quad channel and the hybrid
    hex/tet meshes: 3 time steps of dt = 1e-3 with 4 SIMPLE inner iterations each and
    the 6-equation energy model; fields after every step."""
    from models.two_fluid import TwoFluidSolver
    import contextlib
    import io
    d = {}
    for tag, seed in (("quad", 11), ("hybrid", 12)):
        m = meshes[tag]
        sv = TwoFluidSolver(m)
        two_fluid_setup(sv, m, seed)
        d[tag + "_init_alpha_g"] = sv.alpha_g.values.copy()
        d[tag + "_init_T_l"] = sv.T_l.values.copy()
        d[tag + "_init_T_g"] = sv.T_g.values.copy()
        d[tag + "_init_U_l"] = sv.U_l.values.copy()
        d[tag + "_init_U_g"] = sv.U_g.values.copy()
        for step in range(3):
            with contextlib.redirect_stdout(io.StringIO()):
                r = sv.solve_transient(sv.dt, sv.dt)
            assert r["time_steps"] == 1
            for f in ("alpha_g", "U_l", "U_g", "p", "T_l", "T_g"):
                d[f"{tag}_{step}_{f}"] = getattr(sv, f).values.copy()
            d[f"{tag}_{step}_res"] = np.array(r["residuals"])
    np.savez_compressed(os.path.join(out, "two_fluid.npz"), **d)


def make_partitions(out, meshes):
    """parallel/partitioning.py: RCB part ids and ghost maps of the fixture meshes for
    2-5 parts (the cavity mesh's uniform centres exercise the median ties)."""
    from parallel.partitioning import GeometricPartitioner, GhostCellLayer
    for name, m in meshes.items():
        d = {}
        for n_parts in (2, 3, 4, 5):
            part = GeometricPartitioner(m).partition(n_parts)
            d[f"part{n_parts}"] = np.asarray(part, dtype=np.int64)
            g = GhostCellLayer(m, part)
            trip = [(r, q, c) for r in sorted(g.ghost_map) for q in sorted(g.ghost_map[r])
                    for c in g.ghost_map[r][q]]
            d[f"ghost{n_parts}"] = np.asarray(trip, dtype=np.int64).reshape(-1, 3)
        np.savez_compressed(os.path.join(out, f"part_{name}.npz"), **d)


def make_generators(out):
    """The reference's named generators with non-default arguments: their
    build_fvmesh_from_arrays inputs and the built mesh (gen_<name>.npz)."""
    import mesh.mesh_generator as mg
    import mesh.mesh_generator_3d as mg3
    rec = _Recorder(mg.build_fvmesh_from_arrays)
    mg.build_fvmesh_from_arrays = rec
    mg3.build_fvmesh_from_arrays = rec
    cases = {
        "channel": lambda: mg.generate_channel_mesh(1.2, 0.3, 7, 4),
        "cavity": lambda: mg.generate_cavity_mesh(0.8, 6),
        "tri_channel": lambda: mg.generate_triangle_channel_mesh(1.1, 0.4, 6, 3),
        "bubble_column": lambda: mg.generate_bubble_column_mesh(0.15, 0.45, 9, 12),
        "channel_3d": lambda: mg3.generate_3d_channel_mesh(1.0, 0.5, 0.4, 5, 3, 2),
        "duct_3d": lambda: mg3.generate_3d_duct_mesh(2.0, 0.3, 0.2, 6, 3, 2),
        "cavity_3d": lambda: mg3.generate_3d_cavity_mesh(1.0, 0.7, 0.6, 3, 4, 2),
    }
    for name, fn in cases.items():
        rec.calls.clear()
        m = fn()
        d = _mesh_arrays(m)
        d.update(_inputs_arrays(rec.calls[0]))
        np.savez_compressed(os.path.join(out, f"gen_{name}.npz"), **d)


def make_profiles(out):
    """models/single_phase.py:390-425: velocity profiles through the 8x8 cavity after
    20 outer iterations (the 2d case of make_simple), with the U they were taken from."""
    from mesh.mesh_generator import generate_cavity_mesh
    from models.single_phase import SIMPLESolver
    import contextlib
    import io
    m = generate_cavity_mesh(1.0, 8)
    sv = SIMPLESolver(m, rho=1.0, mu=0.01)
    for pname in m.boundary_patches:
        sv.set_velocity_bc(pname, "dirichlet", [1.0, 0.0] if pname == "lid" else [0.0, 0.0])
        sv.set_pressure_bc(pname, "zero_gradient")
    sv.alpha_u, sv.alpha_p, sv.max_outer_iter, sv.tol = 0.7, 0.3, 20, 0.0
    with contextlib.redirect_stdout(io.StringIO()):
        sv.solve_steady()
    d = {"U": sv.U.values.copy()}
    for tag, (a, b, c) in (("y05", sv.get_velocity_at_y(0.5)), ("y03", sv.get_velocity_at_y(0.3)),
                           ("x05", sv.get_velocity_at_x(0.5)), ("x09", sv.get_velocity_at_x(0.9))):
        d[tag + "_pos"], d[tag + "_u"], d[tag + "_v"] = a, b, c
    np.savez_compressed(os.path.join(out, "profiles.npz"), **d)


def make_time_control(out, meshes):
    """core/time_control.py: compute_dt sequences (CFL- and Fourier-limited steps, the
    growth cap, a non-converged shrink, the clip) on two fixture meshes with seeded
    velocities, plus compute_cfl / compute_fourier arrays."""
    from core.time_control import AdaptiveTimeControl
    d = {}
    for name in ("quad", "hex"):
        m = meshes[name]
        n, nd = m.n_cells, getattr(m, "ndim", 2)
        rng = np.random.default_rng(21)
        ctrl = AdaptiveTimeControl(dt_init=1e-3, dt_min=1e-8, dt_max=0.05, cfl_target=0.5)
        vels, rows = [], []
        for step in range(8):
            vel = rng.normal(size=(n, nd)) * (0.05 if step < 4 else 300.0)
            alpha = 1e-6 if step % 2 == 0 else 50.0
            conv = step != 5
            dt, info = ctrl.compute_dt(m, vel, alpha if step != 7 else None, converged=conv)
            vels.append(vel)
            rows.append([alpha, float(conv), dt, info["cfl_max"], info["fourier_max"],
                         ["cfl", "fourier", "divergence"].index(info["dt_limited_by"])])
        d[f"{name}_vel"] = np.concatenate(vels)
        d[f"{name}_rows"] = np.asarray(rows, dtype=np.float64)
        cmax, carr = ctrl.compute_cfl(m, vels[0], 2e-3)
        fmax, farr = ctrl.compute_fourier(m, 1e-3, 2e-3)
        d[f"{name}_cfl"] = carr
        d[f"{name}_fo"] = farr
        d[f"{name}_cfl1d"] = ctrl.compute_cfl(m, vels[0][:, 0], 2e-3)[1]
    np.savez_compressed(os.path.join(out, "time_control.npz"), **d)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("KCFD_REFERENCE"),
                    help="path of the K-CFD reference checkout (default: $KCFD_REFERENCE)")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default="", help="comma list of fixture groups to write (default: all)")
    a = ap.parse_args()
    if not a.ref:
        ap.error("--ref (or KCFD_REFERENCE) must name the reference checkout")
    _install_stubs()
    sys.path.insert(0, a.ref)
    only = set(x for x in a.only.split(",") if x)
    want = lambda g: not only or g in only
    if only and "meshes" not in only:
        import tempfile
        meshes = make_meshes(tempfile.mkdtemp())  # rebuilt for the other groups, not rewritten
    else:
        meshes = make_meshes(a.out)
    if want("operators"):
        make_operators(a.out, meshes)
    if want("solvers"):
        make_solvers(a.out)
    if want("simple"):
        make_simple(a.out)
    if want("channel"):
        make_channel(a.out)
    if want("c1"):
        make_c1(a.out)
    if want("muscl_case"):
        make_muscl_case(a.out)
    if want("bubble"):
        make_bubble(a.out)
    if want("two_fluid"):
        make_two_fluid(a.out, meshes)
    if want("partitions"):
        make_partitions(a.out, meshes)
    if want("time_control"):
        make_time_control(a.out, meshes)
    if want("generators"):
        make_generators(a.out)
    if want("profiles"):
        make_profiles(a.out)
    print("golden fixtures written to", a.out)


if __name__ == "__main__":
    main()
