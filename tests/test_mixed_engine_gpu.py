"""The graph engine's MIXED form (FP32 Krylov vectors and values, FP64 iterate,
residual replacement against the FP64 matrix) against its FP64 form.

Both stop on the same FP64 relative residual, so: the mixed solve's true residual
b - A x (recomputed here on the host in FP64) meets rtol, its solution agrees with
the FP64 engine's within 1e-8 relative L2 at rtol 1e-10 (the residual bound times
these systems' conditioning), and its Krylov count stays within 1.5x + 3 of the FP64
count (the FP32 recursion converges like the FP64 one between replacements)."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _hex_system(nx, seed):
    from kcfd import meshgen
    from oracle import mesh as om, fvm
    n, c, f, b = meshgen.hex_box_arrays(1, 1, 1, nx, nx, nx, meshgen.CAVITY_3D_NAMES)
    m = om.build_3d(n, c, f, b)
    rng = np.random.default_rng(seed)
    s = fvm.System(m.n_cells)
    fvm.diffusion_operator(m, rng.uniform(0.5, 2.0, m.n_cells), s)
    fvm.convection_operator_upwind(m, rng.normal(size=m.n_faces) * m.area, s)
    fvm.temporal_operator(m, 1.0, 10.0, np.zeros(m.n_cells), s)
    return s.to_sparse(), (n, c, f, b)


def _colors(arrays):
    from kcfd import mesh as km
    n, c, f, b = arrays
    return km.build_mesh(n, c, b, ndim=3, cell_face_node_list=f).cell_color


def _solve(d, B, pc, mode, rtol, nrhs, lev, maxiter=5000):
    import torch
    from kcfd.solver import Solver
    s = Solver(d, precond=pc, mode=mode, rtol=rtol, maxiter=maxiter, team=3, nrhs=nrhs, levels=lev)
    assert s.info()["team"] == 3
    s.setup(d)
    bb = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    x = torch.zeros_like(bb)
    it, rr, st = s.solve(d, bb, x)
    return x.cpu().numpy(), it.cpu().numpy().copy(), rr.cpu().numpy().copy(), st.cpu().numpy().copy()


@pytest.mark.parametrize("pc", ["none", "jacobi", "ilu0"])
@pytest.mark.parametrize("nrhs", [1, 3])
def test_mixed_engine_meets_the_fp64_stopping_test(pc, nrhs):
    from kcfd import _lib
    from kcfd.solver import DeviceCSR
    A, arrays = _hex_system(24, seed=31)
    lev = _colors(arrays) if pc == "ilu0" else None
    d = DeviceCSR.from_scipy(A)
    rng = np.random.default_rng(5)
    B = rng.normal(size=(A.shape[0], nrhs))
    if nrhs == 3:
        B[:, 2] *= 1e-3
    else:
        B = B[:, 0]
    for rtol in (1e-8, 1e-10, 1e-12):
        x64, it64, _, st64 = _solve(d, B, pc, _lib.MODE_FP64, rtol, nrhs, lev)
        x32, it32, rr32, st32 = _solve(d, B, pc, _lib.MODE_MIXED, rtol, nrhs, lev)
        assert list(st64) == [0] * nrhs and list(st32) == [0] * nrhs, (rtol, st64, st32)
        X32 = x32.reshape(A.shape[0], nrhs)
        BB = np.asarray(B).reshape(A.shape[0], nrhs)
        for c in range(nrhs):
            true_rel = np.linalg.norm(BB[:, c] - A @ X32[:, c]) / np.linalg.norm(BB[:, c])
            assert true_rel < 1.5 * rtol, (pc, nrhs, rtol, c, true_rel)
            # the reported residual is the replaced (true) one, up to the rounding of
            # b - A x itself (a few per cent of a 1e-12 residual)
            assert abs(rr32[c] - true_rel) <= 0.05 * true_rel + 0.01 * rtol, (rr32[c], true_rel)
            assert it32[c] <= 1.5 * it64[c] + 3, (pc, nrhs, rtol, c, it32[c], it64[c])
        if rtol == 1e-10:
            assert _rel(x32, x64) < 1e-8, (pc, nrhs, _rel(x32, x64))


def test_mixed_engine_eager_form_is_bitwise_equal(monkeypatch):
    """The eager form launches the same kernels (replacement kernel included)."""
    from kcfd import _lib
    from kcfd.solver import DeviceCSR
    A, arrays = _hex_system(20, seed=17)
    lev = _colors(arrays)
    d = DeviceCSR.from_scipy(A)
    b = np.random.default_rng(3).normal(size=A.shape[0])
    for pc, lv in (("jacobi", None), ("ilu0", lev)):
        out = []
        for eager in ("0", "1"):
            monkeypatch.setenv("KCFD_ENGINE_EAGER", eager)
            out.append(_solve(d, b, pc, _lib.MODE_MIXED, 1e-10, 1, lv))
        assert int(out[0][1][0]) == int(out[1][1][0]) and int(out[0][3][0]) == int(out[1][3][0]) == 0
        np.testing.assert_array_equal(out[0][0], out[1][0])


def test_mixed_engine_maxiter_and_repeat():
    """An iteration cap ends with MAXITER and a true residual; repeated solves are
    bitwise the same."""
    from kcfd import _lib
    from kcfd.solver import DeviceCSR
    A, _ = _hex_system(20, seed=13)
    d = DeviceCSR.from_scipy(A)
    b = np.random.default_rng(4).normal(size=A.shape[0])
    x1, it1, rr1, st1 = _solve(d, b, "jacobi", _lib.MODE_MIXED, 1e-12, 1, None)
    x2, it2, _, st2 = _solve(d, b, "jacobi", _lib.MODE_MIXED, 1e-12, 1, None)
    np.testing.assert_array_equal(x1, x2)
    assert int(it1[0]) == int(it2[0])
    x3, it3, rr3, st3 = _solve(d, b, "jacobi", _lib.MODE_MIXED, 1e-14, 1, None, maxiter=5)
    assert int(st3[0]) == 1 and int(it3[0]) == 5
    true_rel = np.linalg.norm(b - A @ x3) / np.linalg.norm(b)
    assert abs(rr3[0] - true_rel) <= 1e-6 * true_rel


def test_mixed_simple_on_the_engine():
    """SIMPLE's mixed form on a 256^2 cavity (65,536 cells): the momentum solve (2
    right-hand sides) runs the engine's FP32 form; p' runs FP64 with ILU(0) (above
    4,096 cells) or an FP64 Krylov iteration over an FP32 hierarchy (multigrid); after
    5 outer iterations every solve met its FP64 stopping test and the fields agree with
    the FP64 run within 1e-6 relative L2."""
    import torch
    from kcfd import mesh as km, meshgen
    from kcfd.simple import SIMPLESolver
    N = 256
    nodes, cells, bd = meshgen.quad_box_arrays(0, 0, 1, 1, N, N, meshgen.CAVITY_2D_NAMES)
    m = km.build_mesh(nodes, cells, bd)
    for pc in ("ilu0", "amg"):
        runs = {}
        for prec in ("fp64", "mixed"):
            s = SIMPLESolver(m, rho=1.0, mu=0.01, precision=prec, precond_p=pc, rtol=1e-8, graph=True)
            assert s.s_m.graph_engine
            for nm in m.boundary_patches:
                s.set_velocity_bc(nm, "dirichlet", [1.0, 0.0] if nm == "lid" else [0.0, 0.0])
                s.set_pressure_bc(nm, "zero_gradient")
            s.max_outer_iter, s.tol = 5, 0.0
            s.solve_steady()
            torch.cuda.synchronize()
            assert int(s.s_p.status[0]) == 0 and list(s.s_m.status.cpu().numpy()) == [0, 0], (pc, prec)
            runs[prec] = (s.U.values.copy(), s.p.values.copy())
        for k in range(2):
            assert _rel(runs["mixed"][k], runs["fp64"][k]) < 1e-6, (pc, k, _rel(runs["mixed"][k], runs["fp64"][k]))
