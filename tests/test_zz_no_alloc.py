"""The allocation-free BiCGSTAB entry point (kcfd_bicgstab_noalloc) against the
handle-based one (kcfd_solver_create / kcfd_solver_solve).

Callers that cannot allocate device memory -- real-time loops that must not block on
the device allocator, host programs whose device memory is owned by someone else --
use the no-alloc entry point; its Krylov scratch is a fixed array inside libkcfd that
every call shares and that keeps the last call's contents. This file is collected
last so that a run stopping at the first failure has already run every other test.
Both entry points run the same single-CTA FP64 kernel, so their solutions must agree
to the 1e-12 relative L2 tolerance used for same-algorithm comparisons elsewhere.
"""
import ctypes as C

import numpy as np
import pytest

from case16 import channel_mesh, convdiff_system

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
    return s.to_sparse(), rng.normal(size=m.n_cells)


def _noalloc(csr, b, x0, precond, rtol, maxiter=5000):
    import torch
    from kcfd import _lib
    bd = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    xd = torch.from_numpy(np.ascontiguousarray(x0)).cuda()
    it = torch.zeros(1, dtype=torch.int32, device="cuda")
    rr = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    d = csr.desc()
    _lib.check(_lib.lib().kcfd_bicgstab_noalloc(C.byref(d), _lib.ptr(bd), _lib.ptr(xd), _lib.PREC[precond],
                                                _lib.STOP_SCIPY, rtol, 0.0, maxiter, _lib.ptr(it), _lib.ptr(rr),
                                                _lib.ptr(st), _lib.stream_handle()), "kcfd_bicgstab_noalloc")
    torch.cuda.synchronize()
    return xd.cpu().numpy(), int(it[0]), int(st[0])


def _handle(csr, b, x0, precond, rtol, maxiter=5000):
    import torch
    from kcfd.solver import Solver
    s = Solver(csr, precond=precond, rtol=rtol, maxiter=maxiter, team=1, lanes=1, block=1024)
    s.setup(csr)
    xd = torch.from_numpy(np.ascontiguousarray(x0)).cuda()
    it, rr, st = s.solve(csr, torch.from_numpy(np.ascontiguousarray(b)).cuda(), xd)
    torch.cuda.synchronize()
    return xd.cpu().numpy(), int(it[0]), int(st[0])


def test_noalloc_matches_handle_two_calls_in_a_row():
    from kcfd.solver import DeviceCSR
    A1, b1 = convdiff_system(channel_mesh(20, 20))
    A2, b2 = _hex_system(12, seed=4)
    cases = [(A1, b1, np.zeros(len(b1)), "jacobi"),
             (A2, b2, np.linspace(-1.0, 1.0, len(b2)), "none")]
    first = None
    for A, b, x0, pc in cases:  # two calls in a row on the shared scratch
        d = DeviceCSR.from_scipy(A)
        xn, itn, stn = _noalloc(d, b, x0, pc, 1e-10)
        xh, ith, sth = _handle(d, b, x0, pc, 1e-10)
        assert stn == 0 and sth == 0
        assert itn == ith
        assert _rel(xn, xh) < 1e-12
        assert np.linalg.norm(b - A @ xn) / np.linalg.norm(b) < 2e-10
        if first is None:
            first = (xn, itn)
    # the smaller system again after the larger one left its data in the shared array
    A, b, x0, pc = cases[0]
    xn, itn, stn = _noalloc(DeviceCSR.from_scipy(A), b, x0, pc, 1e-10)
    assert stn == 0 and itn == first[1]
    np.testing.assert_array_equal(xn, first[0])


def test_noalloc_records_into_a_cuda_graph():
    """After one call on the device, a call records into a torch CUDA graph in global
    capture mode, where a device allocation or a symbol look-up would invalidate the
    capture; each replay gives the eager call's x, iterations and status bit for bit."""
    import torch
    from kcfd import _lib
    from kcfd.solver import DeviceCSR
    A, b = convdiff_system(channel_mesh(20, 20))
    d = DeviceCSR.from_scipy(A)
    x_ref, it_ref, st_ref = _noalloc(d, b, np.zeros(len(b)), "jacobi", 1e-10)   # the first call, before capture
    assert st_ref == 0
    bd = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    xd = torch.zeros_like(bd)
    it = torch.zeros(1, dtype=torch.int32, device="cuda")
    rr = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    desc = d.desc()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    rc = []
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s, capture_error_mode="global"):
            rc.append(_lib.lib().kcfd_bicgstab_noalloc(
                C.byref(desc), _lib.ptr(bd), _lib.ptr(xd), _lib.PREC["jacobi"], _lib.STOP_SCIPY, 1e-10, 0.0,
                5000, _lib.ptr(it), _lib.ptr(rr), _lib.ptr(st), _lib.stream_handle(s)))
    assert rc == [_lib.OK], _lib.last_error()
    for _ in range(2):
        xd.zero_()
        it.zero_()
        st.fill_(-1)
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        assert int(st[0]) == st_ref and int(it[0]) == it_ref
        np.testing.assert_array_equal(xd.cpu().numpy(), x_ref)
    del g


def test_noalloc_rejects_oversized_systems():
    from kcfd import _lib
    from kcfd.solver import DeviceCSR
    limit = _lib.lib().kcfd_noalloc_max_rows()
    assert limit == 32768
    A, b = _hex_system(33, seed=1)   # 35,937 rows > limit
    assert A.shape[0] > limit
    d = DeviceCSR.from_scipy(A)
    with pytest.raises(_lib.KcfdError, match="rows"):
        _noalloc(d, b, np.zeros(len(b)), "jacobi", 1e-8)
