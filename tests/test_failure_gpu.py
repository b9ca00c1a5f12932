"""Failure detection on the device without a fault: a team barrier that cannot
complete (one member short) gives up after its clock budget, records KCFD_TIMEOUT for
the host, and returns; the context stays usable (a solve right after succeeds). The
complete barrier leaves the flag at zero."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from case16 import channel_mesh, convdiff_system

pytestmark = pytest.mark.gpu


def _run(ctas, team, budget):
    import torch
    from kcfd import _lib
    bar = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = _lib.lib().kcfd_selftest_barrier(ctas, team, budget, _lib.ptr(bar), _lib.ptr(err), _lib.stream_handle())
    assert rc == _lib.OK
    torch.cuda.synchronize()
    return int(err.item())


def test_barrier_wait_runs_out_and_reports():
    import torch
    from kcfd import _lib
    from kcfd.solver import DeviceCSR, Solver
    assert _run(4, 4, 2_000_000) == 0
    assert _run(4, 5, 2_000_000) == _lib.TIMEOUT
    assert _run(1, 2, 2_000_000) == _lib.TIMEOUT
    # the context is intact: an ordinary solve works afterwards
    A, b = convdiff_system(channel_mesh(24, 16))
    d = DeviceCSR.from_scipy(A)
    s = Solver(d, precond="jacobi", rtol=1e-10, maxiter=3000, team=2)
    s.setup(d)
    x = torch.zeros(len(b), dtype=torch.float64, device="cuda")
    it, rr, st = s.solve(d, torch.from_numpy(b).cuda(), x)
    assert int(st[0]) == 0 and s.barrier_error() == 0
    xd = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x.cpu().numpy() - xd) / np.linalg.norm(xd) < 1e-8


def test_selftest_rejects_bad_arguments():
    from kcfd import _lib
    L = _lib.lib()
    assert L.kcfd_selftest_barrier(4, 3, 1000, None, None, None) == _lib.BAD_INPUT
