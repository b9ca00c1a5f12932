"""CUDA-graph capture of kcfd calls through the C ABI (kcfd_graph_*, kcfd.solver.DeviceGraph):
a captured pair of SpMVs and a captured solver set-up + solve (persistent grid kernel),
replayed, give bitwise the results of the same calls issued directly."""
import pytest

from case16 import channel_mesh, convdiff_system

pytestmark = pytest.mark.gpu


def test_captured_spmv_and_solve_replay_bitwise():
    import torch
    from kcfd.solver import DeviceCSR, DeviceGraph, Solver
    A, b = convdiff_system(channel_mesh(40, 30))
    d = DeviceCSR.from_scipy(A)
    n = d.n
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y_ref = d.spmv(d.spmv(x))
    sv = Solver(d, precond="jacobi", rtol=1e-10, maxiter=3000, team=2)
    bd = torch.from_numpy(b).cuda()
    sv.setup(d)
    x_ref = torch.zeros_like(bd)
    sv.solve(d, bd, x_ref)
    it_ref = int(sv.iters[0])
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    y1, y2, xs = torch.empty_like(x), torch.empty_like(x), torch.zeros_like(bd)
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with DeviceGraph(s) as g:
            d.spmv(x, y1, stream=s)
            d.spmv(y1, y2, stream=s)
            sv.setup(d, stream=s)
            sv.solve(d, bd, xs, stream=s)
    for _ in range(2):
        y1.zero_()
        y2.zero_()
        xs.zero_()
        sv.iters.zero_()
        torch.cuda.synchronize()
        g.launch(s)
        s.synchronize()
        assert torch.equal(y2, y_ref)
        assert torch.equal(xs, x_ref) and int(sv.iters[0]) == it_ref


def test_handle_dropped_inside_a_capture_is_released_after_it():
    """A solver handle destroyed while a CUDA graph is being captured on this thread
    (e.g. by the garbage collector) would free device memory inside the capture and
    invalidate it; its release is deferred to the next one outside the capture."""
    import torch
    from kcfd import _lib
    from kcfd.solver import DeviceCSR, Solver
    A, b = convdiff_system(channel_mesh(20, 10))
    d = DeviceCSR.from_scipy(A)
    doomed = Solver(d, precond="jacobi", rtol=1e-8, maxiter=100, team=1)
    x = torch.randn(d.n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    d.spmv(x, y)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            d.spmv(x, y, stream=s)
            del doomed                  # destroyed inside the capture
            assert len(_lib._deferred) == 1
    y.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(y, d.spmv(x))
    Solver(d, precond="jacobi", rtol=1e-8, maxiter=100, team=1)   # created and dropped outside: flushes
    assert len(_lib._deferred) == 0
