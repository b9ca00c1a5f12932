"""Served requests: continuous batching admits overlapping cases, each converges, and
each case's result is the same alone and in the mix (bitwise: a case's solves reduce
in a fixed order on its own buffers whatever runs beside it).

The continuity residual of the reference's SIMPLE discretisation decays roughly like
1/k (about 1.4e-3 after 600 outer iterations on a 16^2 cavity), so these tests serve
to 5e-2, which small cavities reach within tens of iterations."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reqs():
    from kcfd.serve import Request
    # staggered arrivals so later requests join while earlier ones are running
    return [Request(0, 2, 16, 150.0, 0.00), Request(1, 3, 8, 400.0, 0.01), Request(2, 2, 24, 900.0, 0.02),
            Request(3, 3, 10, 250.0, 0.03), Request(4, 2, 20, 600.0, 0.04)]


def test_served_results_same_alone_and_in_the_mix():
    from kcfd.serve import Server, summarize
    srv = Server(max_active=8, iters_per_tick=5, max_iters=400, cont_tol=5e-2, keep_fields=True)
    mixed = {r.rid: r for r in srv.run(_reqs())}
    assert len(mixed) == 5
    s = summarize(list(mixed.values()))
    assert s["converged"] == 5, s
    for r in _reqs():
        r.arrival = 0.0
        alone = srv.run([r])[0]
        m = mixed[r.rid]
        assert alone.iterations == m.iterations
        np.testing.assert_array_equal(alone.fields["U"], m.fields["U"])
        np.testing.assert_array_equal(alone.fields["p"], m.fields["p"])


def test_admission_respects_budget():
    from kcfd.serve import Server, footprint_bytes
    reqs = _reqs()
    one = max(footprint_bytes(r.ndim, r.N) for r in reqs)
    srv = Server(budget_bytes=1.5 * one, max_active=8, iters_per_tick=5, max_iters=400, cont_tol=5e-2)
    res = srv.run(reqs)
    assert len(res) == 5 and all(r.converged for r in res)
    # with room for one resident case at a time, cases finish in admission order
    fin = sorted(res, key=lambda r: r.finished)
    assert [r.rid for r in fin] == [r.rid for r in sorted(res, key=lambda r: r.admitted)]
