"""The serving scheduler (kcfd.serve.Server.run) on the host, with a stand-in for the
device-resident case: the same admission, slot, budget and polling loop that serves
device cases, with each case's work simulated by a timer.

- every request finishes exactly once, with its own id, size and iteration count;
- the admitted footprint never exceeds the HBM budget, except for a lone case larger
  than the budget (admitted when nothing else is resident), and resident cases never
  exceed `max_active`; serial mode keeps one case resident;
- "sjf" admits the queued request with the least estimated work first, "fifo" in
  arrival order;
- a case stops after the first tick whose continuity is below `cont_tol`, or at
  `max_iters` (then not converged)."""
import math
import threading
import time

import numpy as np
import pytest

from kcfd.serve import Request, Server, footprint_bytes, make_requests, summarize, work_estimate


class FakeCase:
    """Continuity falls by `rate` per outer iteration; an iteration takes `sec_per_iter`."""

    def __init__(self, req, log, lock, rate=0.5, sec_per_iter=2e-5):
        self.req = req
        self.cells = req.N ** req.ndim
        self.done_iters = 0
        self.rate = rate
        self.sec = sec_per_iter
        self.t_ready = 0.0
        with lock:
            log.append(req.rid)

    def launch(self, k):
        self.done_iters += k
        self.t_ready = time.perf_counter() + k * self.sec

    def ready(self):
        return time.perf_counter() >= self.t_ready

    def continuity(self):
        return self.rate ** self.done_iters

    def fields(self):
        return {"rid": self.req.rid}


def _factory(rate=0.5, sec_per_iter=2e-5):
    log, lock = [], threading.Lock()
    return (lambda r: FakeCase(r, log, lock, rate, sec_per_iter)), log


def test_every_request_finishes_within_budget_and_slots():
    reqs = make_requests(40, rate=2000.0, seed=3, n2d=(32, 128), n3d=(16, 40))
    fps = [footprint_bytes(r.ndim, r.N) for r in reqs]
    budget = 3 * max(fps)
    srv = Server(budget_bytes=budget, max_active=5, iters_per_tick=4, cont_tol=1e-6, policy="sjf", keep_fields=True)
    fac, log = _factory()
    res = srv.run(reqs, case_factory=fac)
    assert sorted(r.rid for r in res) == list(range(40))
    assert sorted(log) == list(range(40))
    by = {r.rid: r for r in res}
    for q in reqs:
        out = by[q.rid]
        assert (out.ndim, out.N, out.cells) == (q.ndim, q.N, q.N ** q.ndim)
        assert out.fields == {"rid": q.rid}
        assert out.admitted >= q.arrival - 1e-9 and out.finished >= out.admitted
    assert srv.last_stats["peak_bytes"] <= budget
    assert 1 <= srv.last_stats["peak_resident"] <= 5
    s = summarize(res)
    assert s["cases"] == 40 and s["converged"] == 40 and s["p99_ms"] >= s["p50_ms"]


def test_serial_keeps_one_case_resident():
    reqs = make_requests(12, rate=5000.0, seed=1, n2d=(32, 64), n3d=(16, 24))
    srv = Server(max_active=8, iters_per_tick=5)
    fac, _ = _factory()
    res = srv.run(reqs, serial=True, case_factory=fac)
    assert len(res) == 12 and srv.last_stats["peak_resident"] == 1
    fin = sorted(res, key=lambda r: r.finished)
    for a, b in zip(fin, fin[1:]):
        assert b.admitted >= a.admitted


def test_lone_case_larger_than_budget_is_admitted():
    reqs = [Request(0, 3, 64, 400.0, 0.0), Request(1, 2, 32, 400.0, 0.0)]
    budget = footprint_bytes(2, 32) + 1
    assert footprint_bytes(3, 64) > budget
    srv = Server(budget_bytes=budget, max_active=4, iters_per_tick=5, policy="fifo")
    fac, log = _factory()
    res = srv.run(reqs, case_factory=fac)
    assert sorted(r.rid for r in res) == [0, 1]
    # the big case ran alone: the small one waited for it
    assert log == [0, 1]
    r0, r1 = sorted(res, key=lambda r: r.rid)
    assert r1.admitted >= r0.finished - 1e-6


@pytest.mark.parametrize("policy", ["sjf", "fifo"])
def test_admission_order(policy):
    rng = np.random.default_rng(7)
    reqs = [Request(i, int(rng.integers(2, 4)), int(rng.integers(16, 64)), 300.0, 0.0) for i in range(10)]
    srv = Server(max_active=1, iters_per_tick=5, policy=policy)
    fac, log = _factory()
    srv.run(reqs, case_factory=fac)
    if policy == "fifo":
        assert log == list(range(10))
    else:
        # the first pick happens with every request queued; ties keep arrival order
        want = sorted(range(10), key=lambda i: (work_estimate(reqs[i]), i))
        assert log == want


def test_stop_rule_and_iteration_cap():
    k, tol = 7, 1e-6
    reqs = [Request(0, 2, 32, 100.0, 0.0)]
    srv = Server(iters_per_tick=k, cont_tol=tol, max_iters=1000)
    fac, _ = _factory(rate=0.5)
    (r,) = srv.run(reqs, case_factory=fac)
    need = math.floor(math.log(tol) / math.log(0.5)) + 1  # first n with 0.5**n < tol
    assert r.converged and r.iterations == k * math.ceil(need / k)
    assert r.continuity == 0.5 ** r.iterations
    srv = Server(iters_per_tick=k, cont_tol=tol, max_iters=14)
    fac, _ = _factory(rate=0.99)
    (r,) = srv.run(reqs, case_factory=fac)
    assert not r.converged and r.iterations == 14


def test_requests_and_footprints():
    a = make_requests(200, rate=50.0, seed=0)
    b = make_requests(200, rate=50.0, seed=0)
    assert a == b
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert all(32 <= r.N <= 512 for r in a if r.ndim == 2) and all(16 <= r.N <= 96 for r in a if r.ndim == 3)
    assert 60 <= sum(r.ndim == 2 for r in a) <= 140
    assert all(100.0 <= r.Re <= 1000.0 for r in a)
    for nd, lo, hi in ((2, 32, 512), (3, 16, 96)):
        f = [footprint_bytes(nd, N) for N in range(lo, hi + 1, 8)]
        assert all(x < y for x, y in zip(f, f[1:]))
        assert footprint_bytes(nd, hi, "mixed") != footprint_bytes(nd, hi, "fp64")
    with pytest.raises(ValueError):
        Server(policy="lifo")

