"""Host logic of the continuous-batching server (serving.SolveServer) on stand-in 3D
models: first-come-first-served admission under the memory budget and the cap on
requests in flight, the statuses a request can end in (converged, stalled, at the
iteration limit, diverged), iteration accounting per check round, the over-budget
refusal and the summary.  No GPU: each stand-in's residual falls by a fixed factor
per check round."""
import math

import numpy as np
import pytest

from helpers import load_fastice

fi = load_fastice()
from fastice_b200 import serving  # noqa: E402


class FakeModel:
    """Residual norms shrink by `rate` per ncheck iterations; `nan_after` makes
    them non-finite after that many iterations."""

    live = 0

    def __init__(self, r0, rate, ncheck, nan_after=None):
        self.r0, self.rate, self.ncheck, self.nan_after = r0, rate, ncheck, nan_after
        self.iterations = 0
        self.closed = False
        FakeModel.live += 1

    def advance(self, k):
        self.iterations += k

    def residual_norms(self):
        out = np.zeros(12)
        r = self.r0 * self.rate ** (self.iterations / self.ncheck)
        if self.nan_after is not None and self.iterations > self.nan_after:
            r = math.nan
        out[1:4] = r          # r_V (relative to ||ρg|| = 1)
        out[0] = 0.0          # r_P
        out[8:11] = 1.0       # max|V|
        return out

    def get_field(self, name):
        return np.full(3, float(self.iterations))

    def close(self):
        assert not self.closed
        self.closed = True
        FakeModel.live -= 1


def req(rid, arrival, nbytes, rate=0.1, r0=1.0, tol=1e-6, max_iter=100000, nan_after=None, ncheck=10):
    return serving.SolveRequest(rid=rid, arrival=arrival, kind="3d", bytes=nbytes, tol=tol, max_iter=max_iter,
                                build=lambda: FakeModel(r0, rate, ncheck, nan_after))


def serve(reqs, **kw):
    srv = serving.SolveServer(ncheck=10, realtime=False, **kw)
    done = srv.run(reqs)
    return {r.rid: r for r in done}, srv


def test_statuses_and_iterations():
    FakeModel.live = 0
    reqs = [req(0, 0.0, 10, rate=0.1),                      # 1e-6 after 6 rounds of 10
            req(1, 0.0, 10, rate=1.0),                       # never improves: stalls a window after its first check
            req(2, 0.0, 10, rate=0.6, max_iter=50),          # halves every two rounds, runs out of iterations
            req(3, 0.0, 10, rate=0.5, nan_after=25)]         # non-finite on the round after 25 iterations
    done, srv = serve(reqs, budget_bytes=100, window=40)
    assert done[0].status == "converged" and done[0].iterations == 70   # measure < tol first at 7 rounds (1e-7)
    assert done[1].status == "stalled" and done[1].iterations == 50
    assert done[2].status == "max_iter" and done[2].iterations == 50
    assert done[3].status == "diverged" and done[3].iterations == 30
    assert all(r.meta["result"]["Vx"][0] == r.iterations for r in done.values())
    assert FakeModel.live == 0 and srv.peak_bytes == 40


def test_admission_first_come_first_served_under_the_budget():
    FakeModel.live = 0
    reqs = [req(0, 0.0, 60, rate=0.1), req(1, 0.0, 50, rate=0.1), req(2, 0.0, 30, rate=0.1)]
    done, srv = serve(reqs, budget_bytes=100, window=0)
    # request 1 does not fit beside request 0, and request 2 waits behind it (no overtaking)
    assert srv.peak_bytes == 80
    assert done[1].admitted >= done[0].finished and done[2].admitted >= done[0].finished
    assert all(r.status == "converged" for r in done.values())


def test_max_active_one_serves_one_at_a_time():
    FakeModel.live = 0
    reqs = [req(q, 0.0, 10, rate=0.1) for q in range(3)]
    done, srv = serve(reqs, budget_bytes=1000, window=0, max_active=1)
    order = sorted(done.values(), key=lambda r: r.admitted)
    for a, b in zip(order, order[1:]):
        assert b.admitted >= a.finished
    assert srv.peak_bytes == 10


def test_request_over_the_budget_is_refused():
    with pytest.raises(RuntimeError):
        serve([req(0, 0.0, 200)], budget_bytes=100)


def test_summary_counts_and_latencies():
    FakeModel.live = 0
    reqs = [req(0, 0.0, 10, rate=0.1), req(1, 0.0, 10, rate=1.0)]
    done, _ = serve(reqs, budget_bytes=100, window=20)
    s = serving.summarize(list(done.values()), makespan=2.0)
    assert s["requests"] == 2 and s["status"] == {"converged": 1, "stalled": 1}
    assert s["solves_per_s"] == pytest.approx(1.0)
    assert s["p50_latency_s"] >= 0.0 and s["p99_latency_s"] >= s["p50_latency_s"]
