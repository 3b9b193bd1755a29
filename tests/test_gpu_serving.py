"""Continuous-batching solve server: every request's result is the same served
alone (one at a time) and in the mix, admission respects the device-memory
budget, and 2D and 3D requests overlap."""
import numpy as np
import pytest

from conftest import load_fastice

pytestmark = pytest.mark.gpu


def _requests(fi, arrivals, library="fast"):
    from fastice_b200 import scenarios, serving
    reqs = []
    for rid, (t, kind, seed, n) in enumerate(arrivals):
        if kind == "2d":
            build = (lambda seed=seed, n=n: scenarios.inclusion_model(seed, n=n, dtype="f64", max_contrast=100.0)[0])
            reqs.append(serving.SolveRequest(rid=rid, arrival=t, kind="2d", build=build,
                                             bytes=serving.footprint_2d(n, 8), tol=1e-6, max_iter=40000))
        else:
            build = (lambda seed=seed, n=n: scenarios.bed_model(seed, n, library=library)[0])
            reqs.append(serving.SolveRequest(rid=rid, arrival=t, kind="3d", build=build,
                                             bytes=serving.footprint_3d_ib((n, n, n), 8), tol=1e-4, max_iter=3000,
                                             meta={"length_z": 0.6}))
    return reqs


STREAM = [(0.00, "2d", 1, (48, 40)), (0.01, "3d", 2, 16), (0.02, "2d", 3, (64, 56)), (0.05, "2d", 4, (40, 72)),
          (0.08, "3d", 5, 20), (0.10, "2d", 6, (56, 56)), (0.12, "2d", 7, (72, 48))]


def _serve(fi, library="fast", **kw):
    from fastice_b200 import serving
    srv = serving.SolveServer(ncheck=200, window=20000, **kw)
    done = srv.run(_requests(fi, STREAM, library))
    return {r.rid: r for r in done}, srv


# 3D requests sharing launches run the batched kernels, whose products the production
# build may contract into fused multiply-adds where the single-model kernels do not:
# that mode is compared bit for bit in the no-FMA build
@pytest.mark.parametrize("share3d", [False, True], ids=["3d-streams", "3d-shared"])
def test_results_alone_and_in_the_mix_agree(share3d):
    fi = load_fastice()
    lib = "strict" if share3d else "fast"
    mix, srv = _serve(fi, lib, budget_bytes=8 << 30, realtime=True, share3d=share3d)
    alone, _ = _serve(fi, lib, budget_bytes=8 << 30, realtime=False, max_active=1)
    assert set(mix) == set(alone) == set(range(len(STREAM)))
    for rid in mix:
        a, b = mix[rid], alone[rid]
        assert a.status == b.status and a.iterations == b.iterations, (rid, a.status, b.status)
        assert a.status in ("converged", "max_iter", "stalled"), (rid, a.status)
        for f in ("Vx", "P"):
            assert np.array_equal(a.meta["result"][f], b.meta["result"][f]), (rid, f)
    assert all(mix[r].status == "converged" for r in mix if mix[r].kind == "2d")
    assert srv.peak_bytes <= 8 << 30


def test_admission_respects_the_budget():
    fi = load_fastice()
    from fastice_b200 import serving
    reqs = _requests(fi, STREAM)
    budget = max(r.bytes for r in reqs) + min(r.bytes for r in reqs)
    done, srv = _serve(fi, budget_bytes=budget, realtime=False)
    assert len(done) == len(STREAM) and srv.peak_bytes <= budget
    summary = serving.summarize(list(done.values()))
    assert summary["requests"] == len(STREAM) and summary["p99_latency_s"] >= summary["p50_latency_s"] > 0


def test_request_over_budget_is_refused():
    fi = load_fastice()
    with pytest.raises(RuntimeError):
        _serve(fi, budget_bytes=1 << 20, realtime=False)
