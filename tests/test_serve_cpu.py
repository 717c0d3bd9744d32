"""Serving admission logic on the host (no GPU): host stand-ins for the
planner and the solve exercise the HBM budget, the worker slots, arrival
order, error propagation and the latency summary."""
import threading
import time

import numpy as np
import pytest

from uniphot_b200.serve import Server, latency_summary, poisson_stream


class FakeDevice:
    """Records concurrent 'device' occupancy of the stand-in solves."""

    def __init__(self):
        self.lock = threading.Lock()
        self.bytes = 0
        self.peak_bytes = 0
        self.running = 0
        self.peak_running = 0
        self.order = []

    def plan(self, kw):
        return kw["rid"], kw["bytes"], kw.get("islands", 1)

    def solve(self, state, kw, plan):
        if kw.get("fail"):
            raise RuntimeError("RESOURCE_EXHAUSTED: stand-in failure")
        with self.lock:
            self.bytes += kw["bytes"]
            self.running += 1
            self.peak_bytes = max(self.peak_bytes, self.bytes)
            self.peak_running = max(self.peak_running, self.running)
            self.order.append(plan)
        time.sleep(kw.get("t", 0.02))
        with self.lock:
            self.bytes -= kw["bytes"]
            self.running -= 1
        return plan * 10


def _server(dev, workers, budget):
    return Server(workers=workers, hbm_budget_bytes=budget, plan_fn=dev.plan,
                  solve_fn=dev.solve, worker_init=lambda i: {})


def test_budget_and_slots_are_respected():
    dev = FakeDevice()
    with _server(dev, workers=4, budget=100) as srv:
        futs = [srv.submit({"rid": i, "bytes": 40, "t": 0.03}) for i in range(12)]
        res = [f.result(timeout=30) for f in futs]
    assert res == [10 * i for i in range(12)]
    assert dev.peak_bytes <= 100          # never more than two 40-byte requests
    assert dev.peak_running == 2
    assert srv.in_use == 0 and srv.peak_in_use <= 100


def test_small_requests_fill_the_worker_slots():
    dev = FakeDevice()
    with _server(dev, workers=3, budget=1e9) as srv:
        futs = [srv.submit({"rid": i, "bytes": 1, "t": 0.05}) for i in range(9)]
        [f.result(timeout=30) for f in futs]
    assert dev.peak_running == 3


def test_request_larger_than_budget_runs_alone():
    dev = FakeDevice()
    with _server(dev, workers=2, budget=50) as srv:
        f_big = srv.submit({"rid": 0, "bytes": 500, "t": 0.05})
        f_small = srv.submit({"rid": 1, "bytes": 10, "t": 0.01})
        assert f_big.result(timeout=30) == 0 and f_small.result(timeout=30) == 10
    assert dev.peak_running == 1


def test_single_worker_keeps_arrival_order():
    dev = FakeDevice()
    with _server(dev, workers=1, budget=1e9) as srv:
        futs = [srv.submit({"rid": i, "bytes": 1, "t": 0.0}) for i in range(20)]
        [f.result(timeout=30) for f in futs]
    assert dev.order == list(range(20))


def test_errors_reach_the_caller_and_free_the_budget():
    dev = FakeDevice()
    with _server(dev, workers=2, budget=100) as srv:
        bad = srv.submit({"rid": 0, "bytes": 90, "fail": True})
        good = srv.submit({"rid": 1, "bytes": 90, "t": 0.01})
        with pytest.raises(RuntimeError, match="RESOURCE_EXHAUSTED"):
            bad.result(timeout=30)
        assert good.result(timeout=30) == 10
    assert srv.in_use == 0


def test_poisson_stream_and_latency_summary():
    dev = FakeDevice()
    reqs = [{"rid": i, "bytes": 1, "islands": 3, "t": 0.005,
             "data_minus_bg": np.zeros((2, 8, 8), np.float32)} for i in range(30)]
    with _server(dev, workers=2, budget=1e9) as srv:
        futs = poisson_stream(srv, reqs, rate_hz=500.0, seed=1)
        [f.result(timeout=30) for f in futs]
    s = latency_summary(srv.stats)
    assert s["requests"] == 30
    assert 0 < s["p50_ms"] <= s["p95_ms"] <= s["p99_ms"]
    assert s["islands_per_s"] > 0 and s["pixels_per_s"] > 0
    assert all(st.latency >= 0.005 for st in srv.stats)


def test_closed_server_rejects_requests():
    dev = FakeDevice()
    srv = _server(dev, workers=1, budget=10)
    srv.close()
    with pytest.raises(RuntimeError):
        srv.submit({"rid": 0, "bytes": 1})


def test_all_giant_request_returns_seed_rows():
    """A cutout whose only island exceeds the joint size cap has nothing to
    fit: the server answers with the giant rows (seeds kept, flagged)."""
    from uniphot_b200.serve import default_plan, default_solve
    from uniphot_b200.synth import make_serving_request
    f = make_serving_request(17)          # one 48-member island
    kw = f.fit_kwargs("analytic")
    plan, nbytes, n_isl = default_plan(kw)
    assert plan is None and nbytes == 0 and n_isl == 0
    res = default_solve({}, kw, plan)
    assert sorted(res.source_idx.tolist()) == list(range(f.pos_x.size))
    assert res.island_giant.all()
    order = np.argsort(res.source_idx)
    np.testing.assert_array_equal(res.pos_x[order], f.pos_x)


def test_resident_field_bytes_stay_charged_between_requests():
    """A worker keeps its field stacks after a request (they are reused and
    regrown), so those bytes stay charged: with one worker, a 60-byte
    request of which 30 are field leaves 30 in use; a second request with a
    smaller field is charged only its transient bytes; a larger field is
    charged its growth.  Two workers each holding a resident field cannot
    then admit a request that would exceed the budget beside them."""
    def plan(kw):
        return kw["rid"], kw["bytes"], 1, kw["field"]

    def solve(state, kw, p):
        return p

    def run(srv, kw):
        # the future resolves before the worker releases the request's
        # bytes; its stats entry is appended after the release
        n = len(srv.stats)
        srv.submit(kw).result(timeout=10)
        t0 = time.perf_counter()
        while len(srv.stats) <= n and time.perf_counter() - t0 < 10:
            time.sleep(0.001)

    srv = Server(workers=1, hbm_budget_bytes=100, plan_fn=plan, solve_fn=solve,
                 worker_init=lambda i: {})
    with srv:
        run(srv, {"rid": 0, "bytes": 60, "field": 30})
        assert srv.in_use == 30 and srv.resident == [30]
        run(srv, {"rid": 1, "bytes": 50, "field": 20})
        assert srv.in_use == 30 and srv.peak_in_use == 60
        run(srv, {"rid": 2, "bytes": 70, "field": 45})
        assert srv.in_use == 45 and srv.resident == [45]
        assert srv.peak_in_use == 30 + 15 + 25     # resident + growth + transient

    dev = FakeDevice()
    srv = Server(workers=2, hbm_budget_bytes=100, plan_fn=lambda kw: (*dev.plan(kw), kw["field"]),
                 solve_fn=dev.solve, worker_init=lambda i: {})
    with srv:
        futs = [srv.submit({"rid": i, "bytes": 40, "field": 20, "t": 0.05}) for i in range(6)]
        [f.result(timeout=30) for f in futs]
    assert srv.peak_in_use <= 100
    assert srv.in_use == sum(srv.resident) <= 40


def test_a_failing_worker_start_fails_its_requests():
    def bad_init(i):
        raise RuntimeError("stand-in: no device")
    dev = FakeDevice()
    srv = Server(workers=1, hbm_budget_bytes=100, plan_fn=dev.plan, solve_fn=dev.solve,
                 worker_init=bad_init)
    with srv:
        futs = [srv.submit({"rid": i, "bytes": 1}) for i in range(3)]
        for f in futs:
            with pytest.raises(RuntimeError, match="no device"):
                f.result(timeout=30)
