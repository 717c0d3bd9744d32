"""Packed serving on the host (no GPU): host stand-ins for the planner and
the packed solve exercise pack formation while the device is busy, the HBM
budget across packs, the step-limit key, per-request failures and the
resident field charge."""
import threading
import time

import pytest

from uniphot_b200.serve import PackedServer, latency_summary


class FakePacker:
    """Records every pack the stand-in device solves."""

    def __init__(self, t_pack=0.05):
        self.lock = threading.Lock()
        self.t_pack = t_pack
        self.packs = []
        self.running = 0
        self.peak_running = 0
        self.bytes = 0
        self.peak_bytes = 0

    def plan(self, kw):
        if kw.get("plan_fail"):
            raise ValueError("stand-in planning failure")
        return kw["rid"], kw.get("bytes", 1), kw.get("islands", 1), kw.get("field", 0)

    def pack(self, state, reqs):
        nbytes = sum(kw.get("bytes", 1) for kw, _ in reqs)
        with self.lock:
            self.packs.append([p for _, p in reqs])
            self.running += 1
            self.peak_running = max(self.peak_running, self.running)
            self.bytes += nbytes
            self.peak_bytes = max(self.peak_bytes, self.bytes)
        time.sleep(self.t_pack)
        with self.lock:
            self.running -= 1
            self.bytes -= nbytes
        return [RuntimeError("stand-in solve failure") if kw.get("fail") else p * 10
                for kw, p in reqs]


def _server(dev, engines=1, budget=1e9, **kw):
    return PackedServer(planners=2, engines=engines, hbm_budget_bytes=budget,
                        plan_fn=dev.plan, pack_fn=dev.pack,
                        engine_init=lambda i: {}, **kw)


def test_requests_arriving_during_a_solve_form_the_next_pack():
    dev = FakePacker(t_pack=0.1)
    with _server(dev) as srv:
        futs = [srv.submit({"rid": i}) for i in range(24)]
        res = [f.result(timeout=30) for f in futs]
    assert res == [10 * i for i in range(24)]
    assert sum(srv.packs) == 24 and len(srv.packs) == len(dev.packs)
    assert max(srv.packs) > 1                       # requests were packed
    assert len(srv.packs) < 24
    solved = sorted(r for p in dev.packs for r in p)
    assert solved == list(range(24))                # each request once
    for st in srv.stats:
        assert st.pack >= 0 and st.pack_size == srv.packs[st.pack]


def test_pack_size_is_capped():
    dev = FakePacker(t_pack=0.1)
    with _server(dev, max_pack=3) as srv:
        futs = [srv.submit({"rid": i}) for i in range(12)]
        [f.result(timeout=30) for f in futs]
    assert max(srv.packs) <= 3 and sum(srv.packs) == 12


def test_budget_bounds_what_is_packed_and_in_flight():
    dev = FakePacker(t_pack=0.05)
    with _server(dev, engines=2, budget=100) as srv:
        futs = [srv.submit({"rid": i, "bytes": 40}) for i in range(10)]
        [f.result(timeout=30) for f in futs]
    assert dev.peak_bytes <= 100 and srv.peak_in_use <= 100
    assert max(srv.packs) <= 2
    assert srv.in_use == 0


def test_step_limit_key_keeps_packs_homogeneous():
    dev = FakePacker(t_pack=0.1)
    with _server(dev) as srv:
        futs = [srv.submit({"rid": i, "max_steps": 20 if i % 2 else 30})
                for i in range(16)]
        [f.result(timeout=30) for f in futs]
    for p in dev.packs:
        assert len({r % 2 for r in p}) == 1


def test_a_failing_request_fails_alone():
    dev = FakePacker(t_pack=0.05)
    with _server(dev) as srv:
        futs = [srv.submit({"rid": i, "fail": i == 3, "plan_fail": i == 5})
                for i in range(8)]
        for i, f in enumerate(futs):
            if i == 3:
                with pytest.raises(RuntimeError, match="stand-in solve"):
                    f.result(timeout=30)
            elif i == 5:
                with pytest.raises(ValueError, match="stand-in planning"):
                    f.result(timeout=30)
            else:
                assert f.result(timeout=30) == 10 * i
    assert srv.in_use == 0
    assert len(srv.stats) == 8


def test_a_failing_pack_fails_its_requests_and_frees_the_budget():
    def bad_pack(state, reqs):
        raise RuntimeError("RESOURCE_EXHAUSTED: stand-in")
    srv = PackedServer(planners=1, engines=1, hbm_budget_bytes=100,
                       plan_fn=lambda kw: (kw["rid"], 60, 1), pack_fn=bad_pack,
                       engine_init=lambda i: {})
    with srv:
        futs = [srv.submit({"rid": i}) for i in range(3)]
        for f in futs:
            with pytest.raises(RuntimeError, match="RESOURCE_EXHAUSTED"):
                f.result(timeout=30)
    assert srv.in_use == 0


def test_resident_field_bytes_stay_charged_per_engine():
    """The engine's context keeps the last field it uploaded between packs:
    the largest field bytes seen stay charged after the pack."""
    dev = FakePacker(t_pack=0.01)
    with _server(dev, budget=1000) as srv:
        srv.submit({"rid": 0, "bytes": 100, "field": 30}).result(timeout=30)
        srv.submit({"rid": 1, "bytes": 100, "field": 50}).result(timeout=30)
        srv.submit({"rid": 2, "bytes": 100, "field": 20}).result(timeout=30)
    assert srv.resident == [50]
    assert srv.in_use == 50


def test_latency_summary_of_a_packed_stream():
    dev = FakePacker(t_pack=0.02)
    with _server(dev) as srv:
        futs = [srv.submit({"rid": i, "islands": 2}) for i in range(10)]
        [f.result(timeout=30) for f in futs]
    s = latency_summary(srv.stats)
    assert s["requests"] == 10 and s["islands_per_s"] > 0
    assert s["p50_ms"] <= s["p99_ms"]


def test_closed_packed_server_rejects_requests():
    srv = _server(FakePacker())
    srv.close()
    with pytest.raises(RuntimeError):
        srv.submit({"rid": 0})


def test_a_failing_engine_start_fails_its_requests():
    """An engine whose set-up raises (no device, say) answers every request
    it takes with that error instead of leaving it unanswered."""
    def bad_init(i):
        raise RuntimeError("stand-in: no device")
    dev = FakePacker()
    srv = PackedServer(planners=1, engines=1, hbm_budget_bytes=100, plan_fn=dev.plan,
                       pack_fn=dev.pack, engine_init=bad_init)
    with srv:
        futs = [srv.submit({"rid": i}) for i in range(3)]
        for f in futs:
            with pytest.raises(RuntimeError, match="no device"):
                f.result(timeout=30)
    assert srv.in_use == 0
