"""Host logic of the serving loop on CPU, with stand-in contexts and executors: requests are
admitted in arrival order when a slot and device memory are free, the committed memory never
exceeds the budget, oversized requests are rejected, and latency statistics are reported."""

import threading
import time

import numpy as np

from inq_b200 import serving, synthetic


class FakeSystem:
    def __init__(self, n, nst, natoms=2):
        self.npoints = n ** 3
        self.nst = nst
        self.natoms = natoms


def _req(rid, n, nst, arrival, kind="apply"):
    p = serving.Payload(FakeSystem(n, nst), np.zeros(1), np.zeros((1, 1), np.complex64))
    return serving.Request(rid, kind, p, arrival=arrival)


def test_admission_respects_budget_and_slots():
    active = []
    peak = {"slots": 0}
    lock = threading.Lock()

    def execute(req, ctx):
        with lock:
            active.append(req.rid)
            peak["slots"] = max(peak["slots"], len(active))
        time.sleep(0.02)
        with lock:
            active.remove(req.rid)
        req.result = {"happs": req.payload.system.nst}

    reqs = [_req(i, 32, 16, 0.001 * i) for i in range(12)]
    fp = reqs[0].footprint(serving.F32)
    srv = serving.Server(slots=4, budget_bytes=2 * fp + 1, contexts=[object()] * 4, execute=execute)
    stats = srv.run(reqs)
    assert stats["completed"] == 12 and stats["rejected"] == 0
    assert peak["slots"] <= 2                     # memory, not slots, limited concurrency
    assert stats["peak_committed_bytes"] <= stats["budget_bytes"]
    # arrival order is admission order
    adm = [r.admitted for r in sorted(reqs, key=lambda r: r.arrival)]
    assert adm == sorted(adm)
    assert stats["p99_ms"] >= stats["p50_ms"] > 0


def test_oversized_request_rejected():
    def execute(req, ctx):
        req.result = {"happs": 1}

    small = _req(0, 16, 8, 0.0)
    big = _req(1, 96, 256, 0.0)
    srv = serving.Server(slots=2, budget_bytes=small.footprint(serving.F32) * 2, contexts=[object()] * 2,
                         execute=execute)
    stats = srv.run([small, big])
    assert stats["completed"] == 1 and stats["rejected"] == 1
    assert big.error.startswith("rejected")


def test_failing_request_is_reported():
    def execute(req, ctx):
        if req.rid == 1:
            raise RuntimeError("boom")
        req.result = {"happs": 1}

    srv = serving.Server(slots=2, budget_bytes=1 << 40, contexts=[object()] * 2, execute=execute)
    reqs = [_req(i, 16, 8, 0.0) for i in range(3)]
    stats = srv.run(reqs)
    assert stats["completed"] == 2 and "boom" in reqs[1].error


def test_poisson_stream():
    ps = [serving.Payload(FakeSystem(24, 8), None, None)]
    large = serving.Payload(FakeSystem(96, 256), None, None)
    reqs = serving.poisson_requests(ps, 400, rate=100.0, large=large)
    gaps = np.diff([r.arrival for r in reqs])
    assert abs(np.mean(gaps) - 0.01) < 0.003
    frac = np.mean([r.payload is large for r in reqs])
    assert 0.05 < frac < 0.15
    assert any(r.kind == "etrs" for r in reqs) and any(r.kind == "apply" for r in reqs)


def test_size_classes_do_not_block_each_other():
    """With a bulk slot, large requests run only there and a large request waiting for it does not
    hold up the small ones behind it in arrival order."""
    started = {}
    lock = threading.Lock()

    def execute(req, ctx):
        with lock:
            started[req.rid] = ctx
        time.sleep(0.3 if req.payload.system.npoints > 40 ** 3 else 0.01)
        req.result = {"happs": 1}

    ctxs = [object() for _ in range(3)]
    big = [_req(i, 96, 256, 0.0) for i in range(2)]
    small = [_req(10 + i, 16, 8, 0.01 * (i + 1)) for i in range(6)]
    srv = serving.Server(slots=3, budget_bytes=1 << 40, contexts=ctxs, execute=execute, bulk_slots=1,
                         bulk_min_bytes=big[0].footprint(serving.F32))
    stats = srv.run(big + small)
    assert stats["completed"] == 8
    assert all(started[r.rid] is ctxs[0] for r in big)
    assert all(started[r.rid] is not ctxs[0] for r in small)
    assert max(r.finished for r in small) < big[1].admitted


def test_bulk_slots_leave_an_interactive_slot():
    import pytest
    with pytest.raises(ValueError):
        serving.Server(slots=2, budget_bytes=1 << 30, contexts=[object()] * 2, bulk_slots=2)
