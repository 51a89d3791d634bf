"""The /v1/solve front door on the CPU, with a stand-in for the batched engine.

The HTTP layer (python/niryukti/service.py:40-71 in the reference) validates a
request, turns the native JSON model into a Model, submits it and answers with
the reference's result keys.  Here the engine is replaced by a fake service
whose solves finish only when the test releases them, so saturation (429),
validation errors (400, 404) and the JSON round trip are exercised without a
GPU: failures are injected on the host.  The scheduler of SolveService is run
the same way, on a stand-in engine."""
import json
import threading
import time
import urllib.error
import urllib.request
from concurrent.futures import Future

import numpy as np

from niryukti_b200 import serve
from tests.test_oracle import sparse_qp_model


class FakeService:
    """submit() returns a future that completes when `release` is set."""

    tol = 1e-6

    def __init__(self):
        self.release = threading.Event()
        self.submitted = 0

    def submit(self, model, iteration_limit=None, time_limit=None):
        self.submitted += 1
        fut = Future()

        def finish():
            self.release.wait(60)
            fut.set_result({
                "status": "OPTIMAL", "kkt": 0.0, "objective": -7.0, "primal": 0.0, "dual": 0.0,
                "gap": 0.0, "lower_bound": -7.0, "seconds": 0.1, "preprocess_seconds": 0.0,
                "transfer_seconds": 0.0, "iteration_seconds": 0.1, "verification_seconds": 0.0,
                "iterations": 10, "restarts": 0, "weight_updates": 0, "rejected_steps": 0,
                "matrix_precision": "mixed", "removed_rows": 0, "removed_columns": 0,
                "x": np.array([1.0, 2.0]), "y": np.zeros(model.m), "latency_s": 0.1,
                "queue_s": 0.0})

        threading.Thread(target=finish, daemon=True).start()
        return fut


def _post(port, path, payload, raw=None):
    data = raw if raw is not None else json.dumps(payload).encode()
    req = urllib.request.Request(f"http://127.0.0.1:{port}{path}", data=data,
                                 headers={"Content-Type": "application/json"})
    try:
        with urllib.request.urlopen(req, timeout=30) as r:
            return r.status, json.loads(r.read())
    except urllib.error.HTTPError as e:
        return e.code, json.loads(e.read())


def _serve(service, **kw):
    server = serve.make_server(service, port=0, **kw)
    threading.Thread(target=server.serve_forever, daemon=True).start()
    return server, server.server_address[1]


def test_saturated_service_answers_429():
    svc = FakeService()
    server, port = _serve(svc, max_pending=2)
    body = {"model": serve.model_to_json(sparse_qp_model())}
    try:
        held = []
        for _ in range(2):  # two requests occupy both slots
            t = threading.Thread(target=lambda: held.append(_post(port, "/v1/solve", body)))
            t.start()
        for _ in range(100):
            if svc.submitted == 2:
                break
            time.sleep(0.02)
        assert svc.submitted == 2
        code, out = _post(port, "/v1/solve", body)
        assert code == 429 and "occupied" in out["error"]
        svc.release.set()
        for _ in range(200):
            if len(held) == 2:
                break
            time.sleep(0.02)
        assert [c for c, _ in held] == [200, 200]
        code, out = _post(port, "/v1/solve", body)  # a slot is free again
        assert code == 200 and out["status"] == "OPTIMAL"
        assert out["primal"] == [1.0, 2.0] and out["problem_type"] == "QP"
    finally:
        svc.release.set()
        server.shutdown()


def test_request_validation():
    svc = FakeService()
    svc.release.set()
    server, port = _serve(svc)
    model = serve.model_to_json(sparse_qp_model())
    try:
        assert _post(port, "/v1/other", {"model": model})[0] == 404
        assert _post(port, "/v1/solve", {"model": model, "options": {"bogus": 1}})[0] == 400
        assert _post(port, "/v1/solve", {"model": model, "options": {"tol": 1e-3}})[0] == 400
        assert _post(port, "/v1/solve", {"model": model,
                                         "options": {"method": "simplex"}})[0] == 400
        assert _post(port, "/v1/solve", {"model": model,
                                         "options": {"time_limit": 1e9}})[0] == 400
        assert _post(port, "/v1/solve", {"model": model, "extra": 1})[0] == 400
        assert _post(port, "/v1/solve", None, raw=b"[1, 2]")[0] == 400
        integer = json.loads(json.dumps(model))
        integer["variables"][0]["type"] = "integer"
        assert _post(port, "/v1/solve", {"model": integer})[0] == 400
        assert svc.submitted == 0  # nothing invalid reached the engine
    finally:
        server.shutdown()


def test_native_json_round_trip():
    """model_to_json / model_from_json keep the model (the reference's native
    JSON format, src/io.cpp:84-142), including a maximisation sense."""
    m = sparse_qp_model()
    back = serve.model_from_json(serve.model_to_json(m))
    assert back.m == m.m and back.n == m.n
    assert np.array_equal(back.c, m.c) and np.array_equal(back.lb, m.lb)
    assert np.array_equal(back.ub, m.ub) and np.array_equal(back.rl, m.rl)
    d = serve.model_to_json(m)
    d["sense"] = "max"
    mx = serve.model_from_json(d)
    assert np.array_equal(mx.c, -m.c) and getattr(mx, "sense", 1.0) == -1.0


# ---------------------------------------------------------------- the scheduler
class FakeItem:
    def __init__(self, model, opts):
        self.model, self.opts, self.freed = model, opts, False
        self.bytes = float(model.n)  # footprint: one unit per column

    def free(self):
        self.freed = True


class FakeEngine:
    """The BatchEngine surface the scheduler uses: admission by a byte budget,
    and every check interval finishes the oldest running instance."""

    def __init__(self, budget):
        self.budget, self.used = budget, 0.0
        self.running, self.admitted, self.closed = [], [], False
        self.lock = threading.Lock()

    def prepare_with(self, model, opts):
        if model.n == 0:
            raise ValueError("empty model")  # a presolve-time failure
        return FakeItem(model, opts)

    def admit(self, item, ident):
        with self.lock:
            if self.used + item.bytes > self.budget:
                return False
            self.used += item.bytes
            self.running.append((ident, item))
            self.admitted.append(ident)
            return True

    def step(self, checks=1):
        time.sleep(0.005)
        with self.lock:
            if not self.running:
                return []
            ident, item = self.running.pop(0)
            self.used -= item.bytes
            return [ident]

    def result(self, ident):
        return {"status": "OPTIMAL", "ident": ident}

    def info(self):
        return {"active": len(self.running), "used_bytes": self.used}

    def close(self):
        self.closed = True


def _lp(n):
    from niryukti_b200 import synth
    return synth.random_lp(m=n // 2, n=n, per_col=1, seed=n)


def test_scheduler_admits_in_arrival_order_under_the_budget():
    """FIFO admission under the memory budget: requests wait for memory
    (queue_s > 0), are admitted in arrival order, and every future resolves."""
    eng = FakeEngine(budget=250.0)
    svc = serve.SolveService(engine=eng, prepare_workers=1)  # prepared in arrival order
    try:
        models = [_lp(100) for _ in range(6)]  # at most two fit at once
        futs = [svc.submit(m) for m in models]
        res = [f.result(timeout=30) for f in futs]
    finally:
        svc.close()
    assert eng.admitted == list(range(6))
    assert [r["ident"] for r in res] == list(range(6))
    assert max(r["queue_s"] for r in res) > 0
    assert all(r["latency_s"] >= r["queue_s"] >= 0 for r in res)
    assert eng.closed


def test_scheduler_work_cap_runs_one_at_a_time():
    eng = FakeEngine(budget=1e9)
    svc = serve.SolveService(engine=eng, prepare_workers=1, max_active_nnz=1)
    try:
        futs = [svc.submit(_lp(60)) for _ in range(4)]
        [f.result(timeout=30) for f in futs]
        # with a one-nonzero work cap no two instances ever ran together
        assert eng.admitted == list(range(4))
    finally:
        svc.close()


def test_scheduler_reports_failures_through_the_future():
    """A request larger than the whole budget fails with MemoryError and one
    whose preparation raises fails with that error; the others still finish."""
    import pytest
    eng = FakeEngine(budget=150.0)
    svc = serve.SolveService(engine=eng, prepare_workers=1)
    try:
        too_big = svc.submit(_lp(400))
        fine = svc.submit(_lp(100))
        with pytest.raises(MemoryError):
            too_big.result(timeout=30)
        assert fine.result(timeout=30)["status"] == "OPTIMAL"
        from niryukti_b200 import synth
        empty = synth.Model(m=0, n=0, ptr=np.zeros(1, dtype=np.int64),
                            idx=np.zeros(0, dtype=np.int64), val=np.zeros(0), c=np.zeros(0),
                            q=np.zeros(0), lb=np.zeros(0), ub=np.zeros(0), rl=np.zeros(0),
                            ru=np.zeros(0))
        with pytest.raises(ValueError, match="empty model"):
            svc.submit(empty).result(timeout=30)
    finally:
        svc.close()


def test_scheduler_with_out_of_order_preparation():
    """Four prepare workers finish out of arrival order: every request is
    admitted exactly once and every future resolves once."""
    import random

    class SlowPrepare(FakeEngine):
        def prepare_with(self, model, opts):
            time.sleep(random.Random(model.n).uniform(0, 0.02))
            return super().prepare_with(model, opts)

    eng = SlowPrepare(budget=400.0)
    svc = serve.SolveService(engine=eng, prepare_workers=4)
    try:
        futs = [svc.submit(_lp(100 + 2 * k)) for k in range(24)]
        res = [f.result(timeout=60) for f in futs]
    finally:
        svc.close()
    assert sorted(eng.admitted) == list(range(24))
    assert [r["ident"] for r in res] == list(range(24))
