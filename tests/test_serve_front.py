"""The /v1/solve front door on the CPU, with a stand-in for the batched engine.

The HTTP layer (python/niryukti/service.py:40-71 in the reference) validates a
request, turns the native JSON model into a Model, submits it and answers with
the reference's result keys.  Here the engine is replaced by a fake service
whose solves finish only when the test releases them, so saturation (429),
validation errors (400, 404, 413) and the JSON round trip are exercised without
a GPU: failures are injected on the host."""
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
