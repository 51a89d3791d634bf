"""Serving (niryukti_b200.serve): continuous batching behind /v1/solve.

Requests arrive while others are on the GPU, are admitted as memory and the
work cap allow, and run side by side in one batched engine.  Each result must
be the same alone and in the mix, within the stated tolerance: certified to
1e-6 relative KKT, objective within the bound that tolerance implies.
"""
import json
import threading
import time
import urllib.error
import urllib.request

import numpy as np
import pytest

from niryukti_b200 import synth
from tests.test_oracle import sparse_qp_model

pytestmark = pytest.mark.gpu

TOL = 1e-6


def close(a, b, tol=TOL):
    assert abs(a - b) <= 2 * tol * (1 + abs(b)), (a, b)


@pytest.fixture(scope="module")
def serve(gpu):
    from niryukti_b200 import serve as s
    return s


def mix(count=6, seed=21):
    return synth.batch_instances(count=count, m_lo=40, m_hi=400, qp_frac=0.34, seed=seed)


def test_same_result_alone_and_in_the_mix(serve):
    from niryukti_b200 import batch, solver
    models = mix()
    # a request that joins after the first (autotuning) check interval skips its timed
    # trials, so its path to tolerance can be longer than alone: a generous cap
    svc = serve.SolveService(memory_budget=4e9, matrix_precision="mixed", prepare_workers=4,
                             iteration_limit=400000)
    try:
        futs = []
        for k, m in enumerate(models):  # staggered arrivals while earlier ones run
            futs.append(svc.submit(m))
            time.sleep(0.02 * k)
        res = [f.result(timeout=300) for f in futs]
    finally:
        svc.close()
    for m, r in zip(models, res):
        assert r["status"] == "OPTIMAL", (r["status"], r["kkt"])
        assert solver.verify(m, r["x"], r["y"])["kkt"] <= TOL
        alone = batch.solve_batch([m], matrix_precision="mixed")[0]
        assert alone["status"] == "OPTIMAL"
        close(r["objective"], alone["objective"])
        assert r["latency_s"] >= r["queue_s"] >= 0


def test_admission_waits_for_memory(serve):
    """A budget that holds only the largest request: requests queue for memory
    and all finish, at the service's defaults (MIXED matrices, the reference's
    100,000-iteration cap).  The autotuner's probe trials leave no trace, so a
    request's trajectory does not depend on whether it shared the first check
    interval."""
    models = mix(count=4, seed=23)
    from niryukti_b200 import batch
    need = max(batch.BatchEngine(matrix_precision="mixed").prepare(m).device_bytes
               for m in models)
    svc = serve.SolveService(memory_budget=need * 1.2, matrix_precision="mixed")
    try:
        futs = [svc.submit(m) for m in models]
        res = [f.result(timeout=300) for f in futs]
    finally:
        svc.close()
    assert all(r["status"] == "OPTIMAL" for r in res), [(r["status"], r.get("kkt"),
                                                         r.get("iterations")) for r in res]
    assert max(r["queue_s"] for r in res) > 0  # someone waited for memory


def test_http_solve_route(serve):
    svc = serve.SolveService(memory_budget=2e9, matrix_precision="mixed")
    server = serve.make_server(svc, port=0)
    port = server.server_address[1]
    t = threading.Thread(target=server.serve_forever, daemon=True)
    t.start()

    def post(path, payload):
        req = urllib.request.Request(f"http://127.0.0.1:{port}{path}",
                                     data=json.dumps(payload).encode(),
                                     headers={"Content-Type": "application/json"})
        try:
            with urllib.request.urlopen(req, timeout=120) as r:
                return r.status, json.loads(r.read())
        except urllib.error.HTTPError as e:
            return e.code, json.loads(e.read())
    try:
        body = {"model": serve.model_to_json(sparse_qp_model()),
                "options": {"device": "cuda", "method": "pdhg", "tol": 1e-6, "time_limit": 30}}
        code, out = post("/v1/solve", body)
        assert code == 200 and out["status"] == "OPTIMAL", out
        assert abs(out["objective"] + 7) < 1e-5 and out["problem_type"] == "QP"
        assert np.allclose(out["primal"], [1, 2], atol=1e-4)
        # a maximisation model: the objective comes back in the caller's sense
        mx = serve.model_to_json(sparse_qp_model())
        mx["sense"] = "max"
        mx["objective"]["linear"] = [4.0, 5.0]
        mx["objective"]["quadratic_sparse"] = [[a, b, -v] for a, b, v in
                                               mx["objective"]["quadratic_sparse"]]
        code, out = post("/v1/solve", {"model": mx})
        assert code == 200 and abs(out["objective"] - 7) < 1e-5
        assert post("/v1/solve", {"model": body["model"], "options": {"tol": 1e-3}})[0] == 400
        assert post("/v1/solve", {"model": body["model"], "options": {"bogus": 1}})[0] == 400
        assert post("/v1/other", body)[0] == 404
    finally:
        server.shutdown()
        svc.close()
