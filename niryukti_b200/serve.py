"""Continuous-batching solve service behind the reference's ``POST /v1/solve``.

The reference serves ``/v1/solve`` from a ThreadingHTTPServer that runs each
request as a CLI subprocess, at most ``workers`` at a time, and answers 429
when they are busy (python/niryukti/service.py:40-71).  Here every request
joins one resident batched engine on the GPU (niryukti_b200.batch):

* requests are presolved and laid out on host threads while the GPU works;
* they are admitted by device-memory footprint under a budget (150 GB by
  default) in arrival order, and join the running batch at the next check
  boundary (every ``check_every`` PDHG trials, where restarts happen);
* iterates stay on the device until an instance terminates; finished
  instances leave at once and their memory admits the next requests;
* every instance runs its own driver (steps, restarts, termination), so a
  result does not depend on what else is being solved.

The request and response JSON follow the reference: ``{"model": <native JSON
model>, "options": {...}}`` in (io.cpp read_json, service.py:54-68) and the
result_json keys out (src/io.cpp:902-995), plus ``latency`` fields.
"""
from __future__ import annotations

import collections
import json
import math
import threading
import time
from concurrent.futures import Future
from http.server import BaseHTTPRequestHandler, ThreadingHTTPServer

import numpy as np

from . import batch as nb
from .synth import Model

OPTION_KEYS = {"device", "method", "tol", "time_limit", "threads", "iterations"}


# ---------------------------------------------------------------- models
def _bound(v, fallback):
    """The reference's bound(): null -> fallback, "inf"/"-inf" strings, numbers."""
    if v is None:
        return fallback
    if isinstance(v, str):
        s = v.upper()
        if s in ("INF", "+INF"):
            return math.inf
        if s == "-INF":
            return -math.inf
        raise ValueError("Invalid bound string")
    return float(v)


def _build(rows, cols, r, c, v):
    """Sparse::build: sort by (row, column), add duplicates, drop zeros."""
    r, c, v = np.asarray(r, np.int64), np.asarray(c, np.int64), np.asarray(v, float)
    if r.size:
        order = np.lexsort((c, r))
        r, c, v = r[order], c[order], v[order]
        key = r * max(cols, 1) + c
        first = np.ones(r.size, bool)
        first[1:] = key[1:] != key[:-1]
        starts = np.flatnonzero(first)
        v = np.add.reduceat(v, starts)
        r, c = r[starts], c[starts]
        if not np.all(np.isfinite(v)):
            raise ValueError("Coefficient sum overflow")
        keep = v != 0
        r, c, v = r[keep], c[keep], v[keep]
    ptr = np.zeros(rows + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=rows), out=ptr[1:])
    return ptr, c, v


def model_from_json(d: dict) -> Model:
    """The reference's native JSON model (read_json, src/io.cpp:84-142),
    continuous variables only, canonicalised to minimisation."""
    sense = str(d.get("sense", "min")).upper()
    if sense not in ("MIN", "MINIMIZE", "MAX", "MAXIMIZE"):
        raise ValueError("Unknown objective sense")
    sgn = 1.0 if sense.startswith("MIN") else -1.0
    ids, lb, ub = {}, [], []
    for v in d["variables"]:
        name = v["name"]
        if name in ids:
            raise ValueError("Duplicate variable")
        if v.get("type", "continuous") != "continuous":
            raise ValueError("The PDHG service solves continuous models only")
        ids[name] = len(ids)
        lb.append(_bound(v.get("lb", 0), -math.inf))
        ub.append(_bound(v.get("ub"), math.inf))
    n = len(ids)
    obj = d["objective"]
    c = np.asarray(obj["linear"], float) * sgn
    q = np.asarray(obj.get("quadratic_diagonal", [0.0] * n), float) * sgn
    if c.shape != (n,) or q.shape != (n,):
        raise ValueError("Inconsistent model dimensions")
    if "quadratic" in obj:
        raise ValueError("Use explicit symmetric quadratic_sparse triples")
    rr, cc, vv, rl, ru = [], [], [], [], []
    for i, row in enumerate(d["constraints"]):
        rl.append(_bound(row.get("lb"), -math.inf))
        ru.append(_bound(row.get("ub"), math.inf))
        for key, val in row["coefficients"].items():
            if key not in ids:
                raise ValueError("Unknown variable: " + key)
            rr.append(i)
            cc.append(ids[key])
            vv.append(float(val))
    m = len(rl)
    ptr, idx, val = _build(m, n, rr, cc, vv)
    model = Model(m=m, n=n, ptr=ptr, idx=idx, val=val, c=c, q=q, lb=np.array(lb),
                  ub=np.array(ub), rl=np.array(rl), ru=np.array(ru),
                  offset=float(obj.get("offset", 0.0)) * sgn, name=str(d.get("name", "model")))
    if obj.get("quadratic_sparse"):
        t = np.asarray(obj["quadratic_sparse"], float)
        if t.ndim != 2 or t.shape[1] != 3:
            raise ValueError("quadratic_sparse entries must be [row,column,value]")
        model.qptr, model.qidx, model.qval = _build(n, n, t[:, 0].astype(np.int64),
                                                    t[:, 1].astype(np.int64), t[:, 2] * sgn)
    model.sense = sgn
    model.variable_names = list(ids)
    return model


def model_to_json(model: Model) -> dict:
    """The native JSON of a (minimisation) model, as json_model writes it."""
    names = [f"x{j}" for j in range(model.n)]
    cons = []
    for i in range(model.m):
        s, e = int(model.ptr[i]), int(model.ptr[i + 1])
        cons.append({"name": f"r{i}", "lb": _enc(model.rl[i]), "ub": _enc(model.ru[i]),
                     "coefficients": {names[int(j)]: float(v)
                                      for j, v in zip(model.idx[s:e], model.val[s:e])}})
    obj = {"linear": model.c.tolist(), "quadratic_diagonal": model.q.tolist(),
           "offset": float(model.offset)}
    if model.qnnz:
        rows = np.repeat(np.arange(model.n), np.diff(model.qptr))
        obj["quadratic_sparse"] = [[int(a), int(b), float(v)]
                                   for a, b, v in zip(rows, model.qidx, model.qval)]
    return {"name": model.name, "sense": "min",
            "variables": [{"name": names[j], "lb": _enc(model.lb[j]), "ub": _enc(model.ub[j])}
                          for j in range(model.n)],
            "constraints": cons, "objective": obj}


def _finite(o):
    """JSON without NaN/Infinity: non-finite numbers become "inf"/"-inf"/null."""
    if isinstance(o, float):
        return o if math.isfinite(o) else (None if math.isnan(o) else _enc(o))
    if isinstance(o, dict):
        return {k: _finite(v) for k, v in o.items()}
    if isinstance(o, (list, tuple)):
        return [_finite(v) for v in o]
    return o


def _enc(v):
    return v if math.isfinite(v) else ("inf" if v > 0 else "-inf")


def result_json(model: Model, r: dict) -> dict:
    """The reference's result keys (src/io.cpp:902-995) for a continuous solve."""
    sgn = getattr(model, "sense", 1.0)
    finite = math.isfinite(r["kkt"])
    return {
        "solver": "NIRYUKTI-B200", "status": r["status"],
        "problem_type": "QP" if model.is_qp() else "LP",
        "model": {"name": model.name, "rows": model.m, "columns": model.n, "nonzeros": model.nnz},
        "objective": sgn * r["objective"] if finite else None,
        "accuracy": {"finite": finite, "primal_residual": r["primal"],
                     "dual_residual": r["dual"], "relative_gap": r["gap"],
                     "kkt_error": r["kkt"], "dual_bound": r["lower_bound"]},
        "performance": {"total_seconds": r["seconds"],
                        "preprocess_seconds": r["preprocess_seconds"],
                        "transfer_setup_seconds": r["transfer_seconds"],
                        "iteration_seconds": r["iteration_seconds"],
                        "verification_seconds": r["verification_seconds"],
                        "iterations": r["iterations"], "restarts": r["restarts"],
                        "weight_updates": r["weight_updates"],
                        "rejected_steps": r["rejected_steps"]},
        "hardware": {"backend": "cuda-b200-batch", "precision": r["matrix_precision"]},
        "presolve": {"removed_rows": r["removed_rows"],
                     "removed_columns": r["removed_columns"]},
        "primal": r["x"].tolist(), "dual": r["y"].tolist(),
    }


# ---------------------------------------------------------------- the service
class SolveService:
    """One batched engine, a host prepare pool and a scheduler thread."""

    def __init__(self, *, memory_budget=150e9, matrix_precision="mixed", tol=1e-6,
                 iteration_limit=100000, time_limit=600.0, check_every=100,
                 prepare_workers=8, autotune=True, max_active_nnz=16_000_000, engine=None):
        """memory_budget: device bytes for resident instances (admission by
        footprint).  max_active_nnz: work cap of the running batch (nonzeros
        of A and Q over the admitted instances).  A batch trial over 16 M
        nonzeros already keeps the GPU's memory system busy (about 0.2 ms per
        trial); admitting more work makes every trial longer without raising
        throughput, so admitted instances would only finish later.  engine
        (optional): an object with the BatchEngine methods the scheduler uses
        (prepare_with, admit, step, result, info, close) in place of a new
        BatchEngine -- e.g. a stand-in that exercises the scheduling on a host
        without a GPU."""
        self.tol = tol
        self.max_active_nnz = max_active_nnz
        self._active_nnz = 0
        self.limits = dict(iteration_limit=iteration_limit, time_limit=time_limit)
        self.engine = engine if engine is not None else nb.BatchEngine(
            tol=tol, matrix_precision=matrix_precision, memory_budget=memory_budget,
            check_every=check_every, autotune=autotune, **self.limits)
        self.precision = matrix_precision
        self.prefetch = max(2 * prepare_workers, 32)  # prepared requests kept ahead
        self._incoming = collections.deque()  # (id, model, options, future, arrival)
        self._ready = collections.deque()     # prepared, waiting for admission (FIFO)
        self._preparing = 0
        self._running = {}                    # id -> (future, arrival, admitted, nnz)
        self._cv = threading.Condition()
        self._next = 0
        self._stop = False
        self._workers = [threading.Thread(target=self._prepare_loop, name=f"nk-prepare-{k}",
                                          daemon=True) for k in range(prepare_workers)]
        for w in self._workers:
            w.start()
        self._thread = threading.Thread(target=self._loop, name="nk-serve", daemon=True)
        self._thread.start()

    def submit(self, model: Model, iteration_limit=None, time_limit=None) -> Future:
        """Queue a solve; the future resolves to the solver's result dict plus
        ``latency_s`` (arrival to result) and ``queue_s`` (arrival to admission)."""
        fut = Future()
        arrival = time.perf_counter()
        opts = nb.batch_options(tol=self.tol, matrix_precision=self.precision,
                                iteration_limit=int(iteration_limit or self.limits["iteration_limit"]),
                                time_limit=float(time_limit or self.limits["time_limit"]))
        with self._cv:
            ident = self._next
            self._next += 1
            self._incoming.append((ident, model, opts, fut, arrival))
            self._cv.notify_all()
        return fut

    def _prepare_loop(self):
        """Host work (presolve, scaling, layout) for the next requests in
        arrival order, at most `prefetch` ahead of admission."""
        while True:
            with self._cv:
                while not self._stop and (not self._incoming or
                                          len(self._ready) + self._preparing >= self.prefetch):
                    self._cv.wait(timeout=0.1)
                if self._stop:
                    return
                ident, model, opts, fut, arrival = self._incoming.popleft()
                self._preparing += 1
            try:
                item = self.engine.prepare_with(model, opts)
                err = None
            except Exception as exc:  # reported through the future
                item, err = None, exc
            with self._cv:
                self._preparing -= 1
                if err is None:
                    # prepared requests wait in arrival order, whichever worker finished first
                    entry = (ident, item, fut, arrival, model.nnz + model.qnnz)
                    at = len(self._ready)
                    while at > 0 and self._ready[at - 1][0] > ident:
                        at -= 1
                    self._ready.insert(at, entry)
                self._cv.notify_all()
            if err is not None:
                fut.set_exception(err)

    def stats(self) -> dict:
        with self._cv:
            waiting = len(self._ready) + len(self._incoming)
            running = len(self._running)
        return {"waiting": waiting, "running": running, **self.engine.info()}

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        self._thread.join()
        for w in self._workers:
            w.join()
        for _, item, fut, _, _ in self._ready:
            item.free()
            fut.cancel()
        for _, _, _, fut, _ in self._incoming:
            fut.cancel()
        for fut, _, _, _ in self._running.values():
            fut.cancel()
        self.engine.close()

    def _loop(self):
        while True:
            with self._cv:
                if self._stop:
                    return
                if not self._ready and not self._running:
                    self._cv.wait(timeout=0.02)
                    continue
                ready = list(self._ready)
            # admission in arrival order, while the memory budget and the work
            # cap allow (an instance larger than the cap runs alone)
            admitted = set()
            for ident, item, fut, arrival, nnz in ready:
                if self._running and self._active_nnz + nnz > self.max_active_nnz:
                    break
                if not self.engine.admit(item, ident):
                    break
                self._running[ident] = (fut, arrival, time.perf_counter(), nnz)
                self._active_nnz += nnz
                admitted.add(ident)
            if admitted:
                # by identity: a worker may have inserted an earlier arrival meanwhile
                with self._cv:
                    self._ready = collections.deque(e for e in self._ready
                                                    if e[0] not in admitted)
                    self._cv.notify_all()  # room to prepare more
            if not self._running:
                if ready:  # the head does not fit even an empty batch
                    ident, item, fut, _, _ = ready[0]
                    with self._cv:
                        self._ready = collections.deque(e for e in self._ready
                                                        if e[0] != ident)
                    item.free()
                    fut.set_exception(MemoryError("model exceeds the service's memory budget"))
                continue
            for ident in self.engine.step(checks=1):  # one check interval
                fut, arrival, admitted_at, nnz = self._running.pop(ident)
                self._active_nnz -= nnz
                r = self.engine.result(ident)
                now = time.perf_counter()
                r["latency_s"] = now - arrival
                r["queue_s"] = admitted_at - arrival
                fut.set_result(r)


def make_server(service: SolveService, host="127.0.0.1", port=8000, max_time=600.0,
                max_pending=None):
    """HTTP front door: POST /v1/solve as in python/niryukti/service.py:40-71
    (inline native JSON model, options {device, method, tol, time_limit,
    threads, iterations}); the CLI subprocess and worker cap are replaced by
    the batched engine.  max_pending (optional) bounds the requests in flight:
    beyond it a request is answered 429, as the reference answers when all its
    solver workers are occupied (service.py:63-64)."""
    pending = [0]
    lock = threading.Lock()

    class Handler(BaseHTTPRequestHandler):
        def log_message(self, *args):
            pass

        def send(self, code, obj):
            body = json.dumps(_finite(obj), allow_nan=False).encode()
            self.send_response(code)
            self.send_header("Content-Type", "application/json")
            self.send_header("Content-Length", str(len(body)))
            self.end_headers()
            self.wfile.write(body)

        def do_POST(self):
            if self.path != "/v1/solve":
                return self.send(404, {"error": "Unknown route"})
            try:
                length = int(self.headers.get("Content-Length", "0"))
                if not 0 < length <= 256 * 1024 * 1024:
                    return self.send(413, {"error": "JSON payload limit: 256 MiB"})
                data = json.loads(self.rfile.read(length))
                if not isinstance(data, dict):
                    raise ValueError("Expected JSON object")
                if set(data) - {"model", "options"}:
                    raise ValueError("Unknown solve fields")
                if not isinstance(data.get("model"), dict):
                    raise ValueError("Provide an inline native JSON model")
                options = data.get("options", {})
                if not isinstance(options, dict) or set(options) - OPTION_KEYS:
                    raise ValueError("Unsupported solve options")
                if options.get("method", "pdhg") not in ("pdhg", "auto"):
                    raise ValueError("This service runs the PDHG method")
                if options.get("device", "cuda") not in ("cuda", "auto"):
                    raise ValueError("This service runs on the GPU")
                if float(options.get("tol", service.tol)) != service.tol:
                    raise ValueError(f"This service solves to tol={service.tol}")
                tl = float(options.get("time_limit", 60))
                if not 0 < tl <= max_time:
                    raise ValueError("Time limit exceeds API resource policy")
                model = model_from_json(data["model"])
                with lock:
                    full = max_pending is not None and pending[0] >= max_pending
                    if not full:
                        pending[0] += 1
                if full:
                    return self.send(429, {"error": "All solver slots are occupied"})
                try:
                    fut = service.submit(model, iteration_limit=options.get("iterations"),
                                         time_limit=tl)
                    r = fut.result()
                finally:
                    with lock:
                        pending[0] -= 1
                out = result_json(model, r)
                out["latency_seconds"] = r["latency_s"]
                out["queue_seconds"] = r["queue_s"]
                self.send(200, out)
            except (ValueError, TypeError, KeyError, OverflowError, MemoryError,
                    RuntimeError) as error:
                self.send(400, {"error": str(error)[:2048]})

    server = ThreadingHTTPServer((host, port), Handler)
    server.daemon_threads = True
    return server
