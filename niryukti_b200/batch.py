"""Python mirror of the batched engine (include/nk_pdhg.h, nk_batch family).

``solve_batch(models, **options)`` solves many independent LPs / convex QPs
together on one GPU: each instance runs the reference's continuous PDHG driver
(solve_continuous, src/solver.cpp:213-780) with its own steps, restarts and
termination, while one set of kernel launches advances all of them.
``BatchEngine`` is the incremental form the serving loop uses: prepare
requests on any thread, admit them by device-memory footprint, step, collect
results as instances finish.  Every call goes through libnkpdhg.so.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from .engine import PRECISIONS, _D, _I, check, library
from .solver import NkModel, NkSolveResult, STATUS, _ModelView


class NkBatchOptions(C.Structure):
    _fields_ = [("tol", C.c_double), ("time_limit", C.c_double), ("iteration_limit", C.c_int64),
                ("check_every", C.c_int), ("presolve", C.c_int), ("scaling_combined", C.c_int),
                ("scaling_passes", C.c_int), ("adaptive", C.c_int), ("restart", C.c_int),
                ("graphs", C.c_int), ("autotune", C.c_int), ("precision", C.c_int),
                ("phase_tol", C.c_double), ("memory_budget", C.c_double), ("capacity", C.c_int)]


def _bind():
    L = library()
    if getattr(L, "_nk_batch_bound", False):
        return L
    from .solver import _bind as bind_solver
    bind_solver()
    P = C.c_void_p
    L.nk_batch_defaults.argtypes = [C.POINTER(NkBatchOptions)]
    L.nk_batch_defaults.restype = None
    L.nk_batch_create.argtypes = [C.POINTER(NkBatchOptions), C.POINTER(P)]
    L.nk_batch_destroy.argtypes = [P]
    L.nk_batch_destroy.restype = None
    L.nk_batch_estimate.argtypes = [C.POINTER(NkModel), _D]
    L.nk_batch_prepare.argtypes = [C.POINTER(NkModel), C.POINTER(NkBatchOptions), C.POINTER(P), _D]
    L.nk_batch_item_free.argtypes = [P]
    L.nk_batch_item_free.restype = None
    L.nk_batch_admit.argtypes = [P, P, C.c_int64, C.POINTER(C.c_int)]
    L.nk_batch_step.argtypes = [P, C.c_int, _I, C.c_int, C.POINTER(C.c_int)]
    L.nk_batch_result.argtypes = [P, C.c_int64, C.POINTER(NkSolveResult), _D, _D]
    L.nk_batch_info.argtypes = [P, C.POINTER(C.c_int), _D, _D, C.POINTER(C.c_int),
                                C.POINTER(C.c_int)]
    L.nk_batch_time_trials.argtypes = [P, C.c_int, _D, _I]
    L.nk_batch_kernel_times.argtypes = [P, _D, _D]
    L.nk_batch_progress.argtypes = [P, C.c_int64, _D]
    L.nk_batch_phase_seconds.argtypes = [P, _D]
    L._nk_batch_bound = True
    return L


def batch_options(*, tol=1e-6, time_limit=60.0, iteration_limit=100000, check_every=100,
                  presolve=True, scaling="ruiz", scaling_passes=5, adaptive=True, restart=True,
                  cuda_graphs=True, autotune=True, matrix_precision="fp64", phase_tol=0.0,
                  memory_budget=0.0, capacity=4096) -> NkBatchOptions:
    L = _bind()
    if scaling not in ("ruiz", "combined"):
        raise ValueError("scaling must be 'ruiz' or 'combined'")
    o = NkBatchOptions()
    L.nk_batch_defaults(C.byref(o))
    o.tol, o.time_limit, o.iteration_limit = float(tol), float(time_limit), int(iteration_limit)
    o.check_every, o.presolve = int(check_every), int(bool(presolve))
    o.scaling_combined, o.scaling_passes = int(scaling == "combined"), int(scaling_passes)
    o.adaptive, o.restart = int(bool(adaptive)), int(bool(restart))
    o.graphs, o.autotune = int(bool(cuda_graphs)), int(bool(autotune))
    o.precision = PRECISIONS[matrix_precision]
    if matrix_precision not in ("fp64", "mixed"):
        raise ValueError("batched matrices are fp64 or mixed")
    o.phase_tol = float(phase_tol)
    o.memory_budget, o.capacity = float(memory_budget), int(capacity)
    return o


class PreparedInstance:
    """A presolved, scaled, laid-out instance waiting for admission (host only)."""

    def __init__(self, handle, n, m, device_bytes):
        self.handle, self.n, self.m, self.device_bytes = handle, n, m, device_bytes

    def free(self):
        if self.handle:
            _bind().nk_batch_item_free(self.handle)
            self.handle = None

    def __del__(self):
        self.free()


def _result(r: NkSolveResult, x, y, precision) -> dict:
    out = {k: getattr(r, k) for k, _ in NkSolveResult._fields_ if k != "reached"}
    out["status"] = STATUS[r.status]
    out["time_to_kkt"] = {f"1e-{k}": r.reached[k] for k in range(9) if r.reached[k] >= 0}
    out["kkt_error"] = r.kkt
    out["matrix_precision"] = precision
    out["x"], out["y"] = x, y
    return out


class BatchEngine:
    """Many instances on one GPU; single-threaded except for prepare()."""

    def __init__(self, **options):
        self._L = _bind()
        self.precision = options.get("matrix_precision", "fp64")
        self.options = batch_options(**options)
        self._h = C.c_void_p()
        check(self._L.nk_batch_create(C.byref(self.options), C.byref(self._h)))
        self._shapes = {}
        self._lock = threading.Lock()

    def close(self):
        if self._h:
            self._L.nk_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def prepare(self, model) -> PreparedInstance:
        """Thread-safe: presolve, scaling, start-point checks, layout."""
        return self.prepare_with(model, self.options)

    def prepare_with(self, model, options: NkBatchOptions) -> PreparedInstance:
        """prepare() with an instance's own limits (iteration and time limit;
        the tolerance and precision must be the batch's)."""
        view = _ModelView(model)
        h = C.c_void_p()
        b = C.c_double()
        check(self._L.nk_batch_prepare(C.byref(view.s), C.byref(options), C.byref(h),
                                       C.byref(b)))
        return PreparedInstance(h, int(model.n), int(model.m), b.value)

    def admit(self, item: PreparedInstance, ident: int) -> bool:
        ok = C.c_int()
        check(self._L.nk_batch_admit(self._h, item.handle, int(ident), C.byref(ok)))
        if ok.value:
            item.handle = None  # the batch owns it now
            self._shapes[int(ident)] = (item.n, item.m)
        return bool(ok.value)

    def step(self, checks=1, capacity=4096):
        ids = np.zeros(capacity, dtype=np.int64)
        count = C.c_int()
        check(self._L.nk_batch_step(self._h, int(checks), ids.ctypes.data_as(_I), capacity,
                                    C.byref(count)))
        return ids[:count.value].tolist()

    def result(self, ident: int) -> dict:
        n, m = self._shapes.pop(int(ident))
        x, y = np.zeros(n), np.zeros(m)
        r = NkSolveResult()
        check(self._L.nk_batch_result(self._h, int(ident), C.byref(r), x.ctypes.data_as(_D),
                                      y.ctypes.data_as(_D)))
        return _result(r, x, y, self.precision)

    def info(self) -> dict:
        a, vp, vd = C.c_int(), C.c_int(), C.c_int()
        u, b = C.c_double(), C.c_double()
        check(self._L.nk_batch_info(self._h, C.byref(a), C.byref(u), C.byref(b), C.byref(vp),
                                    C.byref(vd)))
        def variant(v):  # the autotuner's choice: chunks per work item, unroll, CTA size
            return {"run": (1, 4, 16)[v // 9], "unroll": (2, 4, 8)[v // 3 % 3],
                    "threads": (128, 256, 512)[v % 3]}
        return {"active": a.value, "used_bytes": u.value, "budget_bytes": b.value,
                "primal_variant": variant(vp.value), "dual_variant": variant(vd.value)}

    def progress(self, ident: int) -> dict:
        v = np.zeros(8)
        check(self._L.nk_batch_progress(self._h, int(ident), v.ctypes.data_as(_D)))
        keys = ("iterations", "restarts", "best_kkt", "weight", "step", "since_restart",
                "restart_kkt", "fp64")
        return dict(zip(keys, v.tolist()))

    def phase_seconds(self) -> dict:
        v = np.zeros(7)
        check(self._L.nk_batch_phase_seconds(self._h, v.ctypes.data_as(_D)))
        return dict(zip(("controls", "trials", "evaluation", "driver", "restarts", "close",
                         "lists"), v.tolist()))

    def kernel_times(self):
        """The autotuner's best primal and dual kernel times (ms)."""
        p, d = C.c_double(), C.c_double()
        check(self._L.nk_batch_kernel_times(self._h, C.byref(p), C.byref(d)))
        return p.value, d.value

    def time_trials(self, trials):
        ms = C.c_double()
        bts = C.c_int64()
        check(self._L.nk_batch_time_trials(self._h, int(trials), C.byref(ms), C.byref(bts)))
        return ms.value, bts.value


def estimate_bytes(model) -> float:
    """The reference's device-memory estimate (48 B/nnz + 240 B per row and column)."""
    L = _bind()
    view = _ModelView(model)
    b = C.c_double()
    check(L.nk_batch_estimate(C.byref(view.s), C.byref(b)))
    return b.value


def solve_batch(models, **options) -> list:
    """Solve every model; results in input order.  Instances that do not fit
    the memory budget wait and join as earlier ones finish."""
    with BatchEngine(**options) as eng:
        items = [eng.prepare(m) for m in models]
        results = [None] * len(models)
        waiting = list(range(len(models)))
        while waiting or eng.info()["active"]:
            still = []
            for k in waiting:
                if not eng.admit(items[k], k):
                    still.append(k)
            if still and len(still) == len(waiting) and not eng.info()["active"]:
                raise MemoryError("an instance does not fit the batch's memory budget")
            waiting = still
            for k in eng.step(checks=1000000):
                results[k] = eng.result(k)
        return results
