"""Python mirror of the engine's solve path (include/nk_pdhg.h, nk_solve family).

``solve(model, **options)`` is the reference's continuous PDHG solve
(``vantage::solve`` with ``method="pdhg"``, src/solver.cpp:213-780) with the
iterations, candidate checks and restarts resident on the GPU; ``prepare`` and
``verify`` expose the host presolve/scaling (src/preprocess.cpp:133-346) and the
reference verifier (src/verify.cpp:103-244) of the same library.  Option names
follow ``vantage::Options`` (include/vantage/vantage.hpp:41-60) and result keys
the reference's result JSON (src/io.cpp:902-995).  Every call goes through
libnkpdhg.so; there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .engine import NkCsr, PRECISIONS, _D, _I, _f64, _i64, check, library

STATUS = {0: "OPTIMAL", 1: "INFEASIBLE", 2: "UNBOUNDED", 3: "ITERATION_LIMIT", 4: "TIME_LIMIT",
          5: "NUMERICAL_ERROR", 6: "INTERRUPTED"}


class CancelToken:
    """Stops a running solve() at its next check (status INTERRUPTED) when
    cancel() is called from another thread -- the reference's
    Options::cancellation."""

    def __init__(self):
        self.flag = C.c_int(0)

    def cancel(self):
        self.flag.value = 1

    @property
    def cancelled(self) -> bool:
        return bool(self.flag.value)
ACCURACY_KEYS = ("objective", "primal", "dual", "gap", "kkt", "primal_absolute", "dual_absolute",
                 "complementarity", "lower_bound", "finite")


class NkModel(C.Structure):
    _fields_ = [("A", NkCsr), ("Q", NkCsr), ("c", _D), ("q", _D), ("lb", _D), ("ub", _D),
                ("rl", _D), ("ru", _D), ("offset", C.c_double)]


class NkSolveOptions(C.Structure):
    _fields_ = [("tol", C.c_double), ("time_limit", C.c_double), ("iteration_limit", C.c_int64),
                ("check_every", C.c_int), ("presolve", C.c_int), ("scaling_combined", C.c_int),
                ("scaling_passes", C.c_int), ("adaptive", C.c_int), ("restart", C.c_int),
                ("graphs", C.c_int), ("index_bits", C.c_int), ("precision", C.c_int),
                ("refine", C.c_int), ("phase_tol", C.c_double), ("verbose", C.c_int),
                ("initial_x", _D), ("initial_y", _D), ("cancel", C.POINTER(C.c_int))]


class NkSolveResult(C.Structure):
    _fields_ = [("status", C.c_int),
                *[(k, C.c_int64) for k in (
                    "iterations", "restarts", "rejected_steps", "weight_updates",
                    "device_checks", "host_checks", "removed_rows", "removed_columns",
                    "phase_iterations", "refine_iterations")],
                *[(k, C.c_double) for k in (
                    "seconds", "preprocess_seconds", "transfer_seconds", "iteration_seconds",
                    "verification_seconds", "phase_seconds", "objective", "kkt", "primal",
                    "dual", "gap", "lower_bound", "phase_objective", "phase_kkt",
                    "phase_primal", "phase_dual", "phase_gap")],
                ("reached", C.c_double * 9)]


def _bind():
    L = library()
    if getattr(L, "_nk_solve_bound", False):
        return L
    L.nk_solve_defaults.argtypes = [C.POINTER(NkSolveOptions)]
    L.nk_solve_defaults.restype = None
    L.nk_solve.argtypes = [C.POINTER(NkModel), C.POINTER(NkSolveOptions),
                           C.POINTER(NkSolveResult), _D, _D]
    L.nk_prepare.argtypes = [C.POINTER(NkModel), C.c_int, C.c_int, C.c_int,
                             C.POINTER(C.c_void_p)]
    L.nk_prepared_free.argtypes = [C.c_void_p]
    L.nk_prepared_free.restype = None
    L.nk_prepared_dims.argtypes = [C.c_void_p, _I]
    L.nk_prepared_get.argtypes = [C.c_void_p, _I, _I, _D, _D, _D, _D, _D, _D, _D, _I, _I, _I,
                                  _I, _D, _D, _D, _D, _I, _I, _D]
    L.nk_verify.argtypes = [C.POINTER(NkModel), _D, _D, C.c_int, _D]
    L.nk_infeasibility_bound.argtypes = [C.POINTER(NkModel), _D, _D]
    L._nk_solve_bound = True
    return L


class _ModelView:
    """Keeps the contiguous arrays of a model alive behind an NkModel."""

    def __init__(self, model):
        n, m = int(model.n), int(model.m)
        self.keep = []

        def arr(a, f):
            v = f(a)
            self.keep.append(v)
            return v

        def csr(rows, cols, ptr, idx, val):
            p, i, v = arr(ptr, _i64), arr(idx, _i64), arr(val, _f64)
            return NkCsr(rows, cols, p.ctypes.data_as(_I), i.ctypes.data_as(_I),
                         v.ctypes.data_as(_D))

        A = csr(m, n, model.ptr, model.idx, model.val)
        if getattr(model, "qnnz", 0):
            Q = csr(n, n, model.qptr, model.qidx, model.qval)
        else:
            Q = NkCsr(0, 0, None, None, None)

        def vec(v, size, fill=0.0):
            a = arr(np.full(size, fill) if v is None else v, _f64)
            if a.shape != (size,):
                raise ValueError(f"vector of {a.shape} where {size} entries are expected")
            return a.ctypes.data_as(_D)

        self.s = NkModel(A, Q, vec(model.c, n), vec(getattr(model, "q", None), n),
                         vec(model.lb, n), vec(model.ub, n), vec(model.rl, m), vec(model.ru, m),
                         float(getattr(model, "offset", 0.0)))


def default_options() -> dict:
    o = NkSolveOptions()
    _bind().nk_solve_defaults(C.byref(o))
    return {k: getattr(o, k) for k, _ in NkSolveOptions._fields_
            if k not in ("initial_x", "initial_y")}


def solve(model, *, tol=1e-6, time_limit=60.0, iteration_limit=100000, check_every=100,
          presolve=True, scaling="ruiz", scaling_passes=5, adaptive=True, restart=True,
          cuda_graphs=True, gpu_indices="auto", matrix_precision="fp64", refine=True,
          phase_tol=0.0, verbose=False, initial_x=None, initial_y=None,
          cancel: "CancelToken | None" = None) -> dict:
    """Solve an LP / convex QP on the GPU; returns the reference's result keys
    plus ``x`` and ``y`` (caller order, original units).  ``cancel``: a
    CancelToken another thread may trigger (status INTERRUPTED)."""
    L = _bind()
    if scaling not in ("ruiz", "combined"):
        raise ValueError("scaling must be 'ruiz' or 'combined'")
    if gpu_indices not in ("auto", "32", "64", 0, 32, 64):
        raise ValueError("gpu_indices must be auto, 32 or 64")
    view = _ModelView(model)
    o = NkSolveOptions()
    L.nk_solve_defaults(C.byref(o))
    o.tol, o.time_limit, o.iteration_limit = float(tol), float(time_limit), int(iteration_limit)
    o.check_every, o.presolve = int(check_every), int(bool(presolve))
    o.scaling_combined, o.scaling_passes = int(scaling == "combined"), int(scaling_passes)
    o.adaptive, o.restart, o.graphs = int(bool(adaptive)), int(bool(restart)), int(bool(cuda_graphs))
    o.index_bits = 0 if gpu_indices in ("auto", 0) else int(gpu_indices)
    o.precision = PRECISIONS[matrix_precision]
    o.refine, o.phase_tol, o.verbose = int(bool(refine)), float(phase_tol), int(bool(verbose))
    ix = iy = None
    if initial_x is not None:
        ix = _f64(initial_x)
        o.initial_x = ix.ctypes.data_as(_D)
    if initial_y is not None:
        iy = _f64(initial_y)
        o.initial_y = iy.ctypes.data_as(_D)
    if cancel is not None:
        o.cancel = C.pointer(cancel.flag)
    x = np.zeros(int(model.n))
    y = np.zeros(int(model.m))
    r = NkSolveResult()
    check(L.nk_solve(C.byref(view.s), C.byref(o), C.byref(r), x.ctypes.data_as(_D),
                     y.ctypes.data_as(_D)))
    out = {k: getattr(r, k) for k, _ in NkSolveResult._fields_ if k != "reached"}
    out["status"] = STATUS[r.status]
    # seconds until the best candidate's KKT error first reached 10^-k
    out["time_to_kkt"] = {f"1e-{k}": r.reached[k] for k in range(9) if r.reached[k] >= 0}
    out["kkt_error"] = r.kkt
    out["primal_residual"], out["dual_residual"], out["relative_gap"] = r.primal, r.dual, r.gap
    out["total_seconds"] = r.seconds
    out["matrix_precision"] = matrix_precision
    out["x"], out["y"] = x, y
    return out


def prepare(model, presolve=True, scaling="ruiz", scaling_passes=5) -> dict:
    """The prepared model and its maps (Prepared, src/internal.hpp:16-25)."""
    L = _bind()
    view = _ModelView(model)
    h = C.c_void_p()
    check(L.nk_prepare(C.byref(view.s), int(bool(presolve)), int(scaling == "combined"),
                       int(scaling_passes), C.byref(h)))
    try:
        dims = np.zeros(5, dtype=np.int64)
        check(L.nk_prepared_dims(h, dims.ctypes.data_as(_I)))
        m, n, nnz, qnnz, failed = (int(v) for v in dims)
        if failed:
            return {"failure": "INFEASIBLE"}
        i64 = lambda k: np.zeros(k, dtype=np.int64)
        out = dict(ptr=i64(m + 1), idx=i64(nnz), val=np.zeros(nnz), c=np.zeros(n), q=np.zeros(n),
                   lb=np.zeros(n), ub=np.zeros(n), rl=np.zeros(m), ru=np.zeros(m), cols=i64(n),
                   rows=i64(m), lower_rows=i64(m), upper_rows=i64(m),
                   fixed=np.zeros(int(model.n)), column_scale=np.zeros(n), row_scale=np.zeros(m),
                   qptr=i64(n + 1), qidx=i64(qnnz), qval=np.zeros(qnnz))
        sc = np.zeros(2)
        P = lambda k: out[k].ctypes.data_as(_I if out[k].dtype == np.int64 else _D)
        check(L.nk_prepared_get(h, P("ptr"), P("idx"), P("val"), P("c"), P("q"), P("lb"), P("ub"),
                                P("rl"), P("ru"), P("cols"), P("rows"), P("lower_rows"),
                                P("upper_rows"), P("fixed"), P("column_scale"), P("row_scale"),
                                sc.ctypes.data_as(_D), P("qptr"), P("qidx"), P("qval")))
        out["objective_scale"], out["offset"] = float(sc[0]), float(sc[1])
        out["m"], out["n"] = m, n
        return out
    finally:
        L.nk_prepared_free(h)


def verify(model, x, y, safe=True) -> dict:
    """Verifier::evaluate(x, y, safe) on the caller's model."""
    L = _bind()
    view = _ModelView(model)
    acc = np.zeros(10)
    xv, yv = _f64(x), _f64(y)
    check(L.nk_verify(C.byref(view.s), xv.ctypes.data_as(_D), yv.ctypes.data_as(_D), int(safe),
                      acc.ctypes.data_as(_D)))
    return dict(zip(ACCURACY_KEYS, acc.tolist()))


def infeasibility_bound(model, y) -> float:
    L = _bind()
    view = _ModelView(model)
    out = C.c_double()
    yv = _f64(y)
    check(L.nk_infeasibility_bound(C.byref(view.s), yv.ctypes.data_as(_D), C.byref(out)))
    return out.value
