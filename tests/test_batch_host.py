"""The batch family's host-only entries on the CPU.

nk_batch_prepare / nk_batch_prepare_from do everything a solve does before its
first iteration (presolve, scaling, start point, the instance's layout) without
touching a device, so a server can prepare requests on many threads while the
GPU runs.  nk_batch_estimate is the reference's device-memory guard
(src/cuda.cu:1294-1295).  An instance that is decided before its first
iteration needs no device memory at all."""
import concurrent.futures as cf
import ctypes as C

import numpy as np
import pytest

from niryukti_b200 import batch, engine, synth
from niryukti_b200.solver import _ModelView
from tests.test_oracle import sparse_qp_model

_D = C.POINTER(C.c_double)


def _lib():
    L = batch._bind()
    L.nk_batch_prepare_from.argtypes = [C.POINTER(batch.NkModel), C.POINTER(batch.NkBatchOptions),
                                        _D, _D, C.POINTER(C.c_void_p), _D]
    return L


def _prepare(model, x0=None, y0=None, **options):
    """The device bytes of one prepared instance (the item is freed after)."""
    L = _lib()
    view = _ModelView(model)
    opts = batch.batch_options(**options)
    h, b = C.c_void_p(), C.c_double(-1.0)
    if x0 is None and y0 is None:
        st = L.nk_batch_prepare(C.byref(view.s), C.byref(opts), C.byref(h), C.byref(b))
    else:
        xs = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
        ys = None if y0 is None else np.ascontiguousarray(y0, dtype=np.float64)
        st = L.nk_batch_prepare_from(C.byref(view.s), C.byref(opts),
                                     None if xs is None else xs.ctypes.data_as(_D),
                                     None if ys is None else ys.ctypes.data_as(_D),
                                     C.byref(h), C.byref(b))
    engine.check(st)
    assert h.value
    L.nk_batch_item_free(h)
    return b.value


def test_estimate_is_the_reference_guard():
    """48 B per nonzero of A and Q plus 240 B per row and column, plus two
    (src/cuda.cu:1294-1295)."""
    lp = synth.random_lp(m=200, n=500, per_col=3, seed=4)
    assert batch.estimate_bytes(lp) == 48 * lp.nnz + 240 * (lp.m + lp.n + 2)
    qp = sparse_qp_model()
    assert qp.qnnz > 0
    assert batch.estimate_bytes(qp) == 48 * (qp.nnz + qp.qnnz) + 240 * (qp.m + qp.n + 2)


def test_prepare_runs_without_a_device():
    lp = synth.random_lp(m=200, n=500, per_col=3, seed=4)
    bytes_lp = _prepare(lp)
    assert 0 < bytes_lp < batch.estimate_bytes(lp)
    assert _prepare(sparse_qp_model()) > 0


def test_prepare_is_thread_safe():
    """Concurrent preparations (the server's prepare workers) give the same
    footprints as serial ones."""
    models = [synth.random_lp(m=150 + 10 * k, n=400, per_col=3, seed=k) for k in range(8)]
    serial = [_prepare(m) for m in models]
    with cf.ThreadPoolExecutor(max_workers=8) as pool:
        parallel = list(pool.map(_prepare, models))
    assert parallel == serial


def test_decided_instances_need_no_device_memory(reference):
    # an empty row that must equal 1: infeasible at presolve
    lp = synth.random_lp(m=50, n=120, per_col=2, seed=7)
    ptr = np.concatenate([lp.ptr, lp.ptr[-1:]])
    bad = synth.Model(**{**lp.__dict__, "m": lp.m + 1, "ptr": ptr,
                         "rl": np.append(lp.rl, 1.0), "ru": np.append(lp.ru, 1.0)})
    assert _prepare(bad) == 0.0
    # a zero time limit: decided before the first iteration
    assert _prepare(lp, time_limit=0.0) == 0.0
    # started at a certified optimum (the reference's own CPU solve): nothing to iterate
    model = sparse_qp_model()
    r = reference.model(model).solve(tol=1e-9)
    assert r["status"] == "OPTIMAL"
    assert _prepare(model, x0=r["x"], y0=r["y"]) == 0.0
    assert _prepare(model) > 0  # from zero it must iterate


def test_invalid_options_are_refused():
    lp = synth.random_lp(m=40, n=80, per_col=2, seed=1)
    with pytest.raises(engine.EngineError, match="invalid batch options") as e:
        _prepare(lp, tol=0.0)
    assert e.value.status == "INVALID"
    with pytest.raises(engine.EngineError, match="invalid batch options"):
        _prepare(lp, check_every=0)
    with pytest.raises(ValueError, match="fp64 or mixed"):
        batch.batch_options(matrix_precision="fp32")


def test_precision_defaults():
    """The batch's C default and its Python default are FP64 matrices; the
    served stream's default is MIXED (each chosen by certified solves per
    second on its own workload)."""
    import inspect
    from niryukti_b200 import serve
    L = _lib()
    o = batch.NkBatchOptions()
    L.nk_batch_defaults(C.byref(o))
    assert o.precision == batch.PRECISIONS["fp64"]
    assert batch.batch_options().precision == batch.PRECISIONS["fp64"]
    sig = inspect.signature(serve.SolveService.__init__)
    assert sig.parameters["matrix_precision"].default == "mixed"
