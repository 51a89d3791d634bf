"""Binary model files: a continuous LP/QP stored as its raw arrays.

The reference ingests models only as text -- its native JSON format, MPS, LP
and QPLIB (read_model, src/io.cpp:800-814) -- and its Python session hands a
model to the library through a temporary JSON file
(python/vantage/native.py:26-31).  For an instance with tens of millions of
nonzeros that parse dominates the time to the first iteration.  A model file
holds the same continuous model (A, Q, c, q, lb, ub, rl, ru, offset) in the
engine's host layout, so loading is a memory map plus checks, and the arrays
reach nk_solve without a copy.

The format, the writer and the checks live in the native library
(nk_model_write, nk_model_view; layout at the top of csrc/nk_modelfile.cpp),
so C, cgo and Python callers share one implementation.  Here `load` maps the
file with numpy and lets the library check the image; the returned model's
arrays are read-only views of the mapping and keep it alive.

    python -m niryukti_b200.modelfile convert model.json model.nkm
    python -m niryukti_b200.modelfile info model.nkm
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import sys
import time

import numpy as np

from . import engine, solver, synth

_bound = False


def _lib() -> C.CDLL:
    global _bound
    L = engine.library()
    if not _bound:
        L.nk_model_write.argtypes = [C.c_char_p, C.POINTER(solver.NkModel), C.c_int]
        L.nk_model_view.argtypes = [C.c_void_p, C.c_int64, C.POINTER(solver.NkModel),
                                    C.POINTER(C.c_int)]
        _bound = True
    return L


def save(model, path) -> None:
    """Write `model` (a synth.Model or anything with its fields) to `path`.  A
    model with sense -1 (a maximisation held in minimisation form, as
    serve.model_from_json builds it) is recorded as such."""
    view = solver._ModelView(model)
    maximise = int(getattr(model, "sense", 1.0) < 0)
    engine.check(_lib().nk_model_write(os.fsencode(path), C.byref(view.s), maximise))


def load(path) -> synth.Model:
    """Map the model file at `path` and return its model; the arrays are
    read-only views of the mapping and `sense` is -1.0 for a recorded
    maximisation (else 1.0).  The arrays hold the minimisation form, so, as in
    the reference's Result, solver.solve reports that form's objective;
    multiply by `sense` for the source objective (serve.result_json does, like
    the reference's result JSON, src/io.cpp:920).  A corrupt, truncated or
    foreign file raises engine.EngineError (status INVALID) naming the failed
    check."""
    path = pathlib.Path(path)
    if path.stat().st_size == 0:
        image = np.zeros(1, dtype=np.uint64)  # let the library report the short file
        engine.check(_lib().nk_model_view(image.ctypes.data, 0, C.byref(solver.NkModel()), None))
    image = np.memmap(path, dtype=np.uint8, mode="r")
    v, maximise = solver.NkModel(), C.c_int(0)
    engine.check(_lib().nk_model_view(image.ctypes.data, image.size, C.byref(v),
                                      C.byref(maximise)))
    base = image.ctypes.data

    def part(pointer, count, dtype):
        start = C.cast(pointer, C.c_void_p).value - base
        return np.asarray(image[start:start + 8 * count]).view(dtype)

    m, n = int(v.A.rows), int(v.A.cols)
    ptr = part(v.A.ptr, m + 1, np.int64)
    nnz = int(ptr[-1])
    q = (None, None, None)
    if v.Q.rows > 0:
        qptr = part(v.Q.ptr, n + 1, np.int64)
        qnnz = int(qptr[-1])
        q = (qptr, part(v.Q.index, qnnz, np.int64), part(v.Q.value, qnnz, np.float64))
    model = synth.Model(
        m=m, n=n, ptr=ptr, idx=part(v.A.index, nnz, np.int64),
        val=part(v.A.value, nnz, np.float64), c=part(v.c, n, np.float64),
        q=part(v.q, n, np.float64), lb=part(v.lb, n, np.float64), ub=part(v.ub, n, np.float64),
        rl=part(v.rl, m, np.float64), ru=part(v.ru, m, np.float64), qptr=q[0], qidx=q[1],
        qval=q[2], offset=float(v.offset), name=path.stem)
    model.sense = -1.0 if maximise.value else 1.0
    return model


def _main(argv) -> int:
    usage = ("usage: python -m niryukti_b200.modelfile convert IN.json OUT.nkm\n"
             "       python -m niryukti_b200.modelfile info FILE.nkm")
    if len(argv) == 3 and argv[0] == "convert":
        import json
        from . import serve
        with open(argv[1]) as f:
            model = serve.model_from_json(json.load(f))
        save(model, argv[2])
        print(f"{argv[2]}: {model.m} rows, {model.n} columns, {model.nnz} nonzeros")
        return 0
    if len(argv) == 2 and argv[0] == "info":
        t = time.perf_counter()
        model = load(argv[1])
        dt = time.perf_counter() - t
        print(f"{argv[1]}: {model.m} rows, {model.n} columns, {model.nnz} nonzeros in A, "
              f"{model.qnnz} in Q; mapped and checked in {dt * 1e3:.1f} ms")
        return 0
    print(usage, file=sys.stderr)
    return 2


if __name__ == "__main__":
    sys.exit(_main(sys.argv[1:]))
