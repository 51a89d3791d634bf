"""Python mirror of the engine's C ABI (include/nk_pdhg.h) over ctypes.

:class:`PdhgBackend` has the member functions of the reference's plugin interface
``IterationBackend`` (src/internal.hpp:102-124) with the same argument meaning
and error behaviour as the reference's ``cuda_backend()`` (src/cuda.cu:1288-1303):
failures raise ``RuntimeError`` with the engine's message, exactly where the
reference throws ``std::runtime_error``.

The shared library is built in-tree (``niryukti_b200/libnkpdhg.so``); importing
this module without it raises immediately -- there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libnkpdhg.so"

PRECISIONS = {"fp64": 0, "mixed": 1, "fp32": 2}
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "MEMORY", 4: "STALLED", 5: "UNSUPPORTED",
                6: "NO_DEVICE"}

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int64)


class NkCsr(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("ptr", _I), ("index", _I),
                ("value", _D)]


class NkOptions(C.Structure):
    _fields_ = [("adaptive", C.c_int), ("halpern", C.c_int), ("reflection", C.c_double),
                ("residual_restarts", C.c_int), ("graphs", C.c_int), ("index_bits", C.c_int),
                ("precision", C.c_int)]


class EngineError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = STATUS_NAMES.get(status, str(status))


_lib = None


def library() -> C.CDLL:
    """Load libnkpdhg.so (once).  Raises if the extension has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m niryukti_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    L.nk_last_error.restype = C.c_char_p
    L.nk_abi_version.restype = C.c_uint
    L.nk_pdhg_create.argtypes = [C.POINTER(NkCsr), C.POINTER(NkCsr), _D, _D, _D, _D, _D, _D, _D,
                                 _D, C.POINTER(NkOptions), C.POINTER(C.c_void_p)]
    L.nk_pdhg_destroy.argtypes = [C.c_void_p]
    L.nk_pdhg_destroy.restype = None
    L.nk_pdhg_advance.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double,
                                  C.POINTER(C.c_int)]
    L.nk_pdhg_rejected_steps.argtypes = [C.c_void_p, _I]
    L.nk_pdhg_restart_requested.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    L.nk_pdhg_monitor.argtypes = [C.c_void_p, _D]
    L.nk_pdhg_candidates.argtypes = [C.c_void_p, _D, _D, _D, _D]
    L.nk_pdhg_reset_candidate.argtypes = [C.c_void_p, C.c_int]
    L.nk_pdhg_reset.argtypes = [C.c_void_p, _D, _D]
    L.nk_pdhg_snapshot_layout.argtypes = [C.c_void_p, C.POINTER(C.c_int), _I]
    L.nk_pdhg_snapshot.argtypes = [C.c_void_p, _D]
    L.nk_pdhg_restore.argtypes = [C.c_void_p, _D, _I, C.c_int]
    L.nk_pdhg_stats.argtypes = [C.c_void_p, _I, _I]
    L.nk_pdhg_profile.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, _D, _D]
    L.nk_pdhg_profile_kernels.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, _D]
    L.nk_pdhg_layout_info.argtypes = [C.c_void_p, _I, _I, C.POINTER(C.c_int), _I,
                                      C.POINTER(C.c_int)]
    L.nk_pdhg_schedule_info.argtypes = [C.c_void_p, C.POINTER(C.c_int), _I, C.POINTER(C.c_int),
                                        _I, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.nk_pdhg_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    L.nk_pdhg_time_spmv.argtypes = [C.c_void_p, C.c_int, C.c_int, _D]
    L.nk_cuda_available.restype = C.c_int
    L.nk_cuda_description.argtypes = [C.c_char_p, C.c_int]
    L.nk_hardware_info.argtypes = [C.POINTER(C.c_int), _D, _D]
    L.nk_compact_csr.argtypes = [C.POINTER(NkCsr), C.c_int64, _I, _I, C.c_int64, _I, _I, _D,
                                 C.c_int64, _I]
    L.nk_propagate_bounds.argtypes = [C.POINTER(NkCsr), C.POINTER(C.c_int), _D, _D, _D, _D,
                                      C.c_int, C.POINTER(C.c_int)]
    L.nk_linear_solve.argtypes = [C.POINTER(NkCsr), _D, C.c_int, C.c_int, C.c_double, _D,
                                  C.POINTER(C.c_int), C.POINTER(C.c_int)]
    _lib = L
    return L


def check(status: int) -> None:
    if status != 0:
        raise EngineError(status, library().nk_last_error().decode())


def _d(a):
    return None if a is None else a.ctypes.data_as(_D)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def cuda_available() -> bool:
    return bool(library().nk_cuda_available())


def cuda_description() -> str:
    buf = C.create_string_buffer(256)
    check(library().nk_cuda_description(buf, 256))
    return buf.value.decode()


def compact_csr(ptr, idx, val, cols, kept_rows, column_map, output_columns):
    """cuda_compact_matrix (src/cuda.cu:978-1032): the CSR of `kept_rows` with
    the columns renumbered by `column_map` (-1 drops a column), on the GPU.
    Returns (ptr, idx, val)."""
    ptr = np.ascontiguousarray(ptr, dtype=np.int64)
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    val = np.ascontiguousarray(val, dtype=np.float64)
    kept = np.ascontiguousarray(kept_rows, dtype=np.int64)
    cmap = np.ascontiguousarray(column_map, dtype=np.int64)
    rows = len(ptr) - 1
    capacity = int(np.sum(ptr[kept + 1] - ptr[kept])) if len(kept) else 0
    out_ptr = np.zeros(len(kept) + 1, dtype=np.int64)
    out_idx = np.zeros(max(1, capacity), dtype=np.int64)
    out_val = np.zeros(max(1, capacity))
    kept_nnz = C.c_int64()
    a = NkCsr(rows, int(cols), ptr.ctypes.data_as(_I), idx.ctypes.data_as(_I), _d(val))
    check(library().nk_compact_csr(C.byref(a), len(kept), kept.ctypes.data_as(_I),
                                   cmap.ctypes.data_as(_I), int(output_columns),
                                   out_ptr.ctypes.data_as(_I), out_idx.ctypes.data_as(_I),
                                   _d(out_val), capacity, C.byref(kept_nnz)))
    k = kept_nnz.value
    return out_ptr, out_idx[:k].copy(), out_val[:k].copy()


def propagate_bounds(model, integer, lb, ub, passes=5):
    """cuda_propagate_integer_bounds (src/cuda.cu:448-529, 1033-1135) on the GPU:
    `passes` rounds of directed-rounding bound proposals.  Returns
    (feasible, lb, ub)."""
    lb = np.array(lb, dtype=np.float64)
    ub = np.array(ub, dtype=np.float64)
    flags = np.ascontiguousarray(np.asarray(integer, dtype=np.int32))
    ptr = np.ascontiguousarray(model.ptr, dtype=np.int64)
    idx = np.ascontiguousarray(model.idx, dtype=np.int64)
    val = np.ascontiguousarray(model.val, dtype=np.float64)
    rl = np.ascontiguousarray(model.rl, dtype=np.float64)
    ru = np.ascontiguousarray(model.ru, dtype=np.float64)
    a = NkCsr(int(model.m), int(model.n), ptr.ctypes.data_as(_I), idx.ctypes.data_as(_I),
              _d(val))
    ok = C.c_int()
    check(library().nk_propagate_bounds(C.byref(a), flags.ctypes.data_as(C.POINTER(C.c_int)),
                                        _d(rl), _d(ru), _d(lb), _d(ub), int(passes),
                                        C.byref(ok)))
    return bool(ok.value), lb, ub


def linear_solve(ptr, idx, val, rhs, fp32_matrix=False, precondition=True, time_limit=60.0):
    """cuda_linear_solve (src/cuda.cu:1328-1434): BiCGSTAB for K x = rhs on the
    GPU (diagonally right-preconditioned unless precondition=False, which runs
    the reference's iteration exactly).  Returns (x, converged)."""
    ptr = np.ascontiguousarray(ptr, dtype=np.int64)
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    val = np.ascontiguousarray(val, dtype=np.float64)
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    n = len(ptr) - 1
    x = np.zeros(n)
    ok, late = C.c_int(), C.c_int()
    a = NkCsr(n, n, ptr.ctypes.data_as(_I), idx.ctypes.data_as(_I), _d(val))
    check(library().nk_linear_solve(C.byref(a), _d(rhs), int(bool(fp32_matrix)),
                                    int(bool(precondition)), float(time_limit), _d(x),
                                    C.byref(ok), C.byref(late)))
    if late.value:
        raise TimeoutError("GPU Newton solve time-limited")
    return x, bool(ok.value)


def hardware_info() -> dict:
    a = C.c_int()
    f = C.c_double()
    t = C.c_double()
    check(library().nk_hardware_info(C.byref(a), C.byref(f), C.byref(t)))
    return {"gpu_available": bool(a.value), "free_gpu_bytes": f.value,
            "total_gpu_bytes": t.value}


class PdhgBackend:
    """cuda_backend(model, x, y, adaptive, halpern, reflection, residual_restarts,
    graphs, indices, precision) -- src/internal.hpp:129-134."""

    def __init__(self, model, x=None, y=None, adaptive=False, halpern=False, reflection=0.0,
                 residual_restarts=False, graphs=False, indices="auto", precision="fp64"):
        L = library()
        self._L = L
        self.n, self.m = int(model.n), int(model.m)
        self._keep = []

        def csr(rows, cols, ptr, idx, val):
            p, i, v = _i64(ptr), _i64(idx), _f64(val)
            self._keep += [p, i, v]
            return NkCsr(rows, cols, p.ctypes.data_as(_I), i.ctypes.data_as(_I), _d(v))

        A = csr(self.m, self.n, model.ptr, model.idx, model.val)
        Q = None
        if getattr(model, "qptr", None) is not None and int(model.qptr[-1]) > 0:
            Q = csr(self.n, self.n, model.qptr, model.qidx, model.qval)
        vecs = [_f64(v) for v in (model.c, model.q, model.lb, model.ub, model.rl, model.ru)]
        x0 = _f64(np.zeros(self.n) if x is None else x)
        y0 = _f64(np.zeros(self.m) if y is None else y)
        self._keep += vecs + [x0, y0]
        bits = {"auto": 0, "32": 32, "64": 64}[str(indices)]
        opts = NkOptions(int(adaptive), int(halpern), float(reflection), int(residual_restarts),
                         int(graphs), bits, PRECISIONS[precision])
        h = C.c_void_p()
        check(L.nk_pdhg_create(C.byref(A), C.byref(Q) if Q is not None else None,
                               *[_d(v) for v in vecs], _d(x0), _d(y0), C.byref(opts),
                               C.byref(h)))
        self._h = h
        self._keep = []  # the engine copied everything

    def close(self):
        if getattr(self, "_h", None):
            self._L.nk_pdhg_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def advance(self, count: int, tau: float, sigma: float) -> int:
        acc = C.c_int()
        check(self._L.nk_pdhg_advance(self._h, int(count), float(tau), float(sigma),
                                      C.byref(acc)))
        return acc.value

    def rejected_steps(self) -> int:
        v = C.c_int64()
        check(self._L.nk_pdhg_rejected_steps(self._h, C.byref(v)))
        return v.value

    def restart_requested(self) -> bool:
        v = C.c_int()
        check(self._L.nk_pdhg_restart_requested(self._h, C.byref(v)))
        return bool(v.value)

    def monitor(self) -> float:
        v = C.c_double()
        check(self._L.nk_pdhg_monitor(self._h, C.byref(v)))
        return v.value

    def candidates(self, out=None):
        """(x, y, x_avg, y_avg) in the caller's order; rebases A x.  ``out``
        (optional): four preallocated C-contiguous float64 arrays of n, m, n
        and m entries to fill, e.g. views of pinned host memory."""
        if out is None:
            out = (np.empty(self.n), np.empty(self.m), np.empty(self.n), np.empty(self.m))
        else:
            for a, k in zip(out, (self.n, self.m, self.n, self.m)):
                if a.dtype != np.float64 or a.shape != (k,) or not a.flags.c_contiguous:
                    raise ValueError("candidates(out=...) needs C-contiguous float64 arrays "
                                     "of n, m, n and m entries")
        x, y, xa, ya = out
        check(self._L.nk_pdhg_candidates(self._h, _d(x), _d(y), _d(xa), _d(ya)))
        return x, y, xa, ya

    def reset_candidate(self, average: bool) -> bool:
        check(self._L.nk_pdhg_reset_candidate(self._h, int(bool(average))))
        return True

    def reset(self, x, y) -> None:
        x, y = _f64(x), _f64(y)
        check(self._L.nk_pdhg_reset(self._h, _d(x), _d(y)))

    def snapshot(self):
        parts = C.c_int()
        sizes = np.zeros(16, dtype=np.int64)
        check(self._L.nk_pdhg_snapshot_layout(self._h, C.byref(parts), sizes.ctypes.data_as(_I)))
        sizes = sizes[: parts.value]
        flat = np.empty(int(sizes.sum()))
        check(self._L.nk_pdhg_snapshot(self._h, _d(flat)))
        return np.split(flat, np.cumsum(sizes)[:-1])

    def restore(self, parts) -> None:
        sizes = np.array([len(p) for p in parts], dtype=np.int64)
        flat = _f64(np.concatenate([np.asarray(p, dtype=np.float64) for p in parts]))
        check(self._L.nk_pdhg_restore(self._h, _d(flat), sizes.ctypes.data_as(_I), len(parts)))

    def profile(self, count: int, tau: float, sigma: float):
        """Mean (primal_ms, dual_ms) kernel durations over `count` single trials."""
        a = C.c_double()
        b = C.c_double()
        check(self._L.nk_pdhg_profile(self._h, int(count), float(tau), float(sigma),
                                      C.byref(a), C.byref(b)))
        return a.value, b.value

    def profile_kernels(self, count: int, tau: float, sigma: float):
        """Mean (primal, panel, dual) kernel durations in ms over `count` single
        trials (panel 0 when A's long rows are not stored by column panel)."""
        ms = np.zeros(3)
        check(self._L.nk_pdhg_profile_kernels(self._h, int(count), float(tau), float(sigma),
                                              _d(ms)))
        return tuple(float(v) for v in ms)

    def layout_info(self):
        """The dual SpMV's layout: long rows stored by column panel, the panel
        width, the panel count, the runs (partial sums) of the long rows and the
        kernel launches per trial."""
        r, w, n = C.c_int64(), C.c_int64(), C.c_int64()
        p, k = C.c_int(), C.c_int()
        check(self._L.nk_pdhg_layout_info(self._h, C.byref(r), C.byref(w), C.byref(p),
                                          C.byref(n), C.byref(k)))
        return {"panel_rows": r.value, "panel_width": w.value, "panels": p.value,
                "panel_runs": n.value, "kernels_per_trial": k.value}

    def time_spmv(self, which: str, reps: int = 20) -> float:
        """Mean ms of a plain SpMV with A ("A") or A^T ("At") on the resident iterate."""
        v = C.c_double()
        check(self._L.nk_pdhg_time_spmv(self._h, {"A": 0, "At": 1}[which], int(reps),
                                        C.byref(v)))
        return v.value

    def stream(self) -> int:
        """Raw cudaStream_t of this handle (for CUDA-event timing)."""
        v = C.c_void_p()
        check(self._L.nk_pdhg_stream(self._h, C.byref(v)))
        return int(v.value or 0)

    def schedule_info(self):
        aw, atw, ai, ati = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        al, atl = C.c_int64(), C.c_int64()
        check(self._L.nk_pdhg_schedule_info(self._h, C.byref(aw), C.byref(al), C.byref(atw),
                                            C.byref(atl), C.byref(ai), C.byref(ati)))
        return {"A": {"width": aw.value, "long_threshold": al.value, "items": ai.value},
                "At": {"width": atw.value, "long_threshold": atl.value, "items": ati.value}}

    def stats(self):
        t = C.c_int64()
        b = C.c_int64()
        check(self._L.nk_pdhg_stats(self._h, C.byref(t), C.byref(b)))
        return {"trials": t.value, "device_bytes": b.value}
