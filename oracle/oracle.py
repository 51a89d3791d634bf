"""Test infrastructure only -- ctypes access to the two oracles.

* :class:`Oracle` wraps ``oracle/liboracle.so``, the plain-C restatement of the
  reference's CPU PDHG path (``pdhg_oracle.c``).
* :class:`Reference` wraps ``oracle/_ref/libvantage_ref.so``: the reference's own
  sources compiled by ``oracle/Makefile`` plus ``ref_harness.cpp``.  It exists
  only where the reference sources were available at build time (the build
  container), or where that build was copied along with the repository.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this
module; the engine package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libvantage_ref.so"
BRIDGE_SO = HERE / "_ref" / "libvantage_nk.so"
REF_CUDA_SO = HERE / "_ref" / "libvantage_cuda.so"  # the reference's own CUDA build

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int64)

STATUS = {0: "OPTIMAL", 1: "ITERATION_LIMIT", 2: "TIME_LIMIT", 3: "NUMERICAL_ERROR"}
ACC_KEYS = ("objective", "primal", "dual", "gap", "kkt", "primal_absolute", "dual_absolute",
            "complementarity", "lower_bound", "finite")


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_D)


def _i(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int64).ctypes.data_as(_I)


def build_oracle() -> pathlib.Path:
    """Compile liboracle.so with gcc if it is missing or stale."""
    src = HERE / "pdhg_oracle.c"
    if not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < src.stat().st_mtime:
        subprocess.check_call(["make", "-s", "-C", str(HERE), "oracle"])
    return ORACLE_SO


class _Arrays:
    """Keeps numpy arrays alive while C holds raw pointers to them."""

    def __init__(self, model):
        self.ptr = np.ascontiguousarray(model.ptr, dtype=np.int64)
        self.idx = np.ascontiguousarray(model.idx, dtype=np.int64)
        self.val = np.ascontiguousarray(model.val, dtype=np.float64)
        self.vecs = [np.ascontiguousarray(v, dtype=np.float64)
                     for v in (model.c, model.q, model.lb, model.ub, model.rl, model.ru)]
        if model.qptr is not None and model.qnnz > 0:
            self.q = (np.ascontiguousarray(model.qptr, dtype=np.int64),
                      np.ascontiguousarray(model.qidx, dtype=np.int64),
                      np.ascontiguousarray(model.qval, dtype=np.float64))
        else:
            self.q = (None, None, None)


class Oracle:
    """The C restatement (pdhg_oracle.c)."""

    def __init__(self, path=None):
        self.lib = C.CDLL(str(path or build_oracle()))
        L = self.lib
        L.orc_last_error.restype = C.c_char_p
        L.orc_model_new.restype = C.c_void_p
        L.orc_model_new.argtypes = [C.c_int64, C.c_int64, _I, _I, _D, _D, _D, _D, _D, _D, _D,
                                    _I, _I, _D, C.c_double]
        L.orc_model_free.argtypes = [C.c_void_p]
        L.orc_quadratic_norm_bound.argtypes = [C.c_void_p]
        L.orc_quadratic_norm_bound.restype = C.c_double
        L.orc_transpose.argtypes = [C.c_int64, C.c_int64, _I, _I, _D, _I, _I, _D]
        L.orc_spmv.argtypes = [C.c_int64, _I, _I, _D, _D, _D]
        L.orc_backend_new.restype = C.c_void_p
        L.orc_backend_new.argtypes = [C.c_void_p, _D, _D, C.c_int, C.c_int, C.c_double, C.c_int]
        L.orc_backend_free.argtypes = [C.c_void_p]
        L.orc_backend_advance.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.orc_backend_rejected.argtypes = [C.c_void_p]
        L.orc_backend_rejected.restype = C.c_int64
        L.orc_backend_restart_requested.argtypes = [C.c_void_p]
        L.orc_backend_candidates.argtypes = [C.c_void_p, _D, _D, _D, _D]
        L.orc_backend_reset.argtypes = [C.c_void_p, _D, _D]
        L.orc_backend_snapshot.argtypes = [C.c_void_p, _D]
        L.orc_backend_snapshot.restype = C.c_int64
        L.orc_verify.argtypes = [C.c_void_p, _D, _D, C.c_int, _D]
        L.orc_infeasibility_bound.argtypes = [C.c_void_p, _D]
        L.orc_infeasibility_bound.restype = C.c_double
        L.orc_scale.restype = C.c_void_p
        L.orc_scale.argtypes = [C.c_void_p, C.c_int, _D, _D, _D]
        L.orc_propagate_bounds.argtypes = [C.c_int64, C.c_int64, _I, _I, _D,
                                           C.POINTER(C.c_int), _D, _D, _D, _D, C.c_int]
        L.orc_model_get.argtypes = [C.c_void_p, _I, _I, _D, _D, _D, _D, _D, _D, _D, _D]
        L.orc_solve.argtypes = [C.c_void_p, C.c_double, C.c_int64, C.c_double, C.c_int, C.c_int,
                                C.c_int, C.c_int, _D, _D, _D]

    def propagate_bounds(self, model, integer, lb, ub, passes=5):
        """Directed-rounding bound proposals (cuda_propagate_integer_bounds,
        src/cuda.cu:448-529); returns (feasible, lb, ub)."""
        lb = np.array(lb, dtype=np.float64)
        ub = np.array(ub, dtype=np.float64)
        flags = np.ascontiguousarray(np.asarray(integer, dtype=np.int32))
        ptr = np.ascontiguousarray(model.ptr, dtype=np.int64)
        idx = np.ascontiguousarray(model.idx, dtype=np.int64)
        val = np.ascontiguousarray(model.val, dtype=np.float64)
        rl = np.ascontiguousarray(model.rl, dtype=np.float64)
        ru = np.ascontiguousarray(model.ru, dtype=np.float64)
        ok = self.lib.orc_propagate_bounds(model.m, model.n, _i(ptr), _i(idx), _d(val),
                                           flags.ctypes.data_as(C.POINTER(C.c_int)),
                                           _d(rl), _d(ru), _d(lb), _d(ub), passes)
        return bool(ok), lb, ub

    def error(self):
        return self.lib.orc_last_error().decode()

    def model(self, model):
        return OracleModel(self, model)

    def transpose(self, ptr, idx, val, rows, cols):
        nnz = int(ptr[rows])
        tptr = np.zeros(cols + 1, dtype=np.int64)
        tidx = np.zeros(nnz, dtype=np.int64)
        tval = np.zeros(nnz)
        self.lib.orc_transpose(rows, cols, _i(ptr), _i(idx), _d(val), _i(tptr), _i(tidx),
                               _d(tval))
        return tptr, tidx, tval

    def spmv(self, ptr, idx, val, x, rows):
        y = np.zeros(rows)
        self.lib.orc_spmv(rows, _i(ptr), _i(idx), _d(val), _d(x), _d(y))
        return y


class OracleModel:
    def __init__(self, orc: Oracle, model):
        self.o = orc
        self.src = model
        self.m, self.n = model.m, model.n
        a = self._arrays = _Arrays(model)
        self.h = orc.lib.orc_model_new(model.m, model.n, _i(a.ptr), _i(a.idx), _d(a.val),
                                       *[_d(v) for v in a.vecs], _i(a.q[0]), _i(a.q[1]),
                                       _d(a.q[2]), float(model.offset))

    def __del__(self):
        if getattr(self, "h", None):
            self.o.lib.orc_model_free(self.h)
            self.h = None

    def verify(self, x, y, safe=True):
        acc = np.zeros(10)
        self.o.lib.orc_verify(self.h, _d(x), _d(y), int(safe), _d(acc))
        return dict(zip(ACC_KEYS, acc.tolist()))

    def infeasibility_bound(self, y):
        return self.o.lib.orc_infeasibility_bound(self.h, _d(y))

    def quadratic_norm_bound(self):
        return self.o.lib.orc_quadratic_norm_bound(self.h)

    def backend(self, x, y, adaptive=False, halpern=False, reflection=0.0, restarts=False):
        return OracleBackend(self, x, y, adaptive, halpern, reflection, restarts)

    def scale(self, passes=5):
        cs = np.zeros(self.n)
        rs = np.zeros(self.m)
        os_ = np.zeros(1)
        h = self.o.lib.orc_scale(self.h, passes, _d(cs), _d(rs), _d(os_))
        if not h:
            raise RuntimeError(self.o.error())
        nnz = self.src.nnz
        out = dict(ptr=np.zeros(self.m + 1, dtype=np.int64), idx=np.zeros(nnz, dtype=np.int64),
                   val=np.zeros(nnz), c=np.zeros(self.n), q=np.zeros(self.n),
                   lb=np.zeros(self.n), ub=np.zeros(self.n), rl=np.zeros(self.m),
                   ru=np.zeros(self.m))
        off = np.zeros(1)
        self.o.lib.orc_model_get(h, _i(out["ptr"]), _i(out["idx"]), _d(out["val"]),
                                 _d(out["c"]), _d(out["q"]), _d(out["lb"]), _d(out["ub"]),
                                 _d(out["rl"]), _d(out["ru"]), _d(off))
        self.o.lib.orc_model_free(h)
        out.update(column_scale=cs, row_scale=rs, objective_scale=float(os_[0]),
                   offset=float(off[0]))
        return out

    def solve(self, tol=1e-6, iteration_limit=100000, time_limit=60.0, check_every=100,
              scaling_passes=5, adaptive=True, restart=True):
        x = np.zeros(self.n)
        y = np.zeros(self.m)
        st = np.zeros(14)
        rc = self.o.lib.orc_solve(self.h, tol, iteration_limit, time_limit, check_every,
                                  scaling_passes, int(adaptive), int(restart), _d(x), _d(y),
                                  _d(st))
        if rc != 0:
            raise RuntimeError(self.o.error())
        keys = ("objective", "primal", "dual", "gap", "kkt", "finite", "iterations", "restarts",
                "rejected_steps", "weight_updates", "seconds", "iteration_seconds",
                "verification_seconds")
        r = dict(zip(keys, st[:13].tolist()))
        r["status"] = STATUS[int(st[13])]
        r["x"], r["y"] = x, y
        return r


class OracleBackend:
    def __init__(self, om: OracleModel, x, y, adaptive, halpern, reflection, restarts):
        self.om = om
        self.L = om.o.lib
        self.h = self.L.orc_backend_new(om.h, _d(x), _d(y), int(adaptive), int(halpern),
                                        float(reflection), int(restarts))
        if not self.h:
            raise RuntimeError(om.o.error())

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_backend_free(self.h)
            self.h = None

    def advance(self, count, tau, sigma):
        r = self.L.orc_backend_advance(self.h, count, tau, sigma)
        if r < 0:
            raise RuntimeError(self.om.o.error())
        return r

    def rejected_steps(self):
        return self.L.orc_backend_rejected(self.h)

    def restart_requested(self):
        return bool(self.L.orc_backend_restart_requested(self.h))

    def candidates(self):
        x, y = np.zeros(self.om.n), np.zeros(self.om.m)
        xa, ya = np.zeros(self.om.n), np.zeros(self.om.m)
        self.L.orc_backend_candidates(self.h, _d(x), _d(y), _d(xa), _d(ya))
        return x, y, xa, ya

    def reset(self, x, y):
        self.L.orc_backend_reset(self.h, _d(x), _d(y))

    def snapshot(self):
        n = self.L.orc_backend_snapshot(self.h, None)
        out = np.zeros(n)
        self.L.orc_backend_snapshot(self.h, _d(out))
        return out


def _kv(opts: dict) -> bytes:
    parts = []
    for k, v in opts.items():
        if isinstance(v, bool):
            v = "1" if v else "0"
        parts.append(f"{k}={v}")
    return ";".join(parts).encode()


class Reference:
    """The reference's own CPU code (oracle/_ref/libvantage_ref.so) through ref_harness.cpp.
    ``path`` may name the bridged build (libvantage_nk.so), whose cuda_backend() is the
    B200 engine."""

    def __init__(self, path=None):
        path = pathlib.Path(path or REF_SO)
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (oracle/Makefile ref)")
        self.lib = C.CDLL(str(path))
        L = self.lib
        L.ref_last_error.restype = C.c_char_p
        L.ref_model_new.restype = C.c_void_p
        L.ref_model_new.argtypes = [C.c_int64, C.c_int64, _I, _I, _D, _D, _D, _D, _D, _D, _D,
                                    _I, _I, _D, C.c_double]
        L.ref_model_free.argtypes = [C.c_void_p]
        L.ref_model_nnz.argtypes = [C.c_void_p]
        L.ref_model_nnz.restype = C.c_int64
        L.ref_model_csr.argtypes = [C.c_void_p, _I, _I, _D]
        L.ref_model_transpose.argtypes = [C.c_void_p, _I, _I, _D]
        L.ref_model_multiply.argtypes = [C.c_void_p, _D, _D]
        L.ref_model_quadratic_norm_bound.argtypes = [C.c_void_p]
        L.ref_model_quadratic_norm_bound.restype = C.c_double
        L.ref_solve.argtypes = [C.c_void_p, C.c_char_p, _D, _D, _D, C.c_char_p, C.c_int]
        L.ref_verify.argtypes = [C.c_void_p, _D, _D, C.c_int, _D]
        L.ref_infeasibility_bound.argtypes = [C.c_void_p, _D]
        L.ref_infeasibility_bound.restype = C.c_double
        L.ref_backend_new.restype = C.c_void_p
        L.ref_backend_new.argtypes = [C.c_void_p, C.c_int, _D, _D, C.c_int, C.c_int, C.c_double,
                                      C.c_int, C.c_int, C.c_char_p, C.c_char_p]
        L.ref_backend_free.argtypes = [C.c_void_p]
        L.ref_backend_advance.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.ref_backend_rejected.argtypes = [C.c_void_p]
        L.ref_backend_rejected.restype = C.c_int64
        L.ref_backend_restart_requested.argtypes = [C.c_void_p]
        L.ref_backend_monitor.argtypes = [C.c_void_p]
        L.ref_backend_monitor.restype = C.c_double
        L.ref_backend_candidates.argtypes = [C.c_void_p, _D, _D, _D, _D]
        L.ref_backend_reset.argtypes = [C.c_void_p, _D, _D]
        L.ref_backend_reset_candidate.argtypes = [C.c_void_p, C.c_int]
        L.ref_backend_snapshot.argtypes = [C.c_void_p, _D, _I, C.c_int]
        L.ref_backend_snapshot.restype = C.c_int64
        L.ref_prepare.restype = C.c_void_p
        L.ref_prepare.argtypes = [C.c_void_p, C.c_char_p]
        L.ref_prepared_free.argtypes = [C.c_void_p]
        L.ref_prepared_dims.argtypes = [C.c_void_p, _I]
        L.ref_prepared_failure.argtypes = [C.c_void_p]
        L.ref_prepared_failure.restype = C.c_char_p
        L.ref_prepared_get.argtypes = [C.c_void_p, _I, _I, _D, _D, _D, _D, _D, _D, _D, _I, _I,
                                       _I, _I, _D, _D, _D, _D, _I, _I, _D]
        L.ref_cuda_available.restype = C.c_int
        L.ref_batch_relaxations.argtypes = [C.c_void_p, C.c_int, _D, _D, _D, _D, C.c_char_p, _D,
                                            C.POINTER(C.c_int), _D, _D]
        L.ref_linear_solve.argtypes = [C.c_int64, _I, _I, _D, _D, C.c_int, C.c_double, _D]
        if hasattr(L, "ref_model_read"):  # absent from builds older than the reader
            L.ref_model_read.restype = C.c_void_p
            L.ref_model_read.argtypes = [C.c_char_p]
            L.ref_model_dims.argtypes = [C.c_void_p, _I]
            L.ref_model_arrays.argtypes = [C.c_void_p, _D, _D, _D, _D, _D, _D, _D, _I, _I, _D]

    def read_model(self, path):
        """The model the reference's read_model (src/io.cpp:800-814) builds from
        a JSON, MPS, LP or QPLIB file, as a synth.Model of its continuous arrays
        (canonical CSR of A and Q, c, q, bounds, offset)."""
        from niryukti_b200 import synth
        if not hasattr(self.lib, "ref_model_read"):
            raise RuntimeError("this reference build predates ref_model_read; rebuild "
                               "(make -C oracle ref bridge)")
        h = self.lib.ref_model_read(str(path).encode())
        if not h:
            raise RuntimeError(self.error())
        try:
            dims = np.zeros(5, dtype=np.int64)
            self.lib.ref_model_dims(h, _i(dims))
            m, n, nnz, qnnz, integer = (int(v) for v in dims)
            if integer:
                raise ValueError(f"{integer} integer columns: not a continuous model")
            ptr = np.zeros(m + 1, dtype=np.int64)
            idx = np.zeros(nnz, dtype=np.int64)
            val = np.zeros(nnz)
            self.lib.ref_model_csr(h, _i(ptr), _i(idx), _d(val))
            vec = {k: np.zeros(n) for k in ("c", "q", "lb", "ub")}
            vec.update({k: np.zeros(m) for k in ("rl", "ru")})
            offset = np.zeros(1)
            qptr = np.zeros(n + 1, dtype=np.int64)
            qidx = np.zeros(qnnz, dtype=np.int64)
            qval = np.zeros(qnnz)
            self.lib.ref_model_arrays(h, *(_d(vec[k]) for k in ("c", "q", "lb", "ub", "rl", "ru")),
                                      _d(offset), _i(qptr), _i(qidx), _d(qval))
        finally:
            self.lib.ref_model_free(h)
        q = (qptr, qidx, qval) if qnnz else (None, None, None)
        return synth.Model(m=m, n=n, ptr=ptr, idx=idx, val=val, c=vec["c"], q=vec["q"],
                           lb=vec["lb"], ub=vec["ub"], rl=vec["rl"], ru=vec["ru"], qptr=q[0],
                           qidx=q[1], qval=q[2], offset=float(offset[0]))

    def linear_solve(self, ptr, idx, val, rhs, fp32_matrix=False, tolerance=1e-7):
        """cuda_linear_solve(K, rhs, Options(), fp32_matrix, tolerance)."""
        ptr = np.ascontiguousarray(ptr, dtype=np.int64)
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        val = np.ascontiguousarray(val, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros(len(ptr) - 1)
        if self.lib.ref_linear_solve(len(ptr) - 1, _i(ptr), _i(idx), _d(val), _d(rhs),
                                     int(bool(fp32_matrix)), float(tolerance), _d(x)) != 0:
            raise RuntimeError(self.error())
        return x

    def error(self):
        return self.lib.ref_last_error().decode()

    def model(self, model):
        return RefModel(self, model)

    def cuda_available(self):
        return bool(self.lib.ref_cuda_available())


class RefModel:
    def __init__(self, ref: Reference, model):
        self.r = ref
        self.src = model
        self.m, self.n = model.m, model.n
        a = self._arrays = _Arrays(model)
        self.h = ref.lib.ref_model_new(model.m, model.n, _i(a.ptr), _i(a.idx), _d(a.val),
                                       *[_d(v) for v in a.vecs], _i(a.q[0]), _i(a.q[1]),
                                       _d(a.q[2]), float(model.offset))
        if not self.h:
            raise RuntimeError(ref.error())

    def __del__(self):
        if getattr(self, "h", None):
            self.r.lib.ref_model_free(self.h)
            self.h = None

    def csr(self):
        nnz = self.r.lib.ref_model_nnz(self.h)
        p = np.zeros(self.m + 1, dtype=np.int64)
        i = np.zeros(nnz, dtype=np.int64)
        v = np.zeros(nnz)
        self.r.lib.ref_model_csr(self.h, _i(p), _i(i), _d(v))
        return p, i, v

    def transpose(self):
        nnz = self.r.lib.ref_model_nnz(self.h)
        p = np.zeros(self.n + 1, dtype=np.int64)
        i = np.zeros(nnz, dtype=np.int64)
        v = np.zeros(nnz)
        self.r.lib.ref_model_transpose(self.h, _i(p), _i(i), _d(v))
        return p, i, v

    def multiply(self, x):
        out = np.zeros(self.m)
        self.r.lib.ref_model_multiply(self.h, _d(x), _d(out))
        return out

    def quadratic_norm_bound(self):
        return self.r.lib.ref_model_quadratic_norm_bound(self.h)

    def solve(self, **opts):
        x = np.zeros(self.n)
        y = np.zeros(self.m)
        st = np.zeros(21)
        status = C.create_string_buffer(64)
        rc = self.r.lib.ref_solve(self.h, _kv(opts), _d(x), _d(y), _d(st), status, 64)
        if rc != 0:
            raise RuntimeError(self.r.error())
        keys = ACC_KEYS + ("iterations", "restarts", "rejected_steps", "seconds",
                           "iteration_seconds", "verification_seconds", "preprocess_seconds",
                           "weight_updates", "host_candidate_checks", "removed_columns",
                           "removed_rows")
        r = dict(zip(keys, st.tolist()))
        r["status"] = status.value.decode()
        r["message"] = self.r.error()
        r["x"], r["y"] = x, y
        return r

    def batch_relaxations(self, lower, upper, x0=None, y0=None, **opts):
        """cuda_batch_relaxations(model, lower, upper, options): one result per box."""
        lower = np.ascontiguousarray(lower, dtype=np.float64)
        upper = np.ascontiguousarray(upper, dtype=np.float64)
        boxes = lower.shape[0]
        st = np.zeros(10 * boxes)
        status = (C.c_int * boxes)()
        xs, ys = np.zeros(boxes * self.n), np.zeros(boxes * self.m)
        x0 = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
        y0 = None if y0 is None else np.ascontiguousarray(y0, dtype=np.float64)
        rc = self.r.lib.ref_batch_relaxations(self.h, boxes, _d(lower), _d(upper),
                                               None if x0 is None else _d(x0),
                                               None if y0 is None else _d(y0), _kv(opts),
                                               _d(st), status, _d(xs), _d(ys))
        if rc != 0:
            raise RuntimeError(self.r.error())
        names = ("OPTIMAL", "INTERRUPTED", "TIME_LIMIT", "ITERATION_LIMIT", "OTHER")
        out = []
        for b in range(boxes):
            s = st[10 * b:10 * b + 10]
            out.append({"status": names[status[b]], "objective": s[0], "kkt": s[1],
                        "finite": bool(s[2]), "iterations": int(s[3]), "restarts": int(s[4]),
                        "seconds": s[5], "x": xs[b * self.n:(b + 1) * self.n],
                        "y": ys[b * self.m:(b + 1) * self.m]})
        return out

    def verify(self, x, y, safe=True):
        acc = np.zeros(10)
        if self.r.lib.ref_verify(self.h, _d(x), _d(y), int(safe), _d(acc)) != 0:
            raise RuntimeError(self.r.error())
        return dict(zip(ACC_KEYS, acc.tolist()))

    def infeasibility_bound(self, y):
        return self.r.lib.ref_infeasibility_bound(self.h, _d(y))

    def backend(self, x, y, adaptive=False, halpern=False, reflection=0.0, restarts=False,
                device="cpu", graphs=False, indices="auto", precision="fp64"):
        return RefBackend(self, x, y, adaptive, halpern, reflection, restarts, device, graphs,
                          indices, precision)

    def prepare(self, **opts):
        h = self.r.lib.ref_prepare(self.h, _kv(opts))
        if not h:
            raise RuntimeError(self.r.error())
        try:
            dims = np.zeros(5, dtype=np.int64)
            self.r.lib.ref_prepared_dims(h, _i(dims))
            m, n, nnz, qnnz, failed = (int(v) for v in dims)
            if failed:
                return {"failure": self.r.lib.ref_prepared_failure(h).decode()}
            out = dict(ptr=np.zeros(m + 1, dtype=np.int64), idx=np.zeros(nnz, dtype=np.int64),
                       val=np.zeros(nnz), c=np.zeros(n), q=np.zeros(n), lb=np.zeros(n),
                       ub=np.zeros(n), rl=np.zeros(m), ru=np.zeros(m),
                       cols=np.zeros(n, dtype=np.int64), rows=np.zeros(m, dtype=np.int64),
                       lower_rows=np.zeros(m, dtype=np.int64),
                       upper_rows=np.zeros(m, dtype=np.int64), fixed=np.zeros(self.n),
                       column_scale=np.zeros(n), row_scale=np.zeros(m),
                       qptr=np.zeros(n + 1, dtype=np.int64), qidx=np.zeros(qnnz, dtype=np.int64),
                       qval=np.zeros(qnnz))
            sc = np.zeros(2)
            o = out
            self.r.lib.ref_prepared_get(h, _i(o["ptr"]), _i(o["idx"]), _d(o["val"]), _d(o["c"]),
                                        _d(o["q"]), _d(o["lb"]), _d(o["ub"]), _d(o["rl"]),
                                        _d(o["ru"]), _i(o["cols"]), _i(o["rows"]),
                                        _i(o["lower_rows"]), _i(o["upper_rows"]), _d(o["fixed"]),
                                        _d(o["column_scale"]), _d(o["row_scale"]), _d(sc),
                                        _i(o["qptr"]), _i(o["qidx"]), _d(o["qval"]))
            out["objective_scale"], out["offset"] = float(sc[0]), float(sc[1])
            out["m"], out["n"] = m, n
            return out
        finally:
            self.r.lib.ref_prepared_free(h)


class RefBackend:
    def __init__(self, rm: RefModel, x, y, adaptive, halpern, reflection, restarts, device,
                 graphs, indices, precision):
        self.rm = rm
        self.L = rm.r.lib
        self.h = self.L.ref_backend_new(rm.h, 0 if device == "cpu" else 1, _d(x), _d(y),
                                        int(adaptive), int(halpern), float(reflection),
                                        int(restarts), int(graphs), indices.encode(),
                                        precision.encode())
        if not self.h:
            raise RuntimeError(rm.r.error())

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_backend_free(self.h)
            self.h = None

    def advance(self, count, tau, sigma):
        r = self.L.ref_backend_advance(self.h, count, tau, sigma)
        if r < 0:
            raise RuntimeError(self.rm.r.error())
        return r

    def rejected_steps(self):
        return self.L.ref_backend_rejected(self.h)

    def restart_requested(self):
        return bool(self.L.ref_backend_restart_requested(self.h))

    def monitor(self):
        return self.L.ref_backend_monitor(self.h)

    def candidates(self):
        x, y = np.zeros(self.rm.n), np.zeros(self.rm.m)
        xa, ya = np.zeros(self.rm.n), np.zeros(self.rm.m)
        if self.L.ref_backend_candidates(self.h, _d(x), _d(y), _d(xa), _d(ya)) != 0:
            raise RuntimeError(self.rm.r.error())
        return x, y, xa, ya

    def reset(self, x, y):
        if self.L.ref_backend_reset(self.h, _d(x), _d(y)) != 0:
            raise RuntimeError(self.rm.r.error())

    def reset_candidate(self, average):
        r = self.L.ref_backend_reset_candidate(self.h, int(average))
        if r < 0:
            raise RuntimeError(self.rm.r.error())
        return bool(r)

    def snapshot(self):
        sizes = np.zeros(32, dtype=np.int64)
        n = self.L.ref_backend_snapshot(self.h, None, _i(sizes), 32)
        out = np.zeros(n)
        self.L.ref_backend_snapshot(self.h, _d(out), _i(sizes), 32)
        return out, sizes
