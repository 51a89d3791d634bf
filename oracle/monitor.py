"""Test infrastructure only -- FP64 host restatement of the reference's GPU KKT
proxy, the checker of the engine's monitor kernel.

The reference computes it on the device (src/cuda.cu:387-446 and 661-738):

* ``monitor_partial`` / ``monitor_reduce`` (src/cuda.cu:387-446): per column j
  ``g = c_j + q_j x_j + (A^T y)_j + (Q x)_j``; primal violation of the bounds
  relative to ``1 + |x_j|``; dual residual ``|min(x_j - lb_j, max(x_j - ub_j, g))|
  / cscale``; objective ``c_j x_j + q_j x_j^2 / 2 + (Q x)_j x_j / 2``;
  complementarity of g against the active bound.  Per row i the row-interval
  violation relative to ``1 + |rl_i|`` / ``1 + |ru_i|``, and for ``y_i != 0`` the
  complementarity against the endpoint its sign selects, or ``|y_i|`` as a dual
  residual when that endpoint is infinite.  Result ``max(primal, dual,
  complement / (1 + |objective|))``, or +inf when anything is not finite.
* ``monitor_point`` (src/cuda.cu:661-690) evaluates that for one point after
  the SpMVs A x, A^T y, Q x; ``monitor`` (src/cuda.cu:691-738) returns the
  smaller value of the current and the averaged point, with
  ``cscale = max(1, max_j 1 + |c_j|)`` (src/cuda.cu:588,731-733).

Here every product and sum is FP64 numpy except the two sums, which use
``math.fsum`` (exactly rounded), so the device result can be held to it at
1e-12 relative.  Only tests/ import this module.
"""
from __future__ import annotations

import math

import numpy as np


def _csr_matvec(ptr, idx, val, x, rows):
    out = np.zeros(rows)
    if len(idx):
        prod = np.asarray(val, dtype=np.float64) * np.asarray(x, dtype=np.float64)[idx]
        lens = np.diff(ptr)
        nz = lens > 0
        out[nz] = np.add.reduceat(prod, ptr[:-1][nz])
    return out


def _transpose_matvec(ptr, idx, val, y, cols):
    rows = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
    out = np.zeros(cols)
    np.add.at(out, idx, np.asarray(val) * np.asarray(y)[rows])
    return out


def cscale_of(c) -> float:
    """max(1, max_j 1 + |c_j|) (src/cuda.cu:588,731-733)."""
    c = np.asarray(c, dtype=np.float64)
    return max(1.0, float(np.max(1.0 + np.abs(c)))) if c.size else 1.0


def products(model, x, y):
    """A x, A^T y and Q x (None for a model without a sparse Q), FP64."""
    ax = _csr_matvec(model.ptr, model.idx, model.val, x, model.m)
    aty = _transpose_matvec(model.ptr, model.idx, model.val, y, model.n)
    qx = None
    if model.qptr is not None and model.qnnz:
        qx = _csr_matvec(model.qptr, model.qidx, model.qval, x, model.n)
    return ax, aty, qx


def monitor_terms(x, y, ax, aty, qx, c, q, lb, ub, rl, ru, cscale) -> float:
    """monitor_partial + monitor_reduce (src/cuda.cu:387-446) for given products."""
    x, y, ax, aty = (np.asarray(v, dtype=np.float64) for v in (x, y, ax, aty))
    c, q, lb, ub, rl, ru = (np.asarray(v, dtype=np.float64) for v in (c, q, lb, ub, rl, ru))
    qxv = np.zeros_like(x) if qx is None else np.asarray(qx, dtype=np.float64)
    with np.errstate(invalid="ignore", over="ignore"):
        g = c + q * x + aty + qxv
        primal = np.fmax(0.0, np.fmax(lb - x, x - ub)) / (1 + np.abs(x))
        dual = np.abs(np.fmin(x - lb, np.fmax(x - ub, g))) / cscale
        objective = c * x + 0.5 * q * x * x + (0.5 * qxv * x if qx is not None else 0.0)
        comp_x = np.where((g > 0) & np.isfinite(lb), np.abs(g * (x - lb)), 0.0) + \
            np.where((g < 0) & np.isfinite(ub), np.abs(g * (ub - x)), 0.0)
        bad = bool(np.any(~np.isfinite(x) | ~np.isfinite(g) | ~np.isfinite(objective)))
        fl, fu = np.isfinite(rl), np.isfinite(ru)
        p_rows = np.where(fl, np.fmax(0.0, rl - ax) / (1 + np.abs(rl)), 0.0)
        p_rows = np.fmax(p_rows, np.where(fu, np.fmax(0.0, ax - ru) / (1 + np.abs(ru)), 0.0))
        endpoint = np.where(y > 0, ru, rl)
        active = y != 0
        fin = np.isfinite(endpoint)
        comp_y = np.where(active & fin, np.abs(y * (endpoint - ax)), 0.0)
        dual_y = np.where(active & ~fin, np.abs(y), 0.0)
        bad = bad or bool(np.any(~np.isfinite(ax) | ~np.isfinite(y)))
    if bad:
        return math.inf
    p = max(float(np.max(primal, initial=0.0)), float(np.max(p_rows, initial=0.0)))
    d = max(float(np.max(dual, initial=0.0)), float(np.max(dual_y, initial=0.0)))
    o = math.fsum(np.broadcast_to(objective, x.shape).tolist())
    v = math.fsum(comp_x.tolist() + comp_y.tolist())
    return max(p, d, v / (1 + abs(o)))


def monitor_point(model, x, y, cscale=None) -> float:
    """One point of the proxy, with A x, A^T y, Q x computed here (FP64)."""
    ax, aty, qx = products(model, x, y)
    cs = cscale_of(model.c) if cscale is None else cscale
    return monitor_terms(x, y, ax, aty, qx, model.c, model.q, model.lb, model.ub, model.rl,
                         model.ru, cs)


def monitor(model, x, y, xa, ya) -> float:
    """IterationBackend::monitor of the CUDA backend: the smaller proxy of the
    current and the averaged point (src/cuda.cu:736)."""
    return min(monitor_point(model, x, y), monitor_point(model, xa, ya))
