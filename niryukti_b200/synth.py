"""Seeded synthetic LP/QP instances with the shapes of the benchmark configurations.

All randomness comes from ``numpy.random.default_rng(seed)`` (PCG64).  Every
matrix is returned in canonical CSR form -- rows sorted, column indices strictly
increasing inside a row, no explicit zeros -- which is exactly what the
reference's ``Sparse::build`` produces (src/model.cpp:11-38), so handing these
arrays to either engine yields the same model bit for bit.

Bounds and row intervals follow the reference ``Model`` conventions
(include/vantage/vantage.hpp:25-39): ``lb/ub`` per column, ``rl/ru`` per row,
``-inf/+inf`` for a missing side, equality rows have ``rl == ru``.

Generators:
  * :func:`random_lp`     - the small equality LP (2,000 x 5,000 in the benchmark): m equality rows, n columns, a fixed number of
                            nonzeros per column at distinct random rows.
  * :func:`power_law_lp`  - the 20M-nonzero power-law LP: power-law row lengths, log-uniform row factors,
                            half equality / half <= rows, 10% free columns.
  * :func:`block_angular_lp` - the block-angular planning LP: diagonal blocks plus dense-ish linking rows.
  * :func:`batch_instances`  - the uneven LP/QP instance mix of the batch and the served stream: uneven LP/QP mix, n = 2m, 4-8 nnz per column,
                            QPs with Q = D + L L^T (D on the diagonal shorthand ``q``).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

INF = float("inf")


@dataclasses.dataclass
class Model:
    """A continuous LP/QP in the reference's canonical form.

    minimise  c'x + 1/2 sum_j q_j x_j^2 + 1/2 x'Qx + offset
    s.t.      rl <= A x <= ru,  lb <= x <= ub
    """

    m: int
    n: int
    ptr: np.ndarray  # int64[m+1]
    idx: np.ndarray  # int64[nnz]
    val: np.ndarray  # float64[nnz]
    c: np.ndarray
    q: np.ndarray
    lb: np.ndarray
    ub: np.ndarray
    rl: np.ndarray
    ru: np.ndarray
    qptr: Optional[np.ndarray] = None  # symmetric Q in CSR (n x n) or None
    qidx: Optional[np.ndarray] = None
    qval: Optional[np.ndarray] = None
    offset: float = 0.0
    name: str = "model"
    x0: Optional[np.ndarray] = None  # the feasible point the instance was built from

    @property
    def nnz(self) -> int:
        return int(self.ptr[-1])

    @property
    def qnnz(self) -> int:
        return 0 if self.qptr is None else int(self.qptr[-1])

    def is_qp(self) -> bool:
        return self.qnnz > 0 or bool(np.any(self.q != 0))

    def multiply(self, x: np.ndarray) -> np.ndarray:
        """A @ x in FP64 (numpy's segment sums; the summation order is numpy's, so the
        last bits can differ from the reference's row-sequential Sparse::multiply).
        Used only to define instances (b = A x0), never as a parity check."""
        return csr_matvec(self.ptr, self.idx, self.val, x, self.m)


def csr_matvec(ptr, idx, val, x, rows):
    prod = val * x[idx]
    out = np.zeros(rows, dtype=np.float64)
    lens = np.diff(ptr)
    nz = lens > 0
    if prod.size:
        sums = np.add.reduceat(prod, ptr[:-1][nz])
        out[nz] = sums
    return out


def _canonical_csr(rows: np.ndarray, cols: np.ndarray, vals: np.ndarray, m: int):
    """Sort COO entries by (row, col) and build CSR; entries must already be unique."""
    order = np.lexsort((cols, rows))
    rows = rows[order]
    cols = cols[order]
    vals = vals[order]
    keep = vals != 0
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    counts = np.bincount(rows, minlength=m)
    ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    return ptr, cols.astype(np.int64), vals.astype(np.float64)


def _dedupe_pairs(rng, major, minor, minor_range, minor_lo=None):
    """Resample ``minor`` until every (major, minor) pair is unique.

    ``minor_lo`` (optional, per entry) offsets the draw range: minor in
    [minor_lo, minor_lo + minor_range).
    """
    for _ in range(64):
        key = major.astype(np.int64) * (np.int64(1) << 32) + minor.astype(np.int64)
        order = np.argsort(key, kind="stable")
        sk = key[order]
        dup = np.zeros(sk.size, dtype=bool)
        dup[1:] = sk[1:] == sk[:-1]
        if not dup.any():
            return minor
        bad = order[dup]
        draw = rng.integers(0, minor_range if np.isscalar(minor_range) else minor_range[bad],
                            size=bad.size)
        minor[bad] = draw + (0 if minor_lo is None else minor_lo[bad])
    raise RuntimeError("could not make sparse pattern unique")


def _names_free(model: Model) -> Model:
    return model


def random_lp(m: int = 2000, n: int = 5000, per_col: int = 5, seed: int = 1,
              x_hi: float = 10.0) -> Model:
    """The small equality LP: m equality rows, n columns, ``per_col`` nonzeros per column at
    uniformly random distinct rows, values N(0,1); x0 ~ U[0,x_hi]; b = A x0;
    0 <= x <= x_hi; c ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    cols = np.repeat(np.arange(n, dtype=np.int64), per_col)
    rows = np.empty(n * per_col, dtype=np.int64)
    for j in range(0, n, 65536):  # distinct rows per column, chunked for memory
        jj = min(n, j + 65536)
        k = jj - j
        r = np.argsort(rng.random((k, m)), axis=1)[:, :per_col] if m <= 4096 else None
        if r is None:
            r = rng.integers(0, m, size=(k, per_col))
            flat = r.reshape(-1)
            flat[:] = _dedupe_pairs(rng, np.repeat(np.arange(k), per_col), flat, m)
        rows[j * per_col: jj * per_col] = r.reshape(-1)
    vals = rng.standard_normal(n * per_col)
    ptr, idx, val = _canonical_csr(rows, cols, vals, m)
    x0 = rng.uniform(0, x_hi, n)
    c = rng.standard_normal(n)
    b = csr_matvec(ptr, idx, val, x0, m)
    return Model(m=m, n=n, ptr=ptr, idx=idx, val=val, c=c, q=np.zeros(n),
                 lb=np.zeros(n), ub=np.full(n, x_hi), rl=b.copy(), ru=b.copy(),
                 name=f"random_lp_m{m}_n{n}_s{seed}", x0=x0)


def power_law_exponent(mean: float, lo: int, hi: int) -> float:
    """Exponent a of P(L) ~ L^-a on [lo, hi] whose mean equals ``mean`` (bisection)."""
    L = np.arange(lo, hi + 1, dtype=np.float64)

    def mean_of(a):
        w = L ** (-a)
        return float((L * w).sum() / w.sum())

    a0, a1 = 0.5, 4.0
    for _ in range(100):
        am = 0.5 * (a0 + a1)
        if mean_of(am) > mean:
            a0 = am
        else:
            a1 = am
    return 0.5 * (a0 + a1)


def power_law_lp(m: int = 1_000_000, n: int = 2_000_000, nnz: int = 20_000_000,
                 seed: int = 2, len_lo: int = 2, len_hi: int = 5000,
                 free_frac: float = 0.10, x_hi: float = 5.0) -> Model:
    """The power-law LP (1,000,000 x 2,000,000, 20M nonzeros at the defaults).

    Row lengths follow a discrete power law on [len_lo, len_hi] whose exponent is
    chosen so the mean is nnz/m, then adjusted by +-1 on random rows to sum to
    exactly ``nnz``.  Every column appears at least once.  Values are N(0,1)
    times a per-row factor log-uniform on [1e-2, 1e2].  Rows [0, m/2) are
    equalities, the rest are ``<=`` rows with slack U[0,1] at x0 ~ U[0,x_hi].
    10% of the columns are free, the rest boxed [0, x_hi].

    The objective is c ~ N(0,1) on boxed columns.  On free columns c is set to
    -(A^T y0)_j for a sign-feasible y0 (free on equality rows, >= 0 on <= rows),
    so the LP has a finite optimum: with c ~ N(0,1) there as well, about
    0.25^k of the free columns whose k entries all sit in <= rows with one
    coefficient sign make the LP unbounded (tens of such columns at this size).
    """
    rng = np.random.default_rng(seed)
    a = power_law_exponent(nnz / m, len_lo, len_hi)
    L = np.arange(len_lo, len_hi + 1, dtype=np.float64)
    w = L ** (-a)
    lens = rng.choice(np.arange(len_lo, len_hi + 1), size=m, p=w / w.sum()).astype(np.int64)
    diff = int(nnz - lens.sum())
    while diff != 0:
        step = 1 if diff > 0 else -1
        pick = rng.integers(0, m, size=abs(diff))
        ok = (lens[pick] + step >= len_lo) & (lens[pick] + step <= len_hi)
        pick = np.unique(pick[ok])
        pick = pick[: abs(diff)]
        lens[pick] += step
        diff = int(nnz - lens.sum())
    ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(lens, out=ptr[1:])
    rows = np.repeat(np.arange(m, dtype=np.int64), lens)
    cols = np.concatenate([rng.permutation(n), rng.integers(0, n, size=nnz - n)]).astype(np.int64)
    cols = cols[rng.permutation(nnz)]
    cols = _dedupe_pairs(rng, rows, cols, n)
    factor = np.exp(rng.uniform(math.log(1e-2), math.log(1e2), m))
    vals = rng.standard_normal(nnz) * factor[rows]
    ptr, idx, val = _canonical_csr(rows, cols, vals, m)
    del rows, cols, vals
    x0 = rng.uniform(0, x_hi, n)
    ax0 = csr_matvec(ptr, idx, val, x0, m)
    half = m // 2
    rl = np.empty(m)
    ru = np.empty(m)
    rl[:half] = ax0[:half]
    ru[:half] = ax0[:half]
    rl[half:] = -INF
    ru[half:] = ax0[half:] + rng.uniform(0, 1, m - half)
    free = rng.random(n) < free_frac
    lb = np.where(free, -INF, 0.0)
    ub = np.where(free, INF, x_hi)
    c = rng.standard_normal(n)
    # sign-feasible dual point, scaled so A^T y0 is O(1) per column
    y0 = rng.standard_normal(m) / factor / math.sqrt(nnz / n)
    y0[half:] = np.abs(y0[half:])
    aty0 = csr_matvec(*_transpose(ptr, idx, val, m, n), y0, n)
    c[free] = -aty0[free]
    return Model(m=m, n=n, ptr=ptr, idx=idx, val=val, c=c, q=np.zeros(n), lb=lb, ub=ub,
                 rl=rl, ru=ru, name=f"power_law_lp_m{m}_n{n}_nnz{nnz}_s{seed}", x0=x0)


def _transpose(ptr, idx, val, m, n):
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(ptr))
    order = np.lexsort((rows, idx))
    tcols = rows[order]
    tval = val[order]
    counts = np.bincount(idx, minlength=n)
    tptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=tptr[1:])
    return tptr, tcols, tval


def transpose(model_or_ptr, idx=None, val=None, m=None, n=None):
    """Explicit transpose in the order Sparse::transpose produces (src/model.cpp:39-58):
    row j of A^T lists the rows i of A in increasing order."""
    if isinstance(model_or_ptr, Model):
        mm = model_or_ptr
        return _transpose(mm.ptr, mm.idx, mm.val, mm.m, mm.n)
    return _transpose(model_or_ptr, idx, val, m, n)


def block_angular_lp(blocks: int = 64, block_rows: int = 20_000, block_cols: int = 40_000,
                     per_col: int = 6, linking_rows: int = 2000, linking_frac: float = 0.05,
                     seed: int = 3, x_hi: float = 10.0, box_hi: float = 20.0) -> Model:
    """The block-angular planning LP: ``blocks`` diagonal blocks of block_rows x block_cols with
    ``per_col`` nonzeros per column, plus ``linking_rows`` rows each touching
    ``linking_frac`` of all columns.  Values U[0.1,2], negated with probability
    0.3.  Block rows are equalities at x0 ~ U[0,x_hi]; linking rows are <= rows
    with slack U[0,1].  Box [0, box_hi]; c ~ U[-1,1]."""
    rng = np.random.default_rng(seed)
    n = blocks * block_cols
    mb = blocks * block_rows
    m = mb + linking_rows
    # block part: per column, per_col distinct rows inside its block
    cols_b = np.repeat(np.arange(n, dtype=np.int64), per_col)
    blk = cols_b // block_cols
    local = rng.integers(0, block_rows, size=cols_b.size)
    local = _dedupe_pairs(rng, cols_b, local, block_rows)
    rows_b = blk * block_rows + local
    vals_b = rng.uniform(0.1, 2.0, rows_b.size)
    vals_b[rng.random(rows_b.size) < 0.3] *= -1
    ptr_b, idx_b, val_b = _canonical_csr(rows_b, cols_b, vals_b, mb)
    del rows_b, cols_b, vals_b, blk, local
    # linking part: rows after the block rows, each already in column order, so
    # the CSR is the block CSR with the linking rows appended (no global sort)
    per_link = int(round(linking_frac * n))
    nb = idx_b.size
    idx = np.empty(nb + linking_rows * per_link, dtype=np.int64)
    idx[:nb] = idx_b
    for r in range(linking_rows):
        idx[nb + r * per_link:nb + (r + 1) * per_link] = np.sort(
            rng.choice(n, per_link, replace=False))
    val = np.empty(idx.size, dtype=np.float64)
    val[:nb] = val_b
    vl = rng.uniform(0.1, 2.0, idx.size - nb)
    vl[rng.random(vl.size) < 0.3] *= -1
    val[nb:] = vl
    ptr = np.empty(m + 1, dtype=np.int64)
    ptr[:mb + 1] = ptr_b
    ptr[mb + 1:] = nb + per_link * np.arange(1, linking_rows + 1, dtype=np.int64)
    del idx_b, val_b, vl
    x0 = rng.uniform(0, x_hi, n)
    ax0 = csr_matvec(ptr, idx, val, x0, m)
    rl = ax0.copy()
    ru = ax0.copy()
    rl[mb:] = -INF
    ru[mb:] = ax0[mb:] + rng.uniform(0, 1, linking_rows)
    c = rng.uniform(-1, 1, n)
    return Model(m=m, n=n, ptr=ptr, idx=idx, val=val, c=c, q=np.zeros(n), lb=np.zeros(n),
                 ub=np.full(n, box_hi), rl=rl, ru=ru,
                 name=f"block_angular_b{blocks}_s{seed}", x0=x0)


def sparse_qp_terms(rng, n: int, rank: int = 4, sigma: float = 0.1):
    """Q = L L^T with L n x rank sparse N(0, sigma^2): each column of L has
    ceil(sqrt(n)) nonzeros at distinct random rows, so nnz(L L^T) <= rank * n.
    Returns the symmetric CSR of L L^T (canonical) and D ~ U[0.1, 1] for the
    diagonal shorthand q."""
    s = max(1, int(math.ceil(math.sqrt(n))))
    s = min(s, n)
    qr, qc, qv = [], [], []
    for t in range(rank):
        rows = np.sort(rng.choice(n, s, replace=False)).astype(np.int64)
        vals = rng.normal(0, sigma, s)
        # outer product of this column of L with itself
        qr.append(np.repeat(rows, s))
        qc.append(np.tile(rows, s))
        qv.append(np.outer(vals, vals).reshape(-1))
    r = np.concatenate(qr)
    cidx = np.concatenate(qc)
    v = np.concatenate(qv)
    key = r * n + cidx
    uk, inv = np.unique(key, return_inverse=True)
    sums = np.zeros(uk.size)
    # sum duplicates in a fixed order (sorted by key, then by input position)
    order = np.argsort(inv, kind="stable")
    np.add.at(sums, inv[order], v[order])
    # (i,j) and (j,i) receive the same products v_i*v_j in the same column order,
    # so the sums are bitwise symmetric, as Model::validate requires.
    rr = uk // n
    cc = uk % n
    keep = sums != 0
    qptr, qidx, qval = _canonical_csr(rr[keep], cc[keep], sums[keep], n)
    d = rng.uniform(0.1, 1.0, n)
    return qptr, qidx, qval, d


def batch_instance(rng, m: int, qp: bool, x_hi: float = 10.0, name: str = "inst") -> Model:
    """One instance of the uneven LP/QP mix: m equality rows at x0 ~ U[0,x_hi], n = 2m columns,
    each column with 4-8 nonzeros (uniform) at distinct random rows, values N(0,1),
    bounds [0, x_hi], c ~ N(0,1); QPs add Q = D + L L^T."""
    n = 2 * m
    per = rng.integers(4, 9, size=n)
    per = np.minimum(per, m)
    cols = np.repeat(np.arange(n, dtype=np.int64), per)
    rows = rng.integers(0, m, size=cols.size)
    rows = _dedupe_pairs(rng, cols, rows, m)
    vals = rng.standard_normal(cols.size)
    ptr, idx, val = _canonical_csr(rows, cols, vals, m)
    x0 = rng.uniform(0, x_hi, n)
    b = csr_matvec(ptr, idx, val, x0, m)
    c = rng.standard_normal(n)
    q = np.zeros(n)
    qptr = qidx = qval = None
    if qp:
        qptr, qidx, qval, q = sparse_qp_terms(rng, n)
    return Model(m=m, n=n, ptr=ptr, idx=idx, val=val, c=c, q=q, lb=np.zeros(n),
                 ub=np.full(n, x_hi), rl=b.copy(), ru=b.copy(), qptr=qptr, qidx=qidx, qval=qval,
                 name=name, x0=x0)


def batch_instances(count: int = 512, m_lo: int = 500, m_hi: int = 50_000, qp_frac: float = 0.2,
                    seed: int = 4) -> list:
    """The uneven LP/QP mix (512 instances with m up to 50,000 for the batch; m up to
    200,000 for the served stream): m log-uniform on
    [m_lo, m_hi], a fraction ``qp_frac`` of convex QPs."""
    rng = np.random.default_rng(seed)
    ms = np.exp(rng.uniform(math.log(m_lo), math.log(m_hi), count)).astype(np.int64)
    kinds = rng.random(count) < qp_frac
    out = []
    for k in range(count):
        sub = np.random.default_rng([seed, k])
        out.append(batch_instance(sub, int(ms[k]), bool(kinds[k]), name=f"inst{k}"))
    return out
