"""Host stages of the solve path, pinned bit-exactly against the reference.

The engine library's presolve/scaling (nk_prepare) and verifier (nk_verify,
nk_infeasibility_bound) must reproduce the reference's prepare()
(src/preprocess.cpp:133-346) and Verifier (src/verify.cpp:6-244) to the bit:
every map, every scaled coefficient, every accuracy field.  Compared against the
reference's own build (oracle/_ref) on models that exercise each presolve rule:
fixed and unused columns, substituted-empty rows, redundant rows, duplicate rows
(tightened and contradictory), disjoint activity bounds, QP couplings with
removed columns, and both scaling schemes.  CPU only (no GPU needed).
"""
import math

import numpy as np
import pytest

from niryukti_b200 import solver, synth
from tests.test_oracle import sparse_qp_model, tiny

INF = math.inf


def from_rows(n, rows, c=None, q=None, lb=None, ub=None, rl=None, ru=None, qentries=None):
    """Model from a list of dense-ish rows [(col, value), ...]."""
    ptr = [0]
    idx, val = [], []
    for r in rows:
        for j, v in sorted(r):
            idx.append(j)
            val.append(v)
        ptr.append(len(idx))
    m = synth.Model(m=len(rows), n=n, ptr=np.array(ptr, dtype=np.int64),
                    idx=np.array(idx, dtype=np.int64), val=np.array(val, dtype=float),
                    c=np.zeros(n) if c is None else np.array(c, float),
                    q=np.zeros(n) if q is None else np.array(q, float),
                    lb=np.full(n, -INF) if lb is None else np.array(lb, float),
                    ub=np.full(n, INF) if ub is None else np.array(ub, float),
                    rl=np.array(rl, float), ru=np.array(ru, float))
    if qentries:
        Q = {}
        for i, j, v in qentries:
            Q[(i, j)] = Q.get((i, j), 0) + v
            if i != j:
                Q[(j, i)] = Q.get((j, i), 0) + v
        keys = sorted(Q)
        qptr = np.zeros(n + 1, dtype=np.int64)
        for i, _ in keys:
            qptr[i + 1] += 1
        m.qptr = np.cumsum(qptr)
        m.qidx = np.array([j for _, j in keys], dtype=np.int64)
        m.qval = np.array([Q[k] for k in keys])
    return m


def presolve_model():
    """Every presolve rule at once (all kept rows feasible)."""
    n = 9
    rows = [
        [(0, 1.0), (1, 2.0), (2, -1.0)],          # 0 kept
        [(0, 1.0), (1, 2.0), (2, -1.0)],          # 1 duplicate of 0 (tighter lower)
        [(3, 2.0)],                               # 2 only a fixed column: empty after substitution
        [(0, 1e-3), (1, 1e-3)],                   # 3 redundant: activity inside [-1, 1]
        [(1, 3.0), (3, 1.0), (4, 5.0)],           # 4 kept, shifted by fixed column 3
        [(0, 250.0), (4, -0.004), (5, 1.0)],      # 5 badly scaled row
        [(0, 1.0), (1, 2.0), (2, -1.0)],          # 6 duplicate of 0 (tighter upper)
        [(5, 1.0), (8, 2.0)],                     # 7 kept
    ]
    c = [1.0, -2.0, 0.5, 3.0, 1.0, -1.0, 2.0, -3.0, 0.0]
    lb = [0, 0, -5, 2, 0, -INF, 0, 0, -1]
    ub = [4, 4, 5, 2, 10, INF, 7, INF, 1]      # col 3 fixed; 6 unused (c>0 -> lb); 7 unused c<0 ub=inf
    rl = [-10, -8, 3.0, -1, -INF, -20, -10, 0]
    ru = [10, 10, 5.0, 1, 30, 20, 6, 4]
    return from_rows(n, rows, c=c, lb=lb, ub=ub, rl=rl, ru=ru)


def presolve_qp():
    m = presolve_model()
    m.ub[7] = 6.0  # bounded so the QP has a minimiser
    q = np.zeros(m.n)
    q[6] = 2.0       # unused column with curvature: clamp(-c/q)
    q[1] = 0.5
    m.q = q
    qm = from_rows(m.n, [[]], rl=[0], ru=[0],
                   qentries=[(0, 0, 2.0), (0, 1, 0.5), (1, 1, 1.0), (3, 4, 0.25), (3, 3, 1.0),
                             (4, 4, 3.0)])
    m.qptr, m.qidx, m.qval = qm.qptr, qm.qidx, qm.qval
    return m


def random_presolve_model(seed, m=300, n=700, per_col=4, fixed=40, dups=25, redundant=10):
    """A random LP with fixed columns, duplicated and redundant rows."""
    base = synth.random_lp(m=m, n=n, per_col=per_col, seed=seed)
    rng = np.random.default_rng(seed)
    lb, ub = base.lb.copy(), base.ub.copy()
    fixed = rng.choice(base.n, fixed, replace=False)
    lb[fixed] = ub[fixed] = base.x0[fixed]
    rows = [list(zip(base.idx[base.ptr[i]:base.ptr[i + 1]].tolist(),
                     base.val[base.ptr[i]:base.ptr[i + 1]].tolist())) for i in range(base.m)]
    rl, ru = base.rl.tolist(), base.ru.tolist()
    for i in rng.choice(base.m, dups, replace=False):   # duplicates with looser/tighter bounds
        rows.append(rows[i])
        slack = float(rng.uniform(0, 1))
        rl.append(rl[i] - slack)
        ru.append(ru[i] + slack)
    for _ in range(redundant):                            # redundant rows
        cols = rng.choice(base.n, 3, replace=False)
        rows.append([(int(j), 1e-4) for j in cols])
        rl.append(-1.0)
        ru.append(1.0)
    return from_rows(base.n, rows, c=base.c, lb=lb, ub=ub, rl=rl, ru=ru)


def infinite_bounds_model():
    """Rows whose activity-bound verdict hinges on infinite column bounds: a
    free or one-sided column first, in the middle or last in a row, with either
    coefficient sign, keeps a row that its finite columns alone would make
    redundant; the duplicate of such a row is still merged."""
    inf = np.inf
    lb = [0, -inf, 0, 0, 0, -inf, 0, 0, 0]
    ub = [1, inf, 1, inf, 1, 5, 1, 1, 1]
    rows = [[(0, 1e-4), (2, 1e-4)],                # finite and redundant: dropped
            [(1, 1e-4), (2, 1e-4), (4, 1e-4)],     # free column first
            [(0, 1e-4), (1, -1e-4), (2, 1e-4)],    # free column in the middle
            [(0, 1e-4), (2, 1e-4), (3, 1e-4)],     # upper bound +inf, last
            [(0, 1e-4), (3, -1e-4)],               # upper bound +inf, negative coefficient
            [(4, 1e-4), (5, 1e-4)],                # lower bound -inf
            [(5, -1e-4), (8, 1e-4)],               # lower bound -inf, negative coefficient
            [(6, 1.0), (7, 1.0)],                  # finite and binding
            [(3, 1.0), (8, 1.0)],                  # disjoint-looking, but x3 is unbounded
            [(1, 1e-4), (2, 1e-4), (4, 1e-4)]]     # duplicate of row 1
    rl = [-1, -1, -1, -1, -1, -1, -1, 0.5, 5, -0.5]
    ru = [1, 1, 1, 1, 1, 1, 1, 1.5, 10, 0.5]
    return from_rows(9, rows, c=[1, 0.5, -1, 1, 0, -0.5, 1, 1, 0], lb=lb, ub=ub, rl=rl, ru=ru)


def subnormal_model():
    """A column holding the smallest subnormal: its entry would underflow to 0
    under the column's Ruiz factor, so the column keeps factor 1; and a row
    whose own factor would zero that entry is left unscaled."""
    tiny = float(np.nextafter(0.0, 1.0))
    rows = [[(0, 1e6), (2, 3.0)],
            [(0, tiny), (1, 1e6)],
            [(1, 2.0), (2, 5e-3)],
            [(2, 7.0), (3, tiny * 4)],
            [(3, 0.5), (0, 2.0)]]
    return from_rows(4, rows, c=[1, -1, 0.5, 2], lb=[0] * 4, ub=[10] * 4,
                     rl=[-1, -1, -1, -1, -1], ru=[10, 10, 10, 10, 10])


MODELS = {
    "subnormal": subnormal_model,
    "infinite_bounds": infinite_bounds_model,
    "presolve": presolve_model,
    "presolve_qp": presolve_qp,
    "sparse_qp": sparse_qp_model,
    "random_11": lambda: random_presolve_model(11),
    "random_12": lambda: random_presolve_model(12),
    "power_law": lambda: synth.power_law_lp(m=2000, n=4000, nnz=40000, seed=5),
}
OPTIONS = [dict(presolve=True, scaling="ruiz", scaling_passes=5),
           dict(presolve=False, scaling="ruiz", scaling_passes=5),
           dict(presolve=True, scaling="combined", scaling_passes=5),
           dict(presolve=True, scaling="ruiz", scaling_passes=0)]


def same(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if a.dtype.kind == "f":
        # bit-identical, NaN-free; +-inf compare equal to themselves
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), (what, a, b)
    else:
        assert np.array_equal(a, b), (what, a, b)


@pytest.mark.parametrize("opts", OPTIONS, ids=lambda o: "-".join(str(v) for v in o.values()))
@pytest.mark.parametrize("name", sorted(MODELS))
def test_prepare_bit_exact(reference, name, opts):
    model = MODELS[name]()
    mine = solver.prepare(model, **opts)
    ref = reference.model(model).prepare(**opts)
    assert ("failure" in mine) == ("failure" in ref)
    if "failure" in ref:
        return
    for key in ("ptr", "idx", "val", "c", "q", "lb", "ub", "rl", "ru", "cols", "rows",
                "lower_rows", "upper_rows", "fixed", "column_scale", "row_scale", "qptr", "qidx",
                "qval"):
        same(mine[key], ref[key], key)
    same([mine["objective_scale"], mine["offset"]], [ref["objective_scale"], ref["offset"]],
         "scalars")


@pytest.mark.parametrize("opts", OPTIONS[:2], ids=["presolve", "no-presolve"])
def test_prepare_bit_exact_threaded(reference, opts):
    """Above 200,000 nonzeros the row pass and the scaling loops run on all
    host threads; the prepared model must still be the reference's, bit for
    bit (fixed columns, duplicated and redundant rows included)."""
    model = random_presolve_model(21, m=30000, n=70000, per_col=6, fixed=4000, dups=2500,
                                  redundant=1000)
    assert model.nnz > 200000
    mine = solver.prepare(model, **opts)
    ref = reference.model(model).prepare(**opts)
    for key in ("ptr", "idx", "val", "c", "lb", "ub", "rl", "ru", "cols", "rows", "lower_rows",
                "upper_rows", "fixed", "column_scale", "row_scale"):
        same(mine[key], ref[key], key)
    same([mine["objective_scale"], mine["offset"]], [ref["objective_scale"], ref["offset"]],
         "scalars")
    if opts["presolve"]:
        assert len(mine["rows"]) < model.m  # the presolve rules did remove rows


def test_presolve_rules_fire(reference):
    """The hand-made model really exercises the reductions the test is about."""
    p = solver.prepare(presolve_model())
    assert 3 not in p["cols"] and 6 not in p["cols"]       # fixed / unused columns removed
    assert 7 in p["cols"]                                   # unused with infinite choice kept
    kept = set(p["rows"].tolist())
    assert 1 not in kept and 6 not in kept                  # duplicates merged
    assert 2 not in kept and 3 not in kept                  # empty-after-substitution, redundant
    r0 = p["rows"].tolist().index(0)
    assert p["lower_rows"][r0] == 1 and p["upper_rows"][r0] == 6


def test_infinite_bounds_keep_rows():
    p = solver.prepare(infinite_bounds_model())
    assert p["rows"].tolist() == [1, 2, 3, 4, 5, 6, 7, 8]  # row 0 dropped, row 9 merged
    assert p["lower_rows"][0] == 9 and p["upper_rows"][0] == 9


def infeasible_models():
    dup = from_rows(2, [[(0, 1.0), (1, 1.0)], [(0, 1.0), (1, 1.0)]], lb=[0, 0], ub=[5, 5],
                    rl=[0, 4], ru=[2, 6])
    act = from_rows(2, [[(0, 1.0), (1, 1.0)]], lb=[0, 0], ub=[1, 1], rl=[3], ru=[4])
    empty = from_rows(2, [[(0, 2.0)], [(1, 1.0)]], lb=[1, 0], ub=[1, 1], rl=[5, 0], ru=[6, 1])
    return {"duplicate": dup, "activity": act, "empty": empty}


@pytest.mark.parametrize("name", ["duplicate", "activity", "empty"])
def test_prepare_infeasible(reference, name):
    model = infeasible_models()[name]
    assert solver.prepare(model) == {"failure": "INFEASIBLE"}
    assert reference.model(model).prepare()["failure"] == "INFEASIBLE"


@pytest.mark.parametrize("safe", [True, False])
@pytest.mark.parametrize("name", sorted(MODELS))
def test_verify_bit_exact(reference, name, safe):
    model = MODELS[name]()
    rng = np.random.default_rng(3)
    ref = reference.model(model)
    for trial in range(3):
        x = rng.normal(size=model.n) * 2
        if trial == 1:  # inside the box: the feasible-side branches
            lo = np.where(np.isfinite(model.lb), model.lb, -3.0)
            hi = np.where(np.isfinite(model.ub), model.ub, 3.0)
            x = rng.uniform(lo, hi)
        y = rng.normal(size=model.m)
        if trial == 2:
            y[rng.random(model.m) < .5] = 0
        a = solver.verify(model, x, y, safe)
        b = ref.verify(x, y, safe)
        same([a[k] for k in solver.ACCURACY_KEYS], [b[k] for k in solver.ACCURACY_KEYS],
             f"accuracy trial {trial}")
        same(solver.infeasibility_bound(model, y), ref.infeasibility_bound(y), "farkas")


def test_verify_bit_exact_threaded(reference):
    """Above a million nonzeros the verifier's transpose is built by row blocks
    on all host threads; the outward-rounded bound and every accuracy field
    must still be the reference's, bit for bit."""
    model = synth.power_law_lp(m=100000, n=200000, nnz=2000000, seed=4, len_hi=3000)
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 5, model.n)
    y = rng.normal(size=model.m) * 1e-2
    ref = reference.model(model)
    for safe in (True, False):
        a = solver.verify(model, x, y, safe)
        b = ref.verify(x, y, safe)
        same([a[k] for k in solver.ACCURACY_KEYS], [b[k] for k in solver.ACCURACY_KEYS],
             f"accuracy safe={safe}")
    same(solver.infeasibility_bound(model, y), ref.infeasibility_bound(y), "farkas")


def test_invalid_model_rejected():
    m = tiny(2, 1, [(0, 0, 1.0)])
    m.lb[0] = 5.0
    m.ub[0] = 1.0
    from niryukti_b200.engine import EngineError
    with pytest.raises(EngineError, match="Invalid bounds"):
        solver.prepare(m)
    m = tiny(2, 1, [(0, 0, 1.0)])
    m.c[1] = math.nan
    with pytest.raises(EngineError, match="Nonfinite objective"):
        solver.verify(m, np.zeros(2), np.zeros(1))
