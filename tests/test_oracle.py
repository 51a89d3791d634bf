"""The oracle (oracle/pdhg_oracle.c) pinned against the reference.

Two pins: (1) the reference's own CPU build (oracle/_ref), run side by side on
seeded instances -- bit-identical results are required; (2) the committed golden
fixtures generated from that build (tests/golden/make_golden.py), and the
known answers in the reference's own tests (tests/test_research.cpp,
tests/test_core.cpp), so the oracle stays pinned where oracle/_ref is absent.
"""
import json
import math

import numpy as np
import pytest

from niryukti_b200 import synth
from tests.conftest import load_golden


def tiny(n, rows, entries):
    """The reference tests' `model(n, rows, entries)` helper (tests/test_research.cpp:18-33):
    bounds [-10, 10], free rows, zero objective."""
    r = np.array([e[0] for e in entries], dtype=np.int64)
    c = np.array([e[1] for e in entries], dtype=np.int64)
    v = np.array([e[2] for e in entries], dtype=np.float64)
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    ptr = np.zeros(rows + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=rows), out=ptr[1:])
    return synth.Model(m=rows, n=n, ptr=ptr, idx=c, val=v, c=np.zeros(n), q=np.zeros(n),
                       lb=np.full(n, -10.0), ub=np.full(n, 10.0), rl=np.full(rows, -math.inf),
                       ru=np.full(rows, math.inf))


def near(a, b, tol=1e-11):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    assert np.all(np.abs(a - b) <= tol * (1 + np.abs(b))), (a, b)


# ---------------------------------------------------------------- known answers
def test_acceptance_known_answer(oracle):
    # tests/test_research.cpp:34-49: first trial has dx=dy=2, E=4, C=4 -> rejected
    m = tiny(1, 1, [(0, 0, 1.0)])
    m.c[:] = -1
    m.rl[:] = m.ru[:] = 3
    om = oracle.model(m)
    b = om.backend(np.zeros(1), np.zeros(1), adaptive=True)
    assert b.advance(1, 2, 2) == 1
    assert b.rejected_steps() > 0
    x, y, ax, ay = b.candidates()
    assert 0 < x[0] < 2
    assert (x[0] ** 2 + y[0] ** 2) / x[0] >= 2 * abs(x[0] * y[0])
    near(ax[0], x[0])
    near(ay[0], y[0])


def halpern_expected():
    """The independent scalar recurrence of tests/test_research.cpp:71-79."""
    ex = ey = 0.0
    out = []
    for k in range(20):
        tx = ex - .5 * ey
        ty = ey + .5 * (2 * tx - ex - 1)
        w = (k + 1) / (k + 2)
        ex, ey = w * tx, w * ty
        out.append((ex, ey, tx, ty))
    return out


def test_halpern_known_answer(oracle):
    m = tiny(1, 1, [(0, 0, 1.0)])
    m.lb[:] = -math.inf
    m.ub[:] = math.inf
    m.rl[:] = m.ru[:] = 1
    b = oracle.model(m).backend(np.zeros(1), np.zeros(1), halpern=True)
    for ex, ey, tx, ty in halpern_expected():
        b.advance(1, .5, .5)
        x, y, rx, ry = b.candidates()
        near(x[0], ex)
        near(y[0], ey)
        near(rx[0], tx)
        near(ry[0], ty)
    b.reset(np.array([2.0]), np.array([3.0]))
    b.advance(1, .5, .5)
    x, y, _, _ = b.candidates()
    near(x[0], 1.25)
    near(y[0], 2.5)


def sparse_qp_model():
    # tests/test_research.cpp:118-125: optimum (1,2), objective -7
    m = tiny(2, 1, [(0, 0, 1.0), (0, 1, 1.0)])
    m.lb[:] = 0
    m.ub[:] = 4
    m.rl[:] = m.ru[:] = 3
    m.qptr = np.array([0, 2, 4], dtype=np.int64)
    m.qidx = np.array([0, 1, 0, 1], dtype=np.int64)
    m.qval = np.array([2.0, 1.0, 1.0, 2.0])
    m.c = np.array([-4.0, -5.0])
    return m


def test_sparse_qp_known_answer(oracle):
    r = oracle.model(sparse_qp_model()).solve()
    assert r["status"] == "OPTIMAL"
    near(r["x"][0], 1, 1e-5)
    near(r["x"][1], 2, 1e-5)
    near(r["objective"], -7, 1e-5)


def test_lp_optimum_known_answer(oracle):
    # tests/test_core.cpp optimum(m, 2): the LP with optimum 2 used across the suite
    m = tiny(2, 2, [(0, 0, 1.0), (0, 1, 1.0), (1, 0, 1.0), (1, 1, -1.0)])
    m.lb[:] = 0
    m.ub[:] = 4
    m.c = np.array([1.0, 2.0])
    m.rl = np.array([2.0, -1.0])
    m.ru = np.array([3.0, 2.0])
    r = oracle.model(m).solve(iteration_limit=200000)
    assert r["status"] == "OPTIMAL"
    near(r["objective"], 2, 1e-5)


# ---------------------------------------------------------------- golden fixtures
@pytest.mark.parametrize("name", ["steps_lp_adaptive", "steps_lp_fixed", "steps_lp_halpern",
                                  "steps_qp", "steps_skewed"])
def test_oracle_matches_golden_steps(oracle, name):
    model, d = load_golden(name)
    kw = json.loads(str(d["options"]))
    b = oracle.model(model).backend(np.zeros(model.n), np.zeros(model.m), **kw)
    for k in range(len(d["progress"])):
        assert b.advance(int(d["count"]), float(d["tau"]), float(d["sigma"])) == d["progress"][k]
        x, y, xa, ya = b.candidates()
        assert np.array_equal(x, d["x"][k]) and np.array_equal(y, d["y"][k])
        assert np.array_equal(xa, d["xa"][k]) and np.array_equal(ya, d["ya"][k])
        assert b.rejected_steps() == d["rejected"][k]


@pytest.mark.parametrize("tag", ["lp", "qp"])
def test_oracle_matches_golden_verifier(oracle, tag):
    model, d = load_golden(f"verify_{tag}")
    om = oracle.model(model)
    for row in d["points"]:
        x, y = row[:model.n], row[model.n:model.n + model.m]
        safe = int(row[model.n + model.m])
        want = row[model.n + model.m + 1:]
        got = om.verify(x, y, safe)
        got = [got[k] for k in ("objective", "primal", "dual", "gap", "kkt", "lower_bound")]
        assert np.array_equal(np.array(got), want)


def test_oracle_matches_golden_solve(oracle):
    model, d = load_golden("solve_small_lp")
    want = json.loads(str(d["result"]))
    r = oracle.model(model).solve(iteration_limit=200000)
    assert r["status"] == want["status"] == "OPTIMAL"
    assert r["iterations"] == want["iterations"] and r["restarts"] == want["restarts"]
    assert r["objective"] == want["objective"] and r["kkt"] == want["kkt"]
    assert np.array_equal(r["x"], d["x"]) and np.array_equal(r["y"], d["y"])


# ---------------------------------------------------------------- beside the reference build
def test_oracle_vs_reference_primitives(oracle, reference):
    m = synth.power_law_lp(m=2000, n=4000, nnz=30000, seed=7, len_hi=600)
    rm = reference.model(m)
    p, i, v = rm.csr()
    assert np.array_equal(p, m.ptr) and np.array_equal(i, m.idx) and np.array_equal(v, m.val)
    t_ref = rm.transpose()
    t_orc = oracle.transpose(m.ptr, m.idx, m.val, m.m, m.n)
    assert all(np.array_equal(a, b) for a, b in zip(t_ref, t_orc))
    x = np.random.default_rng(1).standard_normal(m.n)
    assert np.array_equal(rm.multiply(x), oracle.spmv(m.ptr, m.idx, m.val, x, m.m))


@pytest.mark.parametrize("kw", [dict(adaptive=True), dict(adaptive=False),
                                dict(halpern=True, reflection=1.0),
                                dict(halpern=True, reflection=0.3, restarts=True)])
def test_oracle_vs_reference_backend(oracle, reference, kw):
    m = synth.random_lp(m=300, n=700, per_col=4, seed=3)
    a = oracle.model(m).backend(np.zeros(m.n), np.zeros(m.m), **kw)
    b = reference.model(m).backend(np.zeros(m.n), np.zeros(m.m), **kw)
    for k in range(8):
        assert a.advance(9, 0.03, 0.04) == b.advance(9, 0.03, 0.04)
        ca, cb = a.candidates(), b.candidates()
        assert all(np.array_equal(u, w) for u, w in zip(ca, cb))
        assert a.rejected_steps() == b.rejected_steps()
        assert a.restart_requested() == b.restart_requested()
        if k == 4:
            a.reset(ca[2], ca[3])
            b.reset(cb[2], cb[3])
    sb, _ = b.snapshot()
    assert np.array_equal(a.snapshot(), sb)


def test_oracle_vs_reference_qp(oracle, reference):
    m = synth.batch_instance(np.random.default_rng(9), 80, True)
    om, rm = oracle.model(m), reference.model(m)
    assert om.quadratic_norm_bound() == rm.quadratic_norm_bound()
    a = om.backend(np.zeros(m.n), np.zeros(m.m))
    b = rm.backend(np.zeros(m.n), np.zeros(m.m))
    for _ in range(5):
        assert a.advance(7, 0.2, 0.2) == b.advance(7, 0.2, 0.2)
        assert all(np.array_equal(u, w) for u, w in zip(a.candidates(), b.candidates()))
    rng = np.random.default_rng(2)
    for safe in (0, 1):
        x = np.clip(m.x0 + rng.standard_normal(m.n), m.lb, m.ub)
        y = rng.standard_normal(m.m)
        assert om.verify(x, y, safe) == rm.verify(x, y, safe)


def test_oracle_vs_reference_scaling_and_solve(oracle, reference):
    m = synth.random_lp(m=150, n=400, per_col=4, seed=5)
    sa = oracle.model(m).scale(5)
    pb = reference.model(m).prepare(method="pdhg", device="cpu")
    for k in ("ptr", "idx", "val", "c", "lb", "ub", "rl", "ru", "column_scale", "row_scale"):
        assert np.array_equal(sa[k], pb[k]), k
    assert sa["objective_scale"] == pb["objective_scale"]
    a = oracle.model(m).solve(iteration_limit=50000)
    b = reference.model(m).solve(method="pdhg", device="cpu", iteration_limit=50000)
    assert a["status"] == b["status"]
    assert a["iterations"] == b["iterations"] and a["restarts"] == b["restarts"]
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["y"], b["y"])


def test_oracle_infeasibility_bound(oracle, reference):
    # contradictory rows x0 + x1 >= 3 and x0 + x1 <= 1 inside a box: a Farkas ray
    m = tiny(2, 2, [(0, 0, 1.0), (0, 1, 1.0), (1, 0, 1.0), (1, 1, 1.0)])
    m.lb[:] = 0
    m.ub[:] = 1
    m.rl = np.array([3.0, -math.inf])
    m.ru = np.array([math.inf, 1.0])
    ray = np.array([-1.0, 1.0])
    a = oracle.model(m).infeasibility_bound(ray)
    b = reference.model(m).infeasibility_bound(ray)
    assert a == b and a > 0


def test_reference_cpu_build_has_no_batched_relaxations(reference):
    """The harness reaches cuda_batch_relaxations; in the reference's CPU build
    it is the stub that asks for a CUDA build (src/cuda_stub.cpp:13-17)."""
    model = synth.random_lp(m=50, n=120, per_col=3, seed=2)
    with pytest.raises(RuntimeError, match="require a CUDA build"):
        reference.model(model).batch_relaxations(model.lb[None, :], model.ub[None, :], tol=1e-6)


def _one_row(vals, lb, ub, rl, ru):
    n = len(vals)
    return synth.Model(m=1, n=n, ptr=np.array([0, n]), idx=np.arange(n), val=np.array(vals, float),
                       c=np.zeros(n), q=np.zeros(n), lb=np.array(lb, float),
                       ub=np.array(ub, float), rl=np.array([rl], float), ru=np.array([ru], float))


def test_oracle_propagation_known_answers(oracle):
    """Bound proposals of cuda_propagate_integer_bounds (src/cuda.cu:468-529) on
    one-row cases: integer columns round inward, continuous ones keep the
    directed-rounded bound, a row whose activity range misses its bounds is
    infeasible."""
    m = _one_row([1, 1], [0, 0], [10, 10], -np.inf, 1.5)
    assert oracle.propagate_bounds(m, [1, 1], m.lb, m.ub)[2].tolist() == [1.0, 1.0]
    assert oracle.propagate_bounds(m, [0, 0], m.lb, m.ub)[2].tolist() == [1.5, 1.5]
    m = _one_row([1, 1], [1, 1], [10, 10], -np.inf, 1.5)
    assert oracle.propagate_bounds(m, [0, 0], m.lb, m.ub)[0] is False
    # 3 x = 1: the bounds bracket 1/3 by adjacent doubles (round down / round up)
    m = _one_row([3], [0], [10], 1, 1)
    ok, lb, ub = oracle.propagate_bounds(m, [0], m.lb, m.ub)
    assert ok and lb[0] <= 1 / 3 <= ub[0] and np.nextafter(lb[0], 1) == ub[0]
    # 0 <= x0 - x1 <= 2 with x0 in [0, 5] and x1 free bounds x1 to [-2, 5]; x0
    # gains nothing, since the free x1 leaves the rest of its row unbounded
    m = _one_row([1, -1], [0, -np.inf], [5, np.inf], 0, 2)
    ok, lb, ub = oracle.propagate_bounds(m, [0, 0], m.lb, m.ub)
    assert ok and lb.tolist() == [0.0, -2.0] and ub.tolist() == [5.0, 5.0]


def test_monitor_formula_known_answer():
    """The host restatement of the reference's GPU KKT proxy
    (src/cuda.cu:387-446) on the sparse QP of tests/test_research.cpp:118-125
    at x = (1, 1), y = 0.5, worked by hand: A x = 2 against rl = ru = 3 gives a
    row violation 1/4; g = c + Q x + A^T y = (-0.5, -1.5) gives dual residuals
    0.5/6 and 1.5/6 (cscale = 1 + 5); complementarity 0.5*3 + 1.5*3 + 0.5*(3-2)
    = 6.5 over 1 + |c.x + x'Qx/2| = 1 + |-9 + 3| = 7."""
    from oracle.monitor import cscale_of, monitor, monitor_point
    m = sparse_qp_model()
    x, y = np.array([1.0, 1.0]), np.array([0.5])
    assert cscale_of(m.c) == 6.0
    assert monitor_point(m, x, y) == pytest.approx(6.5 / 7, rel=1e-15)
    # at the optimum (1, 2) with y = 0 every term vanishes
    assert monitor_point(m, np.array([1.0, 2.0]), np.zeros(1)) == 0.0
    assert monitor(m, x, y, np.array([1.0, 2.0]), np.zeros(1)) == 0.0
    # a bound violation relative to 1 + |x|, and a non-finite point
    assert monitor_point(m, np.array([5.0, -2.0]), np.zeros(1)) >= 1.0 / 6
    assert monitor_point(m, np.array([np.nan, 1.0]), np.zeros(1)) == np.inf


def test_monitor_formula_infinite_endpoints():
    """Rows with an infinite endpoint: a dual sign that selects it counts |y_i|
    as a dual residual (src/cuda.cu:414-420); a finite one counts
    complementarity.  One free column at x = 2, c = 0, rows x >= 1 and x <= 4."""
    from oracle.monitor import monitor_point
    m = tiny(1, 2, [(0, 0, 1.0), (1, 0, 1.0)])
    m.lb[:], m.ub[:] = -math.inf, math.inf
    m.rl = np.array([1.0, -math.inf])
    m.ru = np.array([math.inf, 4.0])
    x = np.array([2.0])
    # g = A^T y = 0.25 is the column's dual residual; y_0 < 0 selects rl = 1:
    # 0.25 * |1 - 2|; y_1 > 0 selects ru = 4: 0.5 * |4 - 2|; over 1 + |0|
    assert monitor_point(m, x, np.array([-0.25, 0.5])) == 1.25
    # y_0 > 0 selects ru = +inf: |y_0| = 3 is a dual residual (and so is g = 3)
    assert monitor_point(m, x, np.array([3.0, 0.0])) == 3.0
    # a row violation relative to 1 + |rl|: x = 0.5 against rl = 1
    assert monitor_point(m, np.array([0.5]), np.zeros(2)) == 0.25
