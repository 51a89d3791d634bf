"""Batched engine (nk_batch_*): many uneven LP / QP instances on one GPU.

Each instance runs the same driver as a single solve, so the checks are the
single-solve checks per instance (certified KKT, objective against the CPU
oracle or the reference), plus what is specific to batching: an instance's
result does not depend on what else is in the batch, admission honours the
memory budget, and instances that terminate early leave the rest running.
"""
import math

import numpy as np
import pytest

from niryukti_b200 import synth
from tests.test_host import infeasible_models, presolve_model
from tests.test_oracle import sparse_qp_model

pytestmark = pytest.mark.gpu

TOL = 1e-6


def objective_close(a, b, tol=TOL):
    assert abs(a - b) <= 2 * tol * (1 + abs(b)), (a, b)


@pytest.fixture(scope="module")
def batch(gpu):
    from niryukti_b200 import batch as b
    return b


def small_mix(seed=4, count=6):
    return synth.batch_instances(count=count, m_lo=40, m_hi=300, qp_frac=0.34, seed=seed)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_single_solves(batch, precision):
    from niryukti_b200 import solver
    models = small_mix()
    res = batch.solve_batch(models, matrix_precision=precision, iteration_limit=300000,
                            time_limit=120)
    for k, (m, r) in enumerate(zip(models, res)):
        assert r["status"] == "OPTIMAL", (k, r["status"], r["kkt"], r["iterations"])
        assert r["kkt"] <= TOL
        again = solver.verify(m, r["x"], r["y"])  # certified on the caller's model
        assert again["kkt"] <= TOL
        single = solver.solve(m, iteration_limit=300000, time_limit=120)
        assert single["status"] == "OPTIMAL"
        objective_close(r["objective"], single["objective"])


def test_batch_fp64_matches_oracle_objectives(batch, oracle):
    models = [m for m in small_mix(seed=9) if not m.is_qp()][:3]
    res = batch.solve_batch(models, matrix_precision="fp64", iteration_limit=400000,
                            time_limit=120)
    for m, r in zip(models, res):
        ref = oracle.model(m).solve(tol=TOL, iteration_limit=400000, time_limit=120)
        assert r["status"] == ref["status"] == "OPTIMAL"
        objective_close(r["objective"], ref["objective"])


def test_result_is_the_same_alone_and_in_the_mix(batch):
    """Per-instance sums never mix instances, and every kernel variant adds in
    the same order: the trajectory of an instance is identical alone and in a
    batch, so its iteration count and result match exactly."""
    models = small_mix(seed=7, count=5)
    together = batch.solve_batch(models, matrix_precision="mixed", iteration_limit=300000,
                                 time_limit=120)
    for k in (0, 3):
        alone = batch.solve_batch([models[k]], matrix_precision="mixed",
                                  iteration_limit=300000, time_limit=120)[0]
        assert alone["status"] == together[k]["status"] == "OPTIMAL"
        assert alone["iterations"] == together[k]["iterations"]
        assert alone["objective"] == together[k]["objective"]
        assert np.array_equal(alone["x"], together[k]["x"])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotuning_leaves_no_trace(batch, precision):
    """The autotuner times its kernel variants with probe trials on the first
    work list: they apply no pending average and make no decision.  Every
    instance's trajectory, hence its iteration count and result, is the same
    bit for bit with and without tuning."""
    models = small_mix(seed=12, count=4)
    tuned = batch.solve_batch(models, matrix_precision=precision, iteration_limit=300000,
                              time_limit=120, autotune=True)
    plain = batch.solve_batch(models, matrix_precision=precision, iteration_limit=300000,
                              time_limit=120, autotune=False)
    for a, b in zip(tuned, plain):
        assert a["status"] == b["status"] == "OPTIMAL"
        assert a["iterations"] == b["iterations"]
        assert a["objective"] == b["objective"]
        assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["y"], b["y"])


def test_batch_terminal_statuses(batch):
    from tests.test_host import from_rows
    unbounded = presolve_model()
    infeasible = from_rows(2, [[(0, 1.0), (1, 1.0)], [(0, 2.0), (1, 2.0)]], c=[1.0, 1.0],
                           lb=[0, 0], ub=[5, 5], rl=[3, -math.inf], ru=[math.inf, 2])
    models = [sparse_qp_model(), unbounded, infeasible, infeasible_models()["duplicate"]]
    res = batch.solve_batch(models, matrix_precision="fp64")
    assert [r["status"] for r in res] == ["OPTIMAL", "UNBOUNDED", "INFEASIBLE", "INFEASIBLE"]
    assert abs(res[0]["objective"] + 7) < 1e-5


def test_admission_by_memory_budget(batch):
    models = small_mix(seed=11, count=4)
    with batch.BatchEngine(matrix_precision="mixed", memory_budget=1.0) as eng:
        item = eng.prepare(models[0])
        assert item.device_bytes > 1.0
        assert not eng.admit(item, 0)  # does not fit a 1-byte budget
    sizes = [batch.BatchEngine(matrix_precision="mixed").prepare(m).device_bytes for m in models]
    budget = max(sizes) * 1.5  # room for one instance at a time
    res = batch.solve_batch(models, matrix_precision="mixed", memory_budget=budget,
                            iteration_limit=300000, time_limit=120)
    assert all(r["status"] == "OPTIMAL" for r in res)


def test_autotuner_reports_a_variant(batch):
    with batch.BatchEngine(matrix_precision="mixed") as eng:
        for k, m in enumerate(small_mix(seed=5, count=3)):
            assert eng.admit(eng.prepare(m), k)
        eng.step(1)
        info = eng.info()
        assert info["primal_variant"]["unroll"] in (2, 4, 8)
        assert info["dual_variant"]["threads"] in (128, 256, 512)
        ms, bts = eng.time_trials(10)
        assert ms > 0 and bts > 0
