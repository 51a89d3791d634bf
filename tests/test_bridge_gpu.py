"""The drop-in: the reference's own host code with the B200 engine at its
cuda_backend() seam (oracle/_ref/libvantage_nk.so, built by `make -C oracle
bridge` from the reference sources plus niryukti_b200/bridge/).

Everything above the seam is the reference's unmodified code: its backend
factory, its solve_continuous driver, presolve and verifier.  The tests check
that the bridged CUDA backend steps like the reference's CPU backend and that
the reference's own solve with --device cuda reaches its CPU answer.
"""
import json

import numpy as np
import pytest

from niryukti_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bridged(gpu):
    from oracle.oracle import BRIDGE_SO, Reference
    if not BRIDGE_SO.exists():
        pytest.fail("bridged reference build oracle/_ref/libvantage_nk.so is missing")
    return Reference(BRIDGE_SO)


def test_bridge_reports_the_device(bridged):
    assert bridged.cuda_available()


@pytest.mark.parametrize("kw", [dict(adaptive=False), dict(halpern=True, reflection=1.0)])
def test_bridged_backend_steps_like_cpu(bridged, reference, kw):
    model = synth.random_lp(m=300, n=700, per_col=4, seed=3)
    x0, y0 = np.zeros(model.n), np.zeros(model.m)
    tau = sigma = 0.05
    cpu = reference.model(model).backend(x0, y0, device="cpu", **kw)
    gpu = bridged.model(model).backend(x0, y0, device="cuda", graphs=True, **kw)
    for _ in range(3):  # fixed steps: every trial is accepted on both sides
        assert gpu.advance(50, tau, sigma) == cpu.advance(50, tau, sigma)
        for a, b in zip(gpu.candidates(), cpu.candidates()):
            assert np.allclose(a, b, rtol=1e-11, atol=1e-11)


def test_bridged_solve_matches_cpu_solve(bridged, reference):
    from tests.conftest import load_golden
    model, d = load_golden("solve_small_lp")
    want = json.loads(str(d["result"]))
    r = bridged.model(model).solve(method="pdhg", device="cuda", iteration_limit=200000)
    assert r["status"] == want["status"] == "OPTIMAL"
    assert r["kkt"] <= 1e-6
    assert abs(r["objective"] - want["objective"]) <= 2e-6 * (1 + abs(want["objective"]))


def test_bridged_solve_mixed_precision(bridged):
    from tests.conftest import load_golden
    model, d = load_golden("solve_small_lp")
    want = json.loads(str(d["result"]))
    r = bridged.model(model).solve(method="pdhg", device="cuda", matrix_precision="mixed",
                                   cuda_graphs=True, iteration_limit=200000)
    assert r["status"] == "OPTIMAL" and r["kkt"] <= 1e-6
    assert abs(r["objective"] - want["objective"]) <= 2e-6 * (1 + abs(want["objective"]))


def _branching_boxes(model, x, count=4):
    """Down and up boxes of the first `count` columns that sit strictly inside
    their bounds at a fractional value -- the shortlist the reference's
    branch-and-bound scores (src/mip.cpp:1094-1118)."""
    frac = np.where((x > model.lb + 0.2) & (x < model.ub - 0.2) &
                    (np.abs(x - np.round(x)) > 0.2))[0][:count]
    lows, ups = [], []
    for j in frac:
        for up in (False, True):
            lo, hi = model.lb.copy(), model.ub.copy()
            if up:
                lo[j] = np.ceil(x[j])
            else:
                hi[j] = np.floor(x[j])
            lows.append(lo)
            ups.append(hi)
    return np.array(lows), np.array(ups)


def test_bridged_batch_relaxations(bridged, reference):
    """cuda_batch_relaxations through the bridge: eight strong-branching boxes
    of one LP, warm-started from the parent's solution, solved together by the
    engine's batch.  Every box must come back OPTIMAL under the reference's own
    verify(), with the objective of the reference's CPU solve of that box
    (within 2 tol (1 + |f|))."""
    import copy
    model = synth.random_lp(m=300, n=700, per_col=4, seed=3)
    parent = reference.model(model).solve(method="pdhg", device="cpu", iteration_limit=200000)
    assert parent["status"] == "OPTIMAL"
    lows, ups = _branching_boxes(model, parent["x"])
    assert len(lows) == 8
    got = bridged.model(model).batch_relaxations(lows, ups, x0=parent["x"], y0=parent["y"],
                                                 tol=1e-6, iteration_limit=200000,
                                                 time_limit=120)
    for b, r in enumerate(got):
        child = copy.copy(model)
        child.lb, child.ub = lows[b], ups[b]
        want = reference.model(child).solve(method="pdhg", device="cpu", iteration_limit=200000)
        assert want["status"] == "OPTIMAL"
        assert r["status"] == "OPTIMAL" and r["kkt"] <= 1e-6, (b, r["status"], r["kkt"])
        assert abs(r["objective"] - want["objective"]) <= 2e-6 * (1 + abs(want["objective"]))
        # the returned point is the box's own: within its bounds
        assert np.all(r["x"] >= lows[b] - 1e-9) and np.all(r["x"] <= ups[b] + 1e-9)


def test_bridged_batch_relaxations_checks_bounds(bridged):
    """The reference's argument checks: a box outside the model's bounds is refused."""
    model = synth.random_lp(m=300, n=700, per_col=4, seed=3)
    lo, hi = model.lb.copy()[None, :], model.ub.copy()[None, :]
    hi[0, 5] = model.ub[5] + 1.0
    with pytest.raises(RuntimeError, match="Invalid batch bounds"):
        bridged.model(model).batch_relaxations(lo, hi, tol=1e-6)


@pytest.mark.parametrize("name", ["presolve", "random_11", "power_law", "large"])
def test_bridged_gpu_presolve_compaction_bit_exact(bridged, reference, name):
    """prepare with --gpu-presolve in the reference's own presolve: the kept
    rows and columns are compacted by the engine (cuda_compact_matrix), and the
    prepared model must be bit-identical to the reference's CPU prepare."""
    from tests.test_host import MODELS, random_presolve_model, same
    model = (random_presolve_model(21, m=30000, n=70000, per_col=6, fixed=4000, dups=2500,
                                   redundant=1000) if name == "large" else MODELS[name]())
    mine = bridged.model(model).prepare(presolve=True, gpu_presolve=True)
    ref = reference.model(model).prepare(presolve=True)
    assert ("failure" in mine) == ("failure" in ref)
    for key in ("ptr", "idx", "val", "c", "lb", "ub", "rl", "ru", "cols", "rows", "lower_rows",
                "upper_rows", "fixed", "column_scale", "row_scale"):
        same(mine[key], ref[key], key)


def test_bridged_solve_with_gpu_presolve(bridged, reference):
    """The reference's solve with --gpu-presolve through the bridge: bound
    proposals (cuda_propagate_integer_bounds) proven again by the reference's
    host code, CSR compaction (cuda_compact_matrix), then the engine's PDHG --
    the answer of the plain CPU solve."""
    from tests.conftest import load_golden
    model, d = load_golden("solve_small_lp")
    want = json.loads(str(d["result"]))
    r = bridged.model(model).solve(method="pdhg", device="cuda", gpu_presolve=True,
                                   iteration_limit=200000)
    assert r["status"] == want["status"] == "OPTIMAL"
    assert r["kkt"] <= 1e-6
    assert abs(r["objective"] - want["objective"]) <= 2e-6 * (1 + abs(want["objective"]))


def test_bridged_linear_solve(bridged):
    """cuda_linear_solve through the bridge (the barrier's Newton solve): the
    engine's BiCGSTAB, then the reference's acceptance test of the solution
    (finite, max-norm residual within the tolerance), on a nonsymmetric,
    diagonally dominant system."""
    from tests.test_engine_gpu import _newton_system
    ptr, idx, val, dense, rhs = _newton_system(2000)
    x = bridged.linear_solve(ptr, idx, val, rhs, tolerance=1e-7)
    assert np.max(np.abs(dense @ x - rhs)) <= 1e-7 * (1 + np.max(np.abs(rhs)))
