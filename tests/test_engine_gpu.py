"""The B200 engine against the oracle, step by step (the reference's own parity
contract: tests/test_research.cpp:34-64,740-761,839-907; 1e-11 relative).

Each case runs the engine through its C ABI (niryukti_b200.engine) beside the
C oracle on the same inputs.  Where the engine's SpMV sums a row in a different
order than the CPU, agreement is to rounding (tolerances written per test)."""
import json
import math

import numpy as np
import pytest

from niryukti_b200 import synth
from tests.conftest import load_golden
from tests.test_oracle import halpern_expected, sparse_qp_model, tiny

pytestmark = pytest.mark.gpu


def step_sizes(model):
    """tau, sigma as solve_continuous starts them (src/solver.cpp:299-333)."""
    import bench
    return bench.step_sizes(model)


def near(a, b, tol=1e-11):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    err = np.abs(a - b) / (1 + np.abs(b))
    assert np.all(err <= tol), f"max rel err {err.max():.3e} > {tol}"


def advance_to(g, target, tau, sigma, done=0):
    """Run single trials until `target` accepted steps.  The CPU backend counts
    accepted iterations (retrying each up to 40 times, src/cpu.cpp:103-221); the
    CUDA backend counts trials (src/cuda.cu:849-866), so adaptive trajectories
    line up at equal accepted counts."""
    for _ in range(40 * max(1, target - done) + 40):
        if done >= target:
            return done
        done += g.advance(1, tau, sigma)
    raise AssertionError(f"no progress to {target} accepted steps")


def test_acceptance_parity(gpu, oracle):
    # tests/test_research.cpp:34-64
    m = tiny(1, 1, [(0, 0, 1.0)])
    m.c[:] = -1
    m.rl[:] = m.ru[:] = 3
    cpu = oracle.model(m).backend(np.zeros(1), np.zeros(1), adaptive=True)
    assert cpu.advance(1, 2, 2) == 1
    g = gpu.PdhgBackend(m, adaptive=True)
    accepted = 0
    for _ in range(40):
        if accepted:
            break
        accepted += g.advance(1, 2, 2)
    assert accepted == 1
    assert g.rejected_steps() == cpu.rejected_steps()
    for u, w in zip(g.candidates(), cpu.candidates()):
        near(u, w)


def test_halpern_scalar_recurrence(gpu):
    m = tiny(1, 1, [(0, 0, 1.0)])
    m.lb[:] = -math.inf
    m.ub[:] = math.inf
    m.rl[:] = m.ru[:] = 1
    g = gpu.PdhgBackend(m, halpern=True)
    for ex, ey, tx, ty in halpern_expected():
        g.advance(1, .5, .5)
        x, y, rx, ry = g.candidates()
        near(x[0], ex)
        near(y[0], ey)
        near(rx[0], tx)
        near(ry[0], ty)
    g.reset(np.array([2.0]), np.array([3.0]))
    g.advance(1, .5, .5)
    x, y, _, _ = g.candidates()
    near(x[0], 1.25)
    near(y[0], 2.5)


@pytest.mark.parametrize("reflection", [0.0, 1.0])
@pytest.mark.parametrize("graphs", [False, True])
def test_anchored_parity(gpu, oracle, reflection, graphs):
    # tests/test_research.cpp:864-891
    m = tiny(2, 2, [(0, 0, 1.0), (0, 1, 2.0), (1, 0, -1.0), (1, 1, 1.0)])
    m.c = np.array([1.0, -2.0])
    m.rl = np.array([-1.0, -2.0])
    m.ru = np.array([3.0, 2.0])
    cpu = oracle.model(m).backend(np.zeros(2), np.zeros(2), halpern=True, reflection=reflection)
    g = gpu.PdhgBackend(m, halpern=True, reflection=reflection, graphs=graphs, indices="32")
    for k in range(30):
        assert cpu.advance(1, .1, .1) == g.advance(1, .1, .1)
        c = cpu.candidates()
        d = g.candidates()
        for u, w in zip(d, c):
            near(u, w)
        if k == 14:
            cpu.reset(c[0], c[1])
            g.reset(d[0], d[1])


@pytest.mark.parametrize("width", ["32", "64"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_width_precision_parity(gpu, oracle, width, precision):
    # tests/test_research.cpp:892-907
    m = tiny(2, 2, [(0, 0, 1.0), (0, 1, 2.0), (1, 0, -1.0), (1, 1, 1.0)])
    m.c = np.array([1.0, -2.0])
    m.rl = np.array([-1.0, -2.0])
    m.ru = np.array([3.0, 2.0])
    cpu = oracle.model(m).backend(np.zeros(2), np.zeros(2))
    g = gpu.PdhgBackend(m, graphs=True, indices=width, precision=precision)
    cpu.advance(30, .1, .1)
    g.advance(30, .1, .1)
    mon = g.monitor()
    c, d = cpu.candidates(), g.candidates()
    near(d[0], c[0])
    near(d[1], c[1])
    # the KKT proxy against the FP64 host evaluation of the reference's formula
    # on the engine's own current and averaged points (src/cuda.cu:387-446,736)
    from oracle.monitor import monitor
    expected = monitor(m, *d)
    assert abs(mon - expected) <= 1e-12 * abs(expected), (mon, expected)


def test_resident_restart_and_snapshot(gpu):
    # tests/test_research.cpp:740-761
    lp = tiny(2, 1, [(0, 0, 1.0), (0, 1, 1.0)])
    lp.lb[:] = 0
    lp.ub[:] = 5
    lp.rl = np.array([3.0])
    lp.c = np.array([1.0, 2.0])
    r = gpu.PdhgBackend(lp)
    r.advance(20, .1, .1)
    rx, ry, ra, rb = r.candidates()
    state = r.snapshot()
    assert r.reset_candidate(True)
    r.advance(20, .1, .1)
    sx, sy, _, _ = r.candidates()
    r.restore(state)
    r.reset(ra, rb)
    r.advance(20, .1, .1)
    rx, ry, _, _ = r.candidates()
    near(rx, sx, 1e-12)
    near(ry, sy, 1e-12)


@pytest.mark.parametrize("name,tol", [("steps_lp_adaptive", 1e-10), ("steps_lp_fixed", 1e-10),
                                      ("steps_qp", 1e-10), ("steps_skewed", 1e-9)])
@pytest.mark.parametrize("graphs", [False, True])
def test_golden_step_parity(gpu, name, tol, graphs):
    """Engine vs the reference's own CPU trajectory (golden fixtures)."""
    model, d = load_golden(name)
    kw = json.loads(str(d["options"]))
    kw.pop("restarts", None)
    g = gpu.PdhgBackend(model, graphs=graphs, **kw)
    done = 0
    for k in range(len(d["progress"])):
        done = advance_to(g, done + int(d["progress"][k]), float(d["tau"]), float(d["sigma"]),
                          done)
        assert g.rejected_steps() == d["rejected"][k]
        x, y, xa, ya = g.candidates()
        near(x, d["x"][k], tol)
        near(y, d["y"][k], tol)
        near(xa, d["xa"][k], tol)
        near(ya, d["ya"][k], tol)


def test_golden_halpern_restart_request(gpu):
    model, d = load_golden("steps_lp_halpern")
    g = gpu.PdhgBackend(model, halpern=True, reflection=0.5, residual_restarts=True)
    for k in range(2):
        assert g.advance(5, float(d["tau"]), float(d["sigma"])) == d["progress"][k]
        x, y, xa, ya = g.candidates()
        near(x, d["x"][k], 1e-10)
        near(y, d["y"][k], 1e-10)
    # The tenth accepted step raises the restart request (the CPU then returns one
    # step per call, progress [5, 5, 1, ...]).  Like the reference CUDA backend
    # (src/cuda.cu:298-301), the device freezes every further trial until the
    # driver restarts.
    assert list(d["progress"][:3]) == [5, 5, 1]
    assert g.restart_requested()
    x0, y0, _, _ = g.candidates()
    assert g.advance(5, float(d["tau"]), float(d["sigma"])) == 0
    x1, y1, _, _ = g.candidates()
    assert np.array_equal(x0, x1) and np.array_equal(y0, y1)
    g.reset_candidate(True)
    assert not g.restart_requested()
    assert g.advance(5, float(d["tau"]), float(d["sigma"])) == 5


def test_sparse_qp_parity(gpu, oracle):
    m = sparse_qp_model()
    cpu = oracle.model(m).backend(np.zeros(2), np.zeros(1))
    g = gpu.PdhgBackend(m)
    for _ in range(10):
        assert cpu.advance(7, 0.3, 0.3) == g.advance(7, 0.3, 0.3)
        for u, w in zip(g.candidates(), cpu.candidates()):
            near(u, w)


@pytest.mark.parametrize("seed", [1, 2])
def test_random_lp_adaptive_parity(gpu, oracle, seed):
    """Adaptive steps on a power-law LP with rows of up to 6,000 entries and row
    scales over four decades.  Tolerance 1e-8 relative after 40 accepted steps:
    the device adds a long row's segments and the step rule's sums in a fixed
    tree, the CPU loop adds them one by one, and the adaptive step factor (a
    ratio of those sums) carries those last-bit differences from one step to
    the next."""
    m = synth.power_law_lp(m=4000, n=8000, nnz=80000, seed=seed, len_hi=6000)
    cpu = oracle.model(m).backend(np.zeros(m.n), np.zeros(m.m), adaptive=True)
    g = gpu.PdhgBackend(m, adaptive=True, graphs=True)
    done = 0
    for _ in range(4):
        done = advance_to(g, done + cpu.advance(10, 0.01, 0.01), 0.01, 0.01, done)
        assert g.rejected_steps() == cpu.rejected_steps()
        for u, w in zip(g.candidates(), cpu.candidates()):
            near(u, w, 1e-8)


def test_fp32_precision_tracks_fp64(gpu):
    """FP32 matrix values, FP32 gathers and accumulation; iterates stay FP64.
    Tolerance: 1e-4 relative to the FP64 engine after 40 fixed steps."""
    m = synth.random_lp(m=500, n=1200, per_col=4, seed=8)
    a = gpu.PdhgBackend(m, precision="fp64")
    b = gpu.PdhgBackend(m, precision="fp32")
    a.advance(40, 0.05, 0.05)
    b.advance(40, 0.05, 0.05)
    for u, w in zip(b.candidates(), a.candidates()):
        near(u, w, 1e-4)


def test_empty_and_degenerate_shapes(gpu, oracle):
    # no rows; a row without entries; an all-zero column
    m = tiny(3, 2, [(0, 0, 1.0), (0, 2, -2.0)])
    m.c = np.array([1.0, -1.0, 0.5])
    m.rl = np.array([-1.0, -math.inf])
    m.ru = np.array([2.0, math.inf])
    cpu = oracle.model(m).backend(np.zeros(3), np.zeros(2), adaptive=True)
    g = gpu.PdhgBackend(m, adaptive=True)
    done = 0
    for _ in range(5):
        done = advance_to(g, done + cpu.advance(3, 0.2, 0.2), 0.2, 0.2, done)
        assert g.rejected_steps() == cpu.rejected_steps()
        for u, w in zip(g.candidates(), cpu.candidates()):
            near(u, w)
    e = tiny(4, 0, [])
    e.c = np.array([1.0, -1.0, 0.0, 2.0])
    cpu = oracle.model(e).backend(np.zeros(4), np.zeros(0))
    g = gpu.PdhgBackend(e)
    assert cpu.advance(5, 0.5, 0.5) == g.advance(5, 0.5, 0.5)
    near(g.candidates()[0], cpu.candidates()[0])


def test_fixed_step_nonfinite_is_an_error(gpu):
    m = tiny(1, 1, [(0, 0, 1e300)])
    m.lb[:] = -math.inf
    m.ub[:] = math.inf
    m.c[:] = 1e300
    m.rl[:] = m.ru[:] = 1
    g = gpu.PdhgBackend(m)
    with pytest.raises(gpu.EngineError) as e:
        for _ in range(5):
            g.advance(10, 1e10, 1e10)
    assert "stalled or produced nonfinite" in str(e.value)


def test_very_long_rows_and_columns_parity(gpu, oracle):
    """A row of 20000 entries (split across chunks, combined through slots) and a
    dense column (a long row of A^T), against the oracle."""
    rng = np.random.default_rng(17)
    n, m = 20000, 300
    rows = [np.zeros(n, dtype=np.int64)]          # row 0: every column
    cols = [np.arange(n, dtype=np.int64)]
    for i in range(1, m):
        k = rng.integers(2, 12)
        rows.append(np.full(k, i, dtype=np.int64))
        cols.append(np.sort(rng.choice(n, k, replace=False)))
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    dense_col = 7                                   # column 7 in every row
    extra = np.arange(1, m)
    keep = ~np.isin(extra, r[c == dense_col])
    r = np.concatenate([r, extra[keep]])
    c = np.concatenate([c, np.full(keep.sum(), dense_col)])
    v = rng.standard_normal(r.size)
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=m), out=ptr[1:])
    x0 = rng.uniform(0, 1, n)
    model = synth.Model(m=m, n=n, ptr=ptr, idx=c, val=v, c=rng.standard_normal(n), q=np.zeros(n),
                        lb=np.zeros(n), ub=np.ones(n), rl=np.full(m, -np.inf), ru=np.zeros(m))
    model.ru = synth.csr_matvec(ptr, c, v, x0, m) + 0.5
    cpu = oracle.model(model).backend(np.zeros(n), np.zeros(m), adaptive=True)
    for graphs in (False, True):
        g = gpu.PdhgBackend(model, adaptive=True, graphs=graphs)
        done = 0
        c2 = oracle.model(model).backend(np.zeros(n), np.zeros(m), adaptive=True)
        for _ in range(3):
            done = advance_to(g, done + c2.advance(5, 0.001, 0.001), 0.001, 0.001, done)
            assert g.rejected_steps() == c2.rejected_steps()
            for u, w in zip(g.candidates(), c2.candidates()):
                near(u, w, 1e-9)


@pytest.mark.parametrize("seed", [1, 2])
def test_compact_csr_matches_host_compaction(gpu, seed):
    """cuda_compact_matrix on the GPU against the host restriction of the same
    CSR: kept rows in order, kept columns renumbered, entries in source order --
    bit-identical (an integer / byte operation).  Includes empty rows, rows of
    more than 32 entries and a dropped-everything row."""
    rng = np.random.default_rng(seed)
    m = synth.power_law_lp(m=3000, n=6000, nnz=60000, seed=seed, len_hi=2000)
    kept = np.sort(rng.choice(m.m, 2000, replace=False))
    keep_col = rng.random(m.n) < 0.7
    cmap = np.where(keep_col, np.cumsum(keep_col) - 1, -1)
    out_cols = int(keep_col.sum())
    ptr, idx, val = gpu.compact_csr(m.ptr, m.idx, m.val, m.n, kept, cmap, out_cols)
    want_ptr, want_idx, want_val = [0], [], []
    for i in kept:
        cols = m.idx[m.ptr[i]:m.ptr[i + 1]]
        vals = m.val[m.ptr[i]:m.ptr[i + 1]]
        sel = cmap[cols] >= 0
        want_idx.extend(cmap[cols[sel]].tolist())
        want_val.extend(vals[sel].tolist())
        want_ptr.append(len(want_idx))
    assert np.array_equal(ptr, want_ptr)
    assert np.array_equal(idx, want_idx)
    assert np.array_equal(val.view(np.int64), np.array(want_val).view(np.int64))


def test_compact_csr_rejects_bad_maps(gpu):
    m = synth.random_lp(m=50, n=80, per_col=3, seed=1)
    cmap = np.arange(m.n)
    with pytest.raises(gpu.EngineError, match="row map"):
        gpu.compact_csr(m.ptr, m.idx, m.val, m.n, [3, 2], cmap, m.n)
    bad = cmap.copy()
    bad[5] = 2  # not increasing
    with pytest.raises(gpu.EngineError, match="column map"):
        gpu.compact_csr(m.ptr, m.idx, m.val, m.n, [0, 1], bad, m.n)


def _propagation_case(seed):
    """A random sparse model with mixed-sign rows, equality and one-sided rows,
    free and boxed columns, and a random half of the columns integer."""
    rng = np.random.default_rng(seed)
    m = synth.random_lp(m=400, n=900, per_col=4, seed=seed)
    lb, ub = m.lb.copy(), m.ub.copy()
    free = rng.random(m.n) < 0.1
    lb[free], ub[free] = -np.inf, np.inf
    m.rl = np.where(rng.random(m.m) < 0.5, m.rl - 0.5, -np.inf)
    m.ru = m.ru + rng.uniform(0, 2, m.m)
    integer = (rng.random(m.n) < 0.5).astype(np.int32)
    return m, integer, lb, ub


@pytest.mark.parametrize("seed", [3, 4, 5])
@pytest.mark.parametrize("passes", [1, 5])
def test_propagate_bounds_matches_oracle(gpu, oracle, seed, passes):
    """cuda_propagate_integer_bounds on the GPU against the oracle's sequential
    restatement with the rounding mode switched per operation: bounds and the
    feasibility verdict bit-identical (each row's sums keep their order; the
    tightest proposal per column wins whatever the arrival order)."""
    m, integer, lb, ub = _propagation_case(seed)
    ok_g, lb_g, ub_g = gpu.propagate_bounds(m, integer, lb, ub, passes)
    ok_o, lb_o, ub_o = oracle.propagate_bounds(m, integer, lb, ub, passes)
    assert ok_g == ok_o
    assert np.array_equal(lb_g.view(np.int64), lb_o.view(np.int64))
    assert np.array_equal(ub_g.view(np.int64), ub_o.view(np.int64))
    assert np.sum(lb_g > lb) + np.sum(ub_g < ub) > 0  # something was tightened


def test_propagate_bounds_detects_infeasible_row(gpu, oracle):
    m, integer, lb, ub = _propagation_case(6)
    m.rl = m.rl.copy()
    m.rl[7] = 1e9  # no point in the box reaches it
    ok_g = gpu.propagate_bounds(m, integer, lb, ub, 3)[0]
    assert ok_g is False and oracle.propagate_bounds(m, integer, lb, ub, 3)[0] is False


def _newton_system(n, seed=11):
    """A nonsymmetric, diagonally dominant sparse system (CSR and dense)."""
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n), 6)
    cols = rng.integers(0, n, rows.size)
    vals = rng.standard_normal(rows.size)
    dense = np.zeros((n, n))
    np.add.at(dense, (rows, cols), vals)
    dense[np.arange(n), np.arange(n)] += 8 + np.abs(dense).sum(1)
    nz = dense != 0
    ptr = np.concatenate([[0], np.cumsum(nz.sum(1))]).astype(np.int64)
    idx = np.nonzero(nz)[1].astype(np.int64)
    return ptr, idx, dense[nz], dense, rng.standard_normal(n)


@pytest.mark.parametrize("fp32", [False, True])
def test_linear_solve_bicgstab(gpu, fp32):
    """cuda_linear_solve's BiCGSTAB on a nonsymmetric, diagonally dominant sparse
    system: converged, and the solution within the target the reference sets
    (1e-10 relative residual in FP64, 1e-6 with FP32 values) of the dense solve."""
    ptr, idx, val, dense, rhs = _newton_system(3000)
    x, ok = gpu.linear_solve(ptr, idx, val, rhs, fp32_matrix=fp32)
    assert ok
    want = np.linalg.solve(dense, rhs)
    tol = 1e-5 if fp32 else 1e-9
    assert np.max(np.abs(x - want)) <= tol * (1 + np.max(np.abs(want)))
    if not fp32:
        assert np.linalg.norm(dense @ x - rhs) <= 1e-10 * (1 + np.linalg.norm(rhs)) * 10


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32"])
def test_panel_path_multi_panel_parity(gpu, oracle, precision):
    """A's long rows by column panel (the dual SpMV's panel kernel) with more
    than one panel: 100,000 columns are several panels of the FP64 dx slice a
    CTA holds (two of the FP32 one).  Fixed steps against the oracle, 1e-10
    relative in FP64 over 60 trials: a long row is summed per panel in CSR
    order and the panel sums are added in panel order, where the CPU adds the
    whole row in CSR order.  With FP32 matrices the oracle gets the same
    FP32-rounded values (MIXED: FP64 gathers and sums, 1e-10) or the FP32
    engine is held to 1e-4 (FP32 gathers and sums)."""
    m = synth.power_law_lp(m=20000, n=100000, nnz=500000, seed=3, len_hi=5000)
    if precision != "fp64":
        m.val = m.val.astype(np.float32).astype(np.float64)
    g = gpu.PdhgBackend(m, graphs=True, precision=precision)
    info = g.layout_info()
    assert info["panels"] >= 2 and info["panel_rows"] > 0, info
    assert info["kernels_per_trial"] == 3
    cpu = oracle.model(m).backend(np.zeros(m.n), np.zeros(m.m))
    tol = 1e-4 if precision == "fp32" else 1e-10
    tau, sigma = step_sizes(m)
    for _ in range(3):
        assert cpu.advance(20, tau, sigma) == g.advance(20, tau, sigma)
        for u, w in zip(g.candidates(), cpu.candidates()):
            near(u, w, tol)


def test_panel_path_single_panel_runs(gpu, oracle):
    """With every column in one panel a long row's partials are its runs: its
    entries in CSR order, cut into pieces of 64 or more where one lane would
    otherwise carry far more than its share, each summed sequentially and then
    added in CSR order.  Rows of up to 3,000 entries on a 3,000-row LP are cut
    (more runs than long rows); fixed-step trajectories agree with the CPU's
    sequential row sums to 1e-12 over 50 trials."""
    m = synth.power_law_lp(m=3000, n=6000, nnz=60000, seed=4, len_hi=3000)
    g = gpu.PdhgBackend(m, graphs=True)
    info = g.layout_info()
    assert info["panels"] == 1 and info["panel_rows"] > 0, info
    assert info["panel_runs"] > info["panel_rows"], info
    cpu = oracle.model(m).backend(np.zeros(m.n), np.zeros(m.m))
    tau, sigma = step_sizes(m)
    assert cpu.advance(50, tau, sigma) == g.advance(50, tau, sigma)
    for u, w in zip(g.candidates(), cpu.candidates()):
        near(u, w, 1e-12)


def test_trajectory_parity_above_openmp_threshold(gpu, reference):
    """Step by step against the reference's own CpuBackend (oracle/_ref, all host
    threads) above its OpenMP threshold (10,000 rows or columns,
    src/cpu.cpp:105,123,134), where its step-rule sums are split over threads:
    a power-law LP of 50,000 x 100,000 with 1,000,000 nonzeros and rows of up to
    5,000 entries (several column panels on the device).  Adaptive steps,
    compared at equal accepted counts; tolerance 1e-8 relative after 40
    accepted steps, as for the oracle runs on smaller power-law LPs: both sides
    group the sums differently and the adaptive step factor carries the
    last-bit differences forward."""
    import os
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    m = synth.power_law_lp(m=50000, n=100000, nnz=1_000_000, seed=6, len_hi=5000)
    assert int(np.diff(m.ptr).max()) > 4000
    cpu = reference.model(m).backend(np.zeros(m.n), np.zeros(m.m), adaptive=True)
    g = gpu.PdhgBackend(m, adaptive=True, graphs=True)
    assert g.layout_info()["panels"] >= 2
    tau, sigma = step_sizes(m)
    done = 0
    for _ in range(4):
        done = advance_to(g, done + cpu.advance(10, tau, sigma), tau, sigma, done)
        assert g.rejected_steps() == cpu.rejected_steps()
        for u, w in zip(g.candidates(), cpu.candidates()):
            near(u, w, 1e-8)


@pytest.mark.parametrize("graphs", [False, True])
def test_profiled_trials_are_ordinary_trials(gpu, graphs):
    """nk_pdhg_profile_kernels times the kernels of real trials (with graphs on,
    replays of one captured trial whose events are graph nodes): its trials
    advance the iterate bit for bit as advance() does, and every kernel time is
    positive, the panel kernel's too on an LP with panels."""
    m = synth.power_law_lp(m=20000, n=100000, nnz=500000, seed=3, len_hi=5000)
    tau, sigma = step_sizes(m)
    a = gpu.PdhgBackend(m, adaptive=True, graphs=graphs)
    b = gpu.PdhgBackend(m, adaptive=True, graphs=graphs)
    assert a.layout_info()["panels"] >= 2
    primal, panel, dual = a.profile_kernels(30, tau, sigma)
    assert primal > 0 and panel > 0 and dual > 0
    b.advance(30, tau, sigma)
    for u, w in zip(a.candidates(), b.candidates()):
        assert np.array_equal(u, w)
