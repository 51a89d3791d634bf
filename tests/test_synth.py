"""The seeded workload generators and the benchmark's byte counts (CPU only).

The generators stand in for data: each instance must be a valid canonical CSR,
feasible at its planted point x0, and reproducible from its seed.  The byte
formulas are the numerators of the reported bandwidths."""
import sys
import pathlib

import numpy as np
import pytest

from niryukti_b200 import synth

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _canonical(m):
    assert m.ptr[0] == 0 and m.ptr[-1] == m.idx.size == m.val.size
    assert np.all(np.diff(m.ptr) >= 0)
    assert np.all((m.idx >= 0) & (m.idx < m.n))
    rows = np.repeat(np.arange(m.m), np.diff(m.ptr))
    key = rows * m.n + m.idx
    assert np.all(np.diff(key) > 0), "columns strictly increase within each row"
    assert np.all(m.val != 0) and np.all(np.isfinite(m.val))


def _feasible_at(m, x0, slack=1e-7):
    ax = synth.csr_matvec(m.ptr, m.idx, m.val, x0, m.m)
    scale = 1 + np.abs(ax)
    assert np.all(ax >= m.rl - slack * scale) and np.all(ax <= m.ru + slack * scale)
    assert np.all(x0 >= m.lb) and np.all(x0 <= m.ub)


def test_power_law_lp_shape_and_feasibility():
    m = synth.power_law_lp(m=20000, n=40000, nnz=400000, seed=3)
    _canonical(m)
    assert m.nnz == 400000
    lens = np.diff(m.ptr)
    assert lens.min() >= 2 and lens.max() <= 5000
    assert np.isinf(m.lb).mean() == pytest.approx(0.10, abs=0.01)  # free columns
    assert np.all(m.rl[: m.m // 2] == m.ru[: m.m // 2])             # equality half
    assert np.all(np.isinf(m.rl[m.m // 2:]))                         # <= half
    _feasible_at(m, m.x0)


def test_block_angular_lp_structure():
    blocks, rows_b, cols_b, link = 4, 500, 1000, 20
    m = synth.block_angular_lp(blocks=blocks, block_rows=rows_b, block_cols=cols_b,
                               linking_rows=link)
    _canonical(m)
    mb = blocks * rows_b
    assert m.m == mb + link and m.n == blocks * cols_b
    for r in range(0, mb, 97):  # block rows touch only their block's columns
        cols = m.idx[m.ptr[r]:m.ptr[r + 1]]
        assert np.all(cols // cols_b == r // rows_b)
    per_link = int(round(0.05 * m.n))
    assert np.all(np.diff(m.ptr)[mb:] == per_link)
    assert np.all(np.abs(m.val) >= 0.1) and np.all(np.abs(m.val) <= 2.0)
    assert np.all(np.isinf(m.rl[mb:])) and np.all(m.rl[:mb] == m.ru[:mb])
    # feasible at the point the rows were built from: inside the box [0, 20]
    assert np.all(m.lb == 0) and np.all(m.ub == 20)


def test_generators_are_reproducible():
    a = synth.power_law_lp(m=5000, n=10000, nnz=100000, seed=9)
    b = synth.power_law_lp(m=5000, n=10000, nnz=100000, seed=9)
    assert np.array_equal(a.idx, b.idx) and np.array_equal(a.val, b.val)
    c = synth.batch_instances(count=6, m_lo=50, m_hi=300, qp_frac=0.5, seed=4)
    d = synth.batch_instances(count=6, m_lo=50, m_hi=300, qp_frac=0.5, seed=4)
    for u, v in zip(c, d):
        assert np.array_equal(u.val, v.val) and np.array_equal(u.c, v.c)


def test_batch_instances_qp_terms_are_symmetric():
    for m in synth.batch_instances(count=8, m_lo=50, m_hi=300, qp_frac=0.5, seed=2):
        _canonical(m)
        _feasible_at(m, m.x0)
        assert m.n == 2 * m.m
        if m.qptr is None:
            continue
        q = np.zeros((m.n, m.n))
        rows = np.repeat(np.arange(m.n), np.diff(m.qptr))
        q[rows, m.qidx] = m.qval
        assert np.array_equal(q, q.T)
        assert np.all(np.linalg.eigvalsh(q) >= -1e-9)  # convex


def test_benchmark_byte_counts():
    sys.path.insert(0, str(ROOT))
    import bench
    m, n, nnz = 1_000_000, 2_000_000, 20_000_000
    # one SpMV: matrix once (8 B value + 4 B index), offsets, input and output vectors
    assert bench.spmv_bytes(m, n, nnz) == nnz * 12 + (m + 1) * 4 + n * 8 + m * 8
    assert bench.iteration_spmv_bytes(m, n, nnz) == 268_000_004 + 272_000_004
    primal, dual = bench.fused_kernel_bytes(m, n, nnz)
    assert primal == 384_000_004 and dual == 324_000_004  # an LP's q is not read
    primal_q, _ = bench.fused_kernel_bytes(m, n, nnz, diag_q=True)
    assert primal_q == primal + 8 * n
    assert bench.iteration_spmv_bytes(m, n, nnz, s_v=4) == 188_000_004 + 192_000_004


def test_reference_arm_json_contract():
    """`bench.py --impl reference` (CPU: the reference's own CpuBackend) prints
    one JSON line with the benchmark contract's keys, on the engine arm's
    metric and workload."""
    import json
    import subprocess
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--scale", "0.01", "--steps", "2", "--warmup", "3", "--no-ref-gpu",
                          "--ref-trials", "2"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    sys.path.insert(0, str(ROOT))
    import bench
    assert len(lines[0]) <= bench.HEADLINE_MAX_BYTES
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    sys.path.insert(0, str(ROOT))
    import bench
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "GB/s"
    assert d["steps"] == 2 and d["warmup"] == 3 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "power_law_lp_scaled_0.01" and d["value"] > 0
    assert set(d["cpu_baseline"]) >= {"value", "unit", "cores", "kind", "sample"}
    assert d["cpu_baseline"]["value"] == d["value"] == d["e2e"]["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == d["e2e"]["d2h_bytes_per_step"] == 0


def _fake_engine_line():
    """An engine-arm result with every key at its widest realistic value."""
    sample = [{"instance": k, "m": 50000, "nnz": 600000, "seconds": 12.345678, "status": s,
               "iterations": 100062, "objective_diff": 1.234e-9}
              for k, s in enumerate(["OPTIMAL", "ITERATION_LIMIT"] * 8)]
    line = {"metric": "SpMV HBM GB/s", "value": 2868.123456789, "unit": "GB/s", "n_gpus": 1,
            "steps": 20, "warmup": 5, "ms_per_step": 18.83123456789, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded power-law LP)",
            "config": {"workload": "power_law_lp_m1e6_n2e6_nnz2e7", "m": 1000000,
                       "n": 2000000, "nnz": 20000000, "trials_per_step": 100,
                       "precision": "fp64", "parallelism": "replicas1",
                       "l2": "inputs > L2"},
            "iterations_per_s": 5310.123456789,
            "roofline": {"bound": "hbm", "kernel": "dual_kernel", "achieved": 2830.123456789,
                         "peak": 6468.6, "unit": "GB/s", "frac": 0.4375123456789,
                         "traffic": 332480000.0, "traffic_source": "x" * 80,
                         "peak_source": "measured"},
            "cpu_baseline": {"value": 43.933106912192, "unit": "GB/s", "cores": 16,
                             "kind": "reference", "sample": "y" * 200,
                             "iterations_per_s": 81.357},
            "e2e": {"value": 2624.123456789, "unit": "GB/s", "h2d_bytes_per_step": 24000000,
                    "d2h_bytes_per_step": 48000000},
            "gpu_launches": 4000,
            "clocks": {"sm_mhz": 1927.0, "sm_max_mhz": 1965.0,
                       "reasons": ["sw_power_cap"], "samples": 1879}}
    solve = {name: {"gpu": {"status": "ITERATION_LIMIT", "seconds": 60.123456, "kkt": 2.0123e-2},
                    "reference_cpu": {"status": "TIME_LIMIT", "seconds": 32.3456, "kkt": 5.123}}
             for name in ("random_lp_m2000_n5000", "power_law_lp_m1e6_n2e6_nnz2e7")}
    batch = {"instances": 512, "precision": "mixed", "gpu_phase_s": 110.123456,
             "statuses": {"OPTIMAL": 312, "ITERATION_LIMIT": 199, "PRIMAL_INFEASIBLE": 1},
             "solves_per_s": 4.6543210, "optimal_per_s": 2.8345678,
             "speedup_optimal_vs_plain": 5.123456,
             "plain_fp64_one_by_one": {"sample": sample, "optimal_per_s": 0.4123456,
                                       "statuses": {"OPTIMAL": 10, "ITERATION_LIMIT": 6}},
             "per_instance": [[50000, 1, "OPT", 100062, 9999, 101.98]] * 512}
    return line, {"solve": solve, "batch": batch}


def test_headline_line_is_compact_and_complete():
    """The engine arm's last line stays short enough for a reader that keeps only
    the tail of the output, and still carries the contract's keys and the
    solve/batch summaries (the bulky sections go on earlier lines)."""
    import json
    sys.path.insert(0, str(ROOT))
    import bench
    line, sections = _fake_engine_line()
    h = bench.headline(line, sections)
    text = json.dumps(h)
    assert len(text) <= bench.HEADLINE_MAX_BYTES, len(text)
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert key in h, key
    assert set(h["roofline"]) >= {"bound", "achieved", "peak", "unit", "frac", "traffic"}
    assert set(h["cpu_baseline"]) >= {"value", "unit", "cores", "kind", "sample"}
    assert set(h["e2e"]) == {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"}
    assert h["value"] == pytest.approx(line["value"], rel=1e-5)
    assert h["batch_summary"]["statuses"]["OPT"] == 312
    assert "per_instance" not in text and "sample\": [" not in text
    assert json.loads(text) == h


def test_reference_arm_line_is_compact():
    sys.path.insert(0, str(ROOT))
    import bench
    line, _ = _fake_engine_line()
    ref = {k: line[k] for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup",
                                "ms_per_step", "higher_is_better", "scaling", "vs_baseline",
                                "dtype", "data", "config", "cpu_baseline", "e2e")}
    ref["reference_gpu"] = bench.compact_reference_gpu(
        {"trials": 2000, "seconds": 0.6865915209999969}, 1000000, 2000000, 20000000)
    ref["cpu_baseline"]["sample"] = ref["cpu_baseline"]["sample"][:110]
    import json
    assert len(json.dumps(ref)) <= bench.HEADLINE_MAX_BYTES
