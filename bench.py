#!/usr/bin/env python
"""Benchmark of the PDHG hot path on the power-law LP (m=1e6, n=2e6, 20M nnz,
power-law rows), one B200.

A *step* is one check interval of the reference's driver: 100 PDHG trials
(IterationBackend::advance(100, tau, sigma), src/solver.cpp:524-526).  The
metric is the SpMV HBM bandwidth of those trials: the algorithmic bytes of the
two SpMVs of one PDHG iteration (A^T y and A dx,
nnz*(s_v+s_i) + (rows+1)*s_p + cols*8 + rows*8 each) times iterations per
second.  The instance (synthetic, seeded) is larger than L2 (about 730 MB of
traffic per iteration), so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl nk|reference]

Multi-GPU: a single LP is not partitioned (replicas only); each rank runs its
own replica and `value` is the sum over ranks of the work done in the max-over-
ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SpMV HBM GB/s"
TRIALS_PER_STEP = 100
# The result line is printed last and kept short: whoever reads the benchmark's
# output may keep only its tail.  Bulky sections (the batch's per-instance
# table, the solves, the precision forms) go on earlier lines of their own.
HEADLINE_MAX_BYTES = 1400


def emit(obj) -> None:
    print(json.dumps(obj), flush=True)


def sig(v, digits=4):
    """v rounded to `digits` significant digits (None, ints and strings pass)."""
    if not isinstance(v, float) or not math.isfinite(v) or v == 0:
        return v
    return round(v, max(0, digits - 1 - int(math.floor(math.log10(abs(v))))))


def status_counts(results):
    out = {}
    for r in results:
        out[r] = out.get(r, 0) + 1
    return out


def spmv_bytes(rows, cols, nnz, s_v=8, s_i=4, s_p=4):
    """Algorithmic bytes of one CSR SpMV: matrix once, input vector once, output once."""
    return nnz * (s_v + s_i) + (rows + 1) * s_p + cols * 8 + rows * 8


def iteration_spmv_bytes(m, n, nnz, s_v=8):
    return spmv_bytes(m, n, nnz, s_v) + spmv_bytes(n, m, nnz, s_v)


def fused_kernel_bytes(m, n, nnz, s_v=8, diag_q=False):
    """Algorithmic bytes of the two fused kernels of one trial.
    primal: A^T (nnz, n+1 ptr) + gather y (m) + read x, c, lb, ub, xa (and q when the model has
            a diagonal quadratic term; an LP's q is never read) + write trial, dx, xa (n)
    dual:   A (nnz, m+1 ptr) + gather dx (n) + read y, Ax, rl, ru, ya + write trial, Ax', ya (m)"""
    primal = nnz * (s_v + 4) + (n + 1) * 4 + m * 8 + (9 if diag_q else 8) * 8 * n
    dual = nnz * (s_v + 4) + (m + 1) * 4 + n * 8 + 8 * 8 * m
    return primal, dual


def step_sizes(model):
    """Step and primal weight exactly as solve_continuous initialises them
    (src/solver.cpp:299-333): step = 0.9/sqrt(max row l1 * max col l1),
    weight = clamp(||c|| / ||clamp(0, rl, ru)||, 1e-4, 1e4)."""
    a = np.abs(model.val)
    rows = np.add.reduceat(a, model.ptr[:-1]) if model.nnz else np.zeros(model.m)
    rows[np.diff(model.ptr) == 0] = 0
    cols = np.bincount(model.idx, weights=a, minlength=model.n)
    norm = math.sqrt(rows.max()) * math.sqrt(cols.max())
    step = 0.9 / norm if norm > 0 else 1.0
    c2 = float(np.dot(model.c, model.c))
    b = np.clip(0.0, model.rl, model.ru)
    b2 = float(np.dot(b, b))
    weight = min(1e4, max(1e-4, math.sqrt(c2 / b2))) if c2 > 1e-24 and b2 > 1e-24 else 1.0
    return step / weight, step * weight


class Clocks:
    """nvidia-smi sampling during the timed region (clocks and throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index=0):
        self.idx = device_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if getattr(self, "_summary", None) is not None:
            return self._summary
        if not self.file:
            return None
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        self._summary = {"sm_mhz": statistics.median(sm) if sm else None,
                         "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                         "samples": len(rows)}
        return self._summary


def max_over_ranks(value: float, dist=None, device: str = "cuda") -> float:
    """The slowest rank's time: every rank contributes its own CUDA-event time
    and all of them get the maximum (no-op on one process)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world: int, units_per_rank: float, ms_max: float) -> float:
    """Whole-job rate of independent replicas: the units all ranks processed
    over the max-over-ranks time (weak scaling)."""
    return world * units_per_rank / (ms_max / 1e3)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def build_model(args):
    """The power-law LP (m=1e6, n=2e6, nnz=2e7), or the same generator scaled by
    --scale (profiling captures use a smaller, still larger-than-L2 case)."""
    from niryukti_b200 import synth
    f = 0.1 if args.small else args.scale
    if f == 1.0:
        return synth.power_law_lp(seed=2)
    return synth.power_law_lp(m=int(1_000_000 * f), n=int(2_000_000 * f),
                              nnz=int(20_000_000 * f), seed=2)


def workload_name(args):
    f = 0.1 if args.small else args.scale
    return ("power_law_lp_m1e6_n2e6_nnz2e7" if f == 1.0 else
            f"power_law_lp_scaled_{f:g}")


# ---------------------------------------------------------------- CPU arm
def cpu_rate(model, seconds, threads, trials_per_sample):
    """The reference's CpuBackend (oracle/_ref, the reference's own code) when built,
    else the C oracle port: PDHG iterations/s on the same instance."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as orc
    kind = "reference" if orc.REF_SO.exists() else "port"
    if kind == "reference":
        be = orc.Reference().model(model).backend(np.zeros(model.n), np.zeros(model.m),
                                                  adaptive=True)
    else:
        be = orc.Oracle().model(model).backend(np.zeros(model.n), np.zeros(model.m),
                                               adaptive=True)
        threads = 1
    tau, sigma = step_sizes(model)
    be.advance(1, tau, sigma)  # warm caches
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        done += be.advance(trials_per_sample, tau, sigma)
    dt = time.perf_counter() - t0
    return done / dt, kind, threads, done, dt


def cpu_child(args):
    model = build_model(args)
    rate, kind, threads, done, dt = cpu_rate(model, args.cpu_seconds, args.cpu_threads,
                                            args.cpu_trials)
    print(json.dumps({"rate": rate, "kind": kind, "threads": threads, "done": done, "dt": dt}))


def run_cpu_child(args):
    cmd = [sys.executable, str(pathlib.Path(__file__).resolve()), "--cpu-child",
           "--cpu-seconds", str(args.cpu_seconds), "--cpu-threads", str(args.cpu_threads),
           "--cpu-trials", str(args.cpu_trials), "--scale", str(args.scale)] + \
        (["--small"] if args.small else [])
    env = dict(os.environ, OMP_NUM_THREADS=str(args.cpu_threads))
    out = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
    if out.returncode != 0:
        raise RuntimeError(out.stderr[-2000:])
    return json.loads(out.stdout.strip().splitlines()[-1])


def ref_gpu_child(args):
    """The reference's own CUDA backend (src/cuda.cu built for sm_100a by
    oracle/Makefile refcuda: cuSPARSE SpMVs, its trial kernels and graphs) on
    the same LP: wall-clock time of advance(100) chunks, each of which ends in
    the backend's own stream synchronisation."""
    from oracle import oracle as orc
    model = build_model(args)
    be = orc.Reference(orc.REF_CUDA_SO).model(model).backend(
        np.zeros(model.n), np.zeros(model.m), adaptive=True, device="cuda", graphs=True)
    tau, sigma = step_sizes(model)
    for _ in range(args.warmup):
        be.advance(TRIALS_PER_STEP, tau, sigma)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        be.advance(TRIALS_PER_STEP, tau, sigma)
    dt = time.perf_counter() - t0
    print(json.dumps({"trials": args.steps * TRIALS_PER_STEP, "seconds": dt}))


def reference_gpu(args, m, n, nnz):
    """The reference GPU backend's iteration rate on this LP, in a child process
    (None when its build is absent)."""
    from oracle import oracle as orc
    if not orc.REF_CUDA_SO.exists():
        return None
    cmd = [sys.executable, str(pathlib.Path(__file__).resolve()), "--ref-gpu-child",
           "--steps", str(args.steps), "--warmup", str(args.warmup), "--scale", str(args.scale)] + \
        (["--small"] if args.small else [])
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        if out.returncode != 0:
            return {"error": out.stderr[-200:]}
        r = json.loads(out.stdout.strip().splitlines()[-1])
    except Exception as exc:
        return {"error": str(exc)[-200:]}
    return compact_reference_gpu(r, m, n, nnz)


def compact_reference_gpu(r, m, n, nnz):
    it_s = r["trials"] / r["seconds"]
    return {"impl": "reference src/cuda.cu (cuSPARSE) for sm_100a", "iterations_per_s": sig(it_s),
            "spmv_GBps": sig(it_s * iteration_spmv_bytes(m, n, nnz) / 1e9),
            "timing": "wall clock, synchronising advance(100)", "trials": r["trials"],
            "seconds": sig(r["seconds"])}


def reference_arm(args, world, rank):
    if rank != 0:
        return
    model = build_model(args)
    m, n, nnz = model.m, model.n, model.nnz
    threads = args.cpu_threads
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as orc
    kind = "reference" if orc.REF_SO.exists() else "port"
    if kind == "reference":
        be = orc.Reference().model(model).backend(np.zeros(n), np.zeros(m), adaptive=True)
    else:
        be = orc.Oracle().model(model).backend(np.zeros(n), np.zeros(m), adaptive=True)
        threads = 1
    tau, sigma = step_sizes(model)
    per = args.ref_trials
    for _ in range(args.warmup):
        be.advance(per, tau, sigma)
    t0 = time.perf_counter()
    done = 0
    for _ in range(args.steps):
        done += be.advance(per, tau, sigma)
    dt = time.perf_counter() - t0
    rate = done / dt
    value = rate * iteration_spmv_bytes(m, n, nnz) / 1e9
    line = {"metric": METRIC, "value": value, "unit": "GB/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args), "m": m, "n": n,
                       "nnz": nnz, "trials_per_step": per, "seed": 2},
            "iterations_per_s": rate,
            "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": kind,
                             "sample": f"{args.steps} steps x {per} adaptive FP64 PDHG trials, "
                                       "CpuBackend::advance"},
            "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    if not args.no_ref_gpu:
        # beside the CPU arm: the reference's own CUDA build on the same LP, when built
        line["reference_gpu"] = reference_gpu(args, m, n, nnz)
    emit(line)


# ---------------------------------------------------------------- ingestion
def write_native_json(model, path):
    """The reference's native JSON model (read_json, src/io.cpp:84-142) of a
    minimisation LP, streamed row by row; infinite bounds as "inf" / "-inf"."""
    def num(v):
        v = float(v)
        return repr(v) if math.isfinite(v) else ('"inf"' if v > 0 else '"-inf"')

    with open(path, "w") as f:
        f.write('{"name":"%s","sense":"min","variables":[' % model.name)
        f.write(",".join('{"name":"x%d","lb":%s,"ub":%s}' % (j, num(lo), num(hi))
                         for j, (lo, hi) in enumerate(zip(model.lb, model.ub))))
        f.write('],"constraints":[')
        for i in range(model.m):
            s, e = int(model.ptr[i]), int(model.ptr[i + 1])
            coef = ",".join('"x%d":%r' % (j, v) for j, v in
                            zip(model.idx[s:e].tolist(), model.val[s:e].tolist()))
            f.write('%s{"name":"r%d","lb":%s,"ub":%s,"coefficients":{%s}}'
                    % ("," if i else "", i, num(model.rl[i]), num(model.ru[i]), coef))
        f.write('],"objective":{"linear":[%s],"offset":%r}}'
                % (",".join(map(repr, model.c.tolist())), float(model.offset)))


def model_file_timing(model, loads=3):
    """Writes `model` to a model file in a temporary folder and maps it back
    (memory map plus the header, size, checksum and CSR checks): seconds of the
    write and of the best of `loads` loads on a warm page cache."""
    from niryukti_b200 import modelfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "model.nkm")
        t = time.perf_counter()
        modelfile.save(model, path)
        out = {"save_s": time.perf_counter() - t, "file_mb": os.path.getsize(path) / 1e6}
        best = math.inf
        for _ in range(loads):
            t = time.perf_counter()
            back = modelfile.load(path)
            best = min(best, time.perf_counter() - t)
            del back
        out["load_s"] = best
    return out


def ingest_section(args):
    """Model ingestion of the power-law LP: written to a model file and loaded
    back (memory map plus the header, size, checksum and CSR checks), best of
    three loads on a warm page cache.  With --impl reference also the
    reference's own read_model (src/io.cpp:800-814) on the same model's native
    JSON, and whether it built exactly the arrays the model file holds."""
    from niryukti_b200 import modelfile
    model = build_model(args)
    out = {"workload": workload_name(args), "m": model.m, "n": model.n, "nnz": model.nnz,
           **model_file_timing(model)}
    if args.impl == "reference":
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "model.nkm")
            modelfile.save(model, path)
            from oracle import oracle as orc
            jpath = os.path.join(d, "model.json")
            t = time.perf_counter()
            write_native_json(model, jpath)
            out["json_write_s"] = time.perf_counter() - t
            out["json_mb"] = os.path.getsize(jpath) / 1e6
            t = time.perf_counter()
            ref = orc.Reference().read_model(jpath)
            out["reference_read_s"] = time.perf_counter() - t
            back = modelfile.load(path)
            out["identical"] = all(np.array_equal(getattr(ref, f), getattr(back, f))
                                   for f in ("ptr", "idx", "val", "c", "q", "lb", "ub", "rl",
                                             "ru"))
    print(json.dumps({"ingest": out}))


# ---------------------------------------------------------------- solves
def solve_models(args):
    from niryukti_b200 import synth
    c1 = synth.random_lp(m=2000, n=5000, per_col=5, seed=1)
    c2 = build_model(args)
    return {"random_lp_m2000_n5000": c1, workload_name(args): c2}


def reference_solve(model, budget, threads, iteration_limit=10**9):
    """The reference's own solve (vantage::solve, method pdhg, device cpu) from
    oracle/_ref, with its per-check verbose lines turned into times to each KKT
    decade; None when the reference build is absent."""
    from oracle import oracle as orc
    if not orc.REF_SO.exists():
        return None
    import re
    r, text = None, ""
    fd, path = tempfile.mkstemp(suffix=".log")
    saved = os.dup(2)
    try:
        os.dup2(fd, 2)  # the reference prints its check lines on stderr
        r = orc.Reference().model(model).solve(method="pdhg", device="cpu", verbose=True,
                                               time_limit=budget, threads=threads,
                                               iteration_limit=iteration_limit)
    finally:
        os.dup2(saved, 2)
        os.close(saved)
        os.close(fd)
        text = pathlib.Path(path).read_text()
        os.unlink(path)
    reached, best = {}, math.inf
    for mt in re.finditer(r"iter=(\d+).*?primal=(\S+) dual=(\S+) gap=(\S+) seconds=(\S+)", text):
        kkt = max(float(mt.group(2)), float(mt.group(3)), float(mt.group(4)))
        best = min(best, kkt)
        for k in range(9):
            if best <= 10.0 ** -k and f"1e-{k}" not in reached:
                reached[f"1e-{k}"] = float(mt.group(5))
    return {"status": r["status"], "seconds": r["seconds"], "iterations": r["iterations"],
            "kkt": r["kkt"], "objective": r["objective"], "time_to_kkt": reached,
            "preprocess_seconds": r["preprocess_seconds"], "threads": threads}


def solve_child(args):
    out = {}
    for name, model in solve_models(args).items():
        budget = args.cpu_solve_seconds if name.startswith("power_law_lp") else 300.0
        out[name] = reference_solve(model, budget, args.cpu_threads)
    print(json.dumps(out))


def solve_section(args):
    """Time to 1e-6 relative KKT through the public solve API (host model in,
    certified x, y out): the 2,000 x 5,000 LP to tolerance, the power-law LP within a budget, each
    beside the reference's own CPU solve of the same LP."""
    from niryukti_b200 import solver
    res = {}
    for name, model in solve_models(args).items():
        budget = args.solve_seconds if name.startswith("power_law_lp") else 300.0
        r = solver.solve(model, tol=1e-6, time_limit=budget, iteration_limit=10**9,
                         matrix_precision="fp64")
        res[name] = {"gpu": {k: r[k] for k in (
            "status", "seconds", "iterations", "kkt", "primal", "dual", "gap", "objective",
            "restarts", "preprocess_seconds", "transfer_seconds", "iteration_seconds",
            "verification_seconds", "device_checks", "host_checks", "time_to_kkt")}}
        res[name]["gpu"]["budget_s"] = budget
        # FP32 matrices first, then the closing FP64 refinement from the best
        # reduced-precision point; accuracy of both against the FP64 solve
        precs = ("mixed",) if name.startswith("power_law_lp") else ("mixed", "fp32")
        for prec in precs if not args.no_forms else ():
            q = solver.solve(model, tol=1e-6, time_limit=budget, iteration_limit=10**9,
                             matrix_precision=prec, refine=True)
            f64 = r["objective"]
            rel = (lambda v: abs(v - f64) / (1.0 + abs(f64)))
            res[name][f"gpu_{prec}"] = {k: q[k] for k in (
                "status", "seconds", "iterations", "phase_iterations", "refine_iterations",
                "phase_seconds", "kkt", "primal", "dual", "gap", "objective", "phase_kkt",
                "phase_objective", "time_to_kkt")}
            res[name][f"gpu_{prec}"].update(
                budget_s=budget, objective_rel_diff_vs_fp64=rel(q["objective"]),
                phase_objective_rel_diff_vs_fp64=rel(q["phase_objective"]))
    if not args.no_cpu:
        cmd = [sys.executable, str(pathlib.Path(__file__).resolve()), "--solve-child",
               "--cpu-threads", str(args.cpu_threads), "--cpu-solve-seconds",
               str(args.cpu_solve_seconds), "--scale", str(args.scale)] + \
            (["--small"] if args.small else [])
        env = dict(os.environ, OMP_NUM_THREADS=str(args.cpu_threads))
        try:
            out = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
            cpu = json.loads(out.stdout.strip().splitlines()[-1])
            for name in res:
                res[name]["reference_cpu"] = cpu.get(name)
        except Exception as exc:
            for name in res:
                res[name]["reference_cpu"] = {"error": str(exc)[-300:]}
    return res


# ---------------------------------------------------------------- KKT at equal iterations
CURVE_KEYS = ("status", "iterations", "kkt", "primal", "dual", "gap", "objective", "seconds",
              "preprocess_seconds")


def kkt_curve_child(args):
    """(child process) The reference's own solve of the power-law LP (vantage::solve,
    method pdhg, default options) capped at each of --curve-iters iterations:
    --curve-device cpu runs its CPU backend on --cpu-threads threads, cuda its
    CUDA build (src/cuda.cu for sm_100a, CUDA graphs on)."""
    from oracle import oracle as orc
    model = build_model(args)
    path = orc.REF_CUDA_SO if args.curve_device == "cuda" else orc.REF_SO
    ref = orc.Reference(path).model(model)
    out = []
    for cap in args.curve_iters:
        r = ref.solve(method="pdhg", device=args.curve_device, threads=args.cpu_threads,
                      iteration_limit=cap, time_limit=1e6,
                      cuda_graphs=args.curve_device == "cuda")
        out.append({"cap": cap, **{k: r[k] for k in CURVE_KEYS}})
    print(json.dumps(out))


def kkt_curve_section(args):
    """KKT reached at equal iteration counts on the power-law LP: the engine's
    device-resident solve (FP64), the reference's CPU solve and the reference's
    CUDA build, each stopped by the same iteration limit (the reference's
    default options otherwise: adaptive steps, restarts, checks every 100)."""
    from niryukti_b200 import solver
    model = build_model(args)
    out = {"workload": workload_name(args), "engine": []}
    for cap in args.curve_iters:
        r = solver.solve(model, tol=1e-6, time_limit=1e6, iteration_limit=cap,
                         matrix_precision="fp64")
        out["engine"].append({"cap": cap, **{k: r[k] for k in CURVE_KEYS}})
    from oracle import oracle as orc
    for dev, so in (("cuda", orc.REF_CUDA_SO), ("cpu", orc.REF_SO)):
        if args.no_cpu and dev == "cpu" or not so.exists():
            continue
        cmd = [sys.executable, str(pathlib.Path(__file__).resolve()), "--kkt-curve-child",
               "--curve-device", dev, "--cpu-threads", str(args.cpu_threads), "--scale",
               str(args.scale), "--curve-iters", *map(str, args.curve_iters)]
        env = dict(os.environ, OMP_NUM_THREADS=str(args.cpu_threads))
        try:
            res = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=3600)
            out[f"reference_{dev}"] = json.loads(res.stdout.strip().splitlines()[-1]) \
                if res.returncode == 0 else {"error": res.stderr[-500:]}
        except Exception as exc:
            out[f"reference_{dev}"] = {"error": str(exc)[-300:]}
    out["reference_cpu_threads"] = args.cpu_threads
    return out


# ---------------------------------------------------------------- batch (512 uneven LP/QP instances)
def batch_models(args):
    from niryukti_b200 import synth
    return synth.batch_instances(count=args.batch_count, m_lo=500, m_hi=args.batch_m_hi,
                                 qp_frac=0.2, seed=4)


def batch_section(args):
    """The batch: 512 uneven LP/QP instances (m log-uniform in [500, 50000],
    n = 2m, 20% QPs) solved to 1e-6 relative KKT by the batched engine
    (--batch-precision: FP64, or MIXED with FP32 matrices and FP64 iterates and
    reductions), beside the plain FP64 solve run instance by instance on the same
    GPU (a stratified sample, timed one by one) and the reference's CPU solve of
    the same sample."""
    from concurrent.futures import ThreadPoolExecutor
    from niryukti_b200 import batch as nb, solver
    t0 = time.perf_counter()
    models = batch_models(args)
    gen_s = time.perf_counter() - t0
    # the reference's default limits (100000 iterations; the time limit raised
    # from 60 s so that it never binds here), the same for both forms
    opts = dict(tol=1e-6, matrix_precision=args.batch_precision, iteration_limit=100000,
                time_limit=600)
    with nb.BatchEngine(**opts) as eng:
        w0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as pool:
            items = list(pool.map(eng.prepare, models))
        prep_s = time.perf_counter() - w0
        g0 = time.perf_counter()
        for k, it in enumerate(items):
            if not eng.admit(it, k):
                raise MemoryError("the 512-instance batch does not fit the device budget")
        info = eng.info()
        results, finish_t = {}, {}
        while len(results) < len(models):
            for k in eng.step(checks=1000000):
                results[k] = eng.result(k)
                finish_t[k] = time.perf_counter() - g0
        gpu_s = time.perf_counter() - g0
        phases = eng.phase_seconds()
    statuses = {}
    for r in results.values():
        statuses[r["status"]] = statuses.get(r["status"], 0) + 1
    iters = sorted(r["iterations"] for r in results.values())
    worst = max(r["kkt"] for r in results.values())
    # the plain FP64 single-instance solve on a stratified sample (by size)
    order = sorted(range(len(models)), key=lambda k: models[k].nnz)
    sample = [order[int(q * (len(order) - 1))] for q in np.linspace(0, 1, args.batch_sample)]
    plain = []
    for k in sample:
        p0 = time.perf_counter()
        r = solver.solve(models[k], tol=1e-6, iteration_limit=100000, time_limit=600)
        plain.append({"instance": k, "m": models[k].m, "nnz": models[k].nnz,
                      "seconds": time.perf_counter() - p0, "status": r["status"],
                      "iterations": r["iterations"],
                      "objective_diff": abs(r["objective"] - results[k]["objective"]) /
                      (1 + abs(r["objective"]))})
    # the sample sits at evenly spaced size quantiles, so its mean time per
    # instance times the instance count estimates the one-by-one total; its
    # share of OPTIMAL results estimates how many of them would be certified
    total_nnz = sum(m.nnz for m in models)
    plain_s = sum(p["seconds"] for p in plain) / len(plain) * len(models)
    plain_opt = sum(p["status"] == "OPTIMAL" for p in plain) / len(plain)
    n_opt = statuses.get("OPTIMAL", 0)
    out = {"workload": f"uneven_lp_qp_{len(models)}_m500_{args.batch_m_hi}",
           "instances": len(models), "qp": sum(1 for m in models if m.is_qp()),
           "total_nnz": total_nnz, "precision": args.batch_precision, "tol": 1e-6,
           "statuses": statuses, "worst_certified_kkt": worst,
           "iterations": {"min": iters[0], "median": iters[len(iters) // 2], "max": iters[-1]},
           "generate_s": gen_s, "prepare_s_parallel": prep_s, "gpu_phase_s": gpu_s,
           "solves_per_s": len(models) / gpu_s,
           "optimal_per_s": n_opt / gpu_s,
           "solves_per_s_with_prepare": len(models) / (gpu_s + prep_s),
           "kernel_variants": {"primal": info["primal_variant"], "dual": info["dual_variant"]},
           "check_interval_seconds": phases,
           "plain_fp64_one_by_one": {"sample": plain, "extrapolated_s": plain_s,
                                     "statuses": status_counts(p["status"] for p in plain),
                                     "solves_per_s": len(models) / plain_s,
                                     "optimal_per_s": plain_opt * len(models) / plain_s},
           "speedup_vs_plain": plain_s / gpu_s,
           "speedup_optimal_vs_plain": (n_opt / gpu_s) / (plain_opt * len(models) / plain_s)
           if plain_opt else None,
           # per instance: m, QP?, status, iterations, reduced-precision iterations,
           # seconds from admission to its result
           "per_instance": [[models[k].m, int(models[k].is_qp()), results[k]["status"][:3],
                             results[k]["iterations"], results[k]["phase_iterations"],
                             round(finish_t[k], 2)] for k in range(len(models))],
           "finished_by_time": {f"{q}%": sorted(finish_t.values())[
               min(len(finish_t) - 1, int(q / 100 * len(finish_t)))] for q in (50, 90, 99, 100)}}
    if not args.no_cpu:
        from oracle import oracle as orc
        if orc.REF_SO.exists():
            cpu = []
            for k in sample[: args.batch_cpu_sample]:
                r = reference_solve(models[k], args.cpu_solve_seconds, args.cpu_threads, 100000)
                cpu.append({"instance": k, "m": models[k].m, "seconds": r["seconds"],
                            "status": r["status"], "iterations": r["iterations"]})
            cpu_s = sum(c["seconds"] for c in cpu) / len(cpu) * len(models)
            out["reference_cpu_one_by_one"] = {"sample": cpu, "extrapolated_s": cpu_s,
                                               "solves_per_s": len(models) / cpu_s,
                                               "threads": args.cpu_threads}
    return out


def batch_throughput(args):
    """Trial throughput of the 512-instance batch (no solve): admit every
    instance, run one check interval (this also autotunes the kernels), then
    time --batch-trials PDHG trials of the whole batch with CUDA events."""
    from concurrent.futures import ThreadPoolExecutor
    from niryukti_b200 import batch as nb
    models = batch_models(args)
    with nb.BatchEngine(matrix_precision=args.batch_precision, iteration_limit=10**9,
                        time_limit=1e9) as eng:
        with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as pool:
            items = list(pool.map(eng.prepare, models))
        for k, it in enumerate(items):
            if not eng.admit(it, k):
                raise MemoryError("the 512-instance batch does not fit the device budget")
        eng.step(1)
        ms, bts = eng.time_trials(args.batch_trials)
        kp, kd = eng.kernel_times()
        info = eng.info()
    per = ms / max(1, args.batch_trials)
    return {"workload": f"uneven_lp_qp_{len(models)}", "precision": args.batch_precision,
            "trials": args.batch_trials, "ms_per_trial": per,
            "spmv_bytes_per_trial": bts, "spmv_GBps": bts / per / 1e6,
            "tuned_kernel_ms": {"batch_primal": kp, "batch_dual": kd},
            "variants": {"primal": info["primal_variant"], "dual": info["dual_variant"]}}


# ---------------------------------------------------------------- serving (Poisson stream)
def serve_section(args):
    """The served stream: Poisson arrivals at --serve-rate requests/s for --serve-seconds,
    each request drawn from a pool of instances of the uneven LP/QP mix with m
    log-uniform in [500, 200000]; served by continuous batching at
    --serve-precision (admission by device-memory footprint under a 150 GB
    budget), and by the plain FP64
    solve one request at a time on the same arrival stream.  Reported over the
    arrival window plus a drain of --serve-drain seconds: completed solves per
    second and the latency percentiles of the completed requests; requests
    still open at the end are counted, not timed."""
    from niryukti_b200 import serve, solver
    pool = synth_pool(args)
    rng = np.random.default_rng(6)
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / args.serve_rate)
        if t >= args.serve_seconds:
            break
        arrivals.append(t)
    picks = rng.integers(0, len(pool), len(arrivals))
    horizon = args.serve_seconds + args.serve_drain

    def summary(lat, done, t_total):
        lat = sorted(lat)
        pct = (lambda q: lat[min(len(lat) - 1, int(q * len(lat)))] if lat else None)
        return {"offered": len(arrivals), "completed": done, "open_at_end": len(arrivals) - done,
                "solves_per_s": done / t_total, "p50_s": pct(.5), "p95_s": pct(.95),
                "p99_s": pct(.99)}

    # served: a feeder submits at the arrival times
    svc = serve.SolveService(memory_budget=150e9, matrix_precision=args.serve_precision,
                             prepare_workers=os.cpu_count() or 8,
                             iteration_limit=100000, time_limit=horizon,
                             max_active_nnz=int(args.serve_active_nnz))
    lat, statuses = [], {}
    futs = []
    t0 = time.perf_counter()
    for a, k in zip(arrivals, picks):
        delay = t0 + a - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        f = svc.submit(pool[int(k)])
        f.arrival = a
        futs.append(f)
    deadline = t0 + horizon
    for f in futs:
        left = deadline - time.perf_counter()
        if left <= 0:
            break
        try:
            r = f.result(timeout=left)
        except Exception:
            continue
        statuses[r["status"]] = statuses.get(r["status"], 0) + 1
        lat.append(r["latency_s"])
    done_served = len(lat)
    served = summary(lat, done_served, horizon)
    served["statuses"] = statuses
    served["engine"] = {k: v for k, v in svc.stats().items() if k != "budget_bytes"}
    svc.close()
    # plain FP64, one request at a time, first come first served
    lat, clock, done = [], 0.0, 0
    t0 = time.perf_counter()
    for a, k in zip(arrivals, picks):
        now = time.perf_counter() - t0
        if now < a:
            time.sleep(a - now)
        now = time.perf_counter() - t0
        if now >= horizon:
            break
        r = solver.solve(pool[int(k)], tol=1e-6, iteration_limit=100000,
                         time_limit=max(1e-3, horizon - now))
        end = time.perf_counter() - t0
        if end <= horizon:
            lat.append(end - a)
            done += 1
    plain = summary(lat, done, horizon)
    return {"workload": f"poisson_{args.serve_rate:g}_per_s_{args.serve_seconds:g}s_"
                        f"m500_200000", "pool": len(pool), "window_s": horizon,
            "served_continuous_batching": served, "plain_fp64_one_at_a_time": plain}


def synth_pool(args):
    from niryukti_b200 import synth
    return synth.batch_instances(count=args.serve_pool, m_lo=500, m_hi=200000, qp_frac=0.2,
                                 seed=5)


# ---------------------------------------------------------------- engine arm
S_V = {"fp64": 8, "mixed": 4, "fp32": 4}
# DRAM bytes (read + write) per launch of each step of the power-law LP at
# scale 0.5 from one ncu capture of the current kernels
# (profiles/fused_pdhg_kernels_power_law_lp_half_scale.md); on this LP the dual
# step is the dual kernel alone (its long rows average fewer than 32 entries
# per column panel, so they take no panel kernel)
HALF_SCALE_TRAFFIC = {"primal_kernel": 168.526e6 + 5.193e6, "dual_step": 162.280e6 + 4.179e6}


def step_kernels(g, model, s_v, trials, tau, sigma):
    """CUDA-event durations of a trial's steps over `trials` single trials: the
    primal kernel, and the dual step (the panel kernel, when A's long rows are
    stored by column panel, plus the dual kernel), each with the algorithmic
    bytes of fused_kernel_bytes."""
    bp, bd = fused_kernel_bytes(model.m, model.n, model.nnz, s_v, diag_q=bool(np.any(model.q)))
    ms_p, ms_k, ms_d = g.profile_kernels(trials, tau, sigma)
    return {"primal_kernel": {"ms": ms_p, "bytes": bp, "GBps": bp / ms_p / 1e6},
            "dual_step": {"ms": ms_k + ms_d, "bytes": bd, "GBps": bd / (ms_k + ms_d) / 1e6,
                          "panel_kernel_ms": ms_k, "dual_kernel_ms": ms_d}}


def time_form(model, precision, steps, warmup, profile_trials):
    """Iteration rate of one precision form of the engine on `model`: CUDA
    events on the engine's stream around `steps` check intervals of 100 trials
    after `warmup` untimed ones, then per-kernel event timings.  SpMV bytes
    count matrix values at the form's width (8 B FP64, 4 B FP32)."""
    import torch
    from niryukti_b200 import engine
    m, n, nnz = model.m, model.n, model.nnz
    tau, sigma = step_sizes(model)
    g = engine.PdhgBackend(model, adaptive=True, graphs=True, precision=precision)
    try:
        ext = torch.cuda.ExternalStream(g.stream())
        for _ in range(warmup):
            g.advance(TRIALS_PER_STEP, tau, sigma)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(steps):
            g.advance(TRIALS_PER_STEP, tau, sigma)
        e1.record(ext)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        it_s = steps * TRIALS_PER_STEP / (ms / 1e3)
        s_v = S_V[precision]
        kernels = step_kernels(g, model, s_v, profile_trials, tau, sigma)
        bp, bd = kernels["primal_kernel"]["bytes"], kernels["dual_step"]["bytes"]
        return {"matrix_precision": precision, "iterations_per_s": it_s,
                "ms_per_iteration": 1e3 / it_s,
                "spmv_GBps": it_s * iteration_spmv_bytes(m, n, nnz, s_v) / 1e9,
                "whole_iteration_GBps": it_s * (bp + bd) / 1e9,
                "kernels": kernels, "layout": g.layout_info()}
    finally:
        del g
        torch.cuda.synchronize()


def block_angular_section(args):
    """The block-angular planning LP (64 blocks of 20,000 x 40,000
    with 6 nonzeros per column, 2,000 linking rows over 5% of all columns
    each), iteration rate in FP64 and with FP32 matrices."""
    import torch
    from niryukti_b200 import synth
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    model = synth.block_angular_lp(blocks=args.block_angular_blocks)
    gen_s = time.perf_counter() - t0
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = float(peaks.get("hbm_gbs", 6650.0))
    out = {"workload": f"block_angular_b{args.block_angular_blocks}_20000x40000_link2000",
           "m": model.m, "n": model.n, "nnz": model.nnz, "generate_s": gen_s,
           "peak_GBps": peak, "forms": {}}
    for prec in ("fp64", "mixed"):
        r = time_form(model, prec, args.steps, args.warmup, args.profile_trials)
        r["spmv_frac_of_measured_peak"] = r["spmv_GBps"] / peak
        r["whole_iteration_frac"] = r["whole_iteration_GBps"] / peak
        out["forms"][prec] = r
    return out


def engine_arm(args, world, rank, local):
    import torch
    from niryukti_b200 import engine

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    model = build_model(args)
    m, n, nnz = model.m, model.n, model.nnz
    tau, sigma = step_sizes(model)
    g = engine.PdhgBackend(model, adaptive=True, graphs=True, precision=args.precision)
    sched = g.schedule_info()
    ext = torch.cuda.ExternalStream(g.stream())
    s_v = 8 if args.precision == "fp64" else 4

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        g.advance(TRIALS_PER_STEP, tau, sigma)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local)
    with clocks:
        e0.record(ext)
        accepted = 0
        for _ in range(args.steps):
            accepted += g.advance(TRIALS_PER_STEP, tau, sigma)
        e1.record(ext)
        e1.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    trials = args.steps * TRIALS_PER_STEP
    it_s = trials / (ms / 1e3)
    value = replica_rate(world, trials, ms) * iteration_spmv_bytes(m, n, nnz, s_v) / 1e9

    # per-kernel durations (CUDA events around each kernel, same stream)
    layout = g.layout_info()
    kernels = step_kernels(g, model, s_v, args.profile_trials, tau, sigma)
    bp, bd = kernels["primal_kernel"]["bytes"], kernels["dual_step"]["bytes"]
    top = max(kernels, key=lambda k: kernels[k]["ms"])
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    peak = float(peaks.get("hbm_gbs", 6650.0))
    traffic, traffic_source = args.traffic, "--traffic" if args.traffic else None
    if traffic is None and args.precision == "fp64" and not args.small and args.scale == 1.0 \
            and top in HALF_SCALE_TRAFFIC:
        # DRAM bytes per launch from the ncu capture of the power-law LP at half
        # size (read + write, summed over the step's kernels), scaled by 2: every
        # unit (nonzeros, rows, columns) doubles
        traffic = 2 * HALF_SCALE_TRAFFIC[top]
        traffic_source = "ncu dram__bytes_read.sum + dram__bytes_write.sum at scale 0.5, x2"
    roofline = {"bound": "hbm", "kernel": top, "achieved": kernels[top]["GBps"], "peak": peak,
                "unit": "GB/s", "frac": kernels[top]["GBps"] / peak, "traffic": traffic,
                "traffic_source": traffic_source,
                "peak_source": "measured" if pk.exists() else "fallback"}

    # e2e through the C ABI with host buffers: per step upload (x, y), 100 trials,
    # download the four candidates -- the reference driver's per-check pattern
    hx = torch.zeros(n, dtype=torch.float64).pin_memory()
    hy = torch.zeros(m, dtype=torch.float64).pin_memory()
    outs = [torch.empty(k, dtype=torch.float64).pin_memory() for k in (n, m, n, m)]
    hxn, hyn = hx.numpy(), hy.numpy()
    on = [o.numpy() for o in outs]
    g.candidates(out=on)
    hxn[:] = on[0]
    hyn[:] = on[1]
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(ext)
    w0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        g.reset(hxn, hyn)
        g.advance(TRIALS_PER_STEP, tau, sigma)
        g.candidates(out=on)  # straight into the pinned host buffers
    f1.record(ext)
    f1.synchronize()
    wall = time.perf_counter() - w0
    e2e_ms = max_over_ranks(max(f0.elapsed_time(f1), 1e3 * wall), dist)
    e2e_value = replica_rate(world, args.e2e_steps * TRIALS_PER_STEP, e2e_ms) * \
        iteration_spmv_bytes(m, n, nnz, s_v) / 1e9

    del g
    forms = {}
    if not args.no_forms:
        # the same LP with FP32 matrices: MIXED (FP64 gathers and sums) and FP32
        # (FP32 gathers and sums); iterates, averages and reductions stay FP64
        for prec in ("mixed", "fp32"):
            if prec != args.precision:
                forms[prec] = time_form(model, prec, args.steps, args.warmup, args.profile_trials)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu:
        try:
            c = run_cpu_child(args)
            cpu = {"value": c["rate"] * iteration_spmv_bytes(m, n, nnz) / 1e9, "unit": "GB/s",
                   "cores": c["threads"], "kind": c["kind"],
                   "sample": f"{c['done']} adaptive FP64 PDHG trials in {c['dt']:.1f} s "
                             f"(CpuBackend::advance, {c['threads']} threads)",
                   "iterations_per_s": c["rate"]}
        except Exception as exc:  # reported, never silently replaced
            cpu = {"error": str(exc)[-500:]}
    clock_summary = clocks.summary()
    e2e = {"value": e2e_value, "unit": "GB/s",
           "h2d_bytes_per_step": 8 * (n + m), "d2h_bytes_per_step": 16 * (n + m)}
    line = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32-matrix/f64-iterates",
            "data": "synthetic (seeded power-law LP)",
            "config": {"workload": workload_name(args), "m": m, "n": n, "nnz": nnz,
                       "trials_per_step": TRIALS_PER_STEP, "precision": args.precision,
                       "parallelism": f"replicas{world}", "l2": "inputs > L2"},
            "iterations_per_s": it_s, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": layout["kernels_per_trial"] * (args.steps * TRIALS_PER_STEP),
            "clocks": clock_summary}
    # the detail first, one section per line; the compact result line last
    emit({"section": "iteration", "workload": workload_name(args),
          "iterations_per_s": it_s, "whole_iteration_GBps": it_s * (bp + bd) / 1e9,
          "kernels": kernels, "schedule": sched, "layout": layout, "roofline": roofline,
          "cpu_baseline": cpu,
          "e2e": dict(e2e, path="nk_pdhg_reset + nk_pdhg_advance(100) + nk_pdhg_candidates"),
          "accepted_trials": accepted, "clocks": clock_summary})
    if forms:
        emit({"section": "precision_forms", **forms})
    if not args.no_ingest:
        # this host's model-file write and load of the same LP (CPU only)
        try:
            emit({"section": "model_file", **model_file_timing(model)})
        except Exception as exc:  # reported, never raised: the result line comes last
            emit({"section": "model_file", "error": str(exc)[-300:]})
    sections = {}
    for name, run in (("solve", solve_section), ("batch", batch_section)):
        if getattr(args, f"no_{name}") or world != 1:
            continue
        try:
            sections[name] = run(args)
            emit({"section": name, **sections[name]})
        except Exception as exc:  # reported; the result line still comes last
            emit({"section": name, "error": repr(exc)[-500:]})
    emit(headline(line, sections))
    if dist:
        dist.destroy_process_group()


def headline(line, sections):
    """The result line: the benchmark contract's keys with compact values, plus
    one-line summaries of the time-to-tolerance solves and of the batch (no
    arrays; the full sections are printed on the lines before it)."""
    out = dict(line)
    for k in ("value", "ms_per_step", "iterations_per_s"):
        out[k] = sig(out[k], 6)
    out["roofline"] = {k: sig(v, 5) for k, v in line["roofline"].items()
                       if k not in ("traffic_source",)}
    cpu = line.get("cpu_baseline")
    if cpu and "error" not in cpu:
        out["cpu_baseline"] = {"value": sig(cpu["value"]), "unit": cpu["unit"],
                               "cores": cpu["cores"], "kind": cpu["kind"],
                               "sample": cpu["sample"][:80]}
    elif cpu:
        out["cpu_baseline"] = {"error": cpu["error"][-120:]}
    out["e2e"] = {k: sig(v) for k, v in line["e2e"].items()}
    ck = line.get("clocks")
    if ck:
        out["clocks"] = {"sm_mhz": ck.get("sm_mhz"), "sm_max_mhz": ck.get("sm_max_mhz"),
                         "reasons": ck.get("reasons")}
    solve = sections.get("solve")
    if solve:
        # per solved LP: status, seconds and KKT reached on the GPU, and the
        # reference CPU solve's seconds and KKT
        tt = {}
        for name, r in solve.items():
            g = r["gpu"]
            ref = r.get("reference_cpu") or {}
            tt[name.split("_m")[0]] = [g["status"][:3], sig(g["seconds"], 3), sig(g["kkt"], 2),
                                       sig(ref.get("seconds"), 3), sig(ref.get("kkt"), 2)]
        out["time_to_tol"] = tt
    b = sections.get("batch")
    if b:
        p = b["plain_fp64_one_by_one"]
        out["batch_summary"] = {
            "instances": b["instances"], "precision": b["precision"],
            "statuses": {k[:3]: v for k, v in b["statuses"].items()},
            "solves_per_s": sig(b["solves_per_s"]), "opt_per_s": sig(b["optimal_per_s"]),
            "plain_statuses": {k[:3]: v for k, v in p["statuses"].items()},
            "plain_opt_per_s": sig(p["optimal_per_s"]),
            "speedup_opt": sig(b["speedup_optimal_vs_plain"], 3)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="nk", choices=["nk", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed", "fp32"])
    ap.add_argument("--small", action="store_true", help="10x smaller instance (testing)")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="scale m, n and nnz of the power-law generator (profiling cases)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--ref-gpu-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="--impl reference: skip the reference's own CUDA backend on the same LP")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--cpu-threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--cpu-trials", type=int, default=5)
    ap.add_argument("--ref-trials", type=int, default=10)
    ap.add_argument("--profile-trials", type=int, default=20)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-solve", action="store_true", help="skip the time-to-tolerance solves")
    ap.add_argument("--solve-seconds", type=float, default=60.0,
                    help="time budget of the power-law LP solve on the GPU")
    ap.add_argument("--cpu-solve-seconds", type=float, default=30.0,
                    help="time budget of the reference's CPU solve of the power-law LP")
    ap.add_argument("--solve-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-instance batched solves")
    ap.add_argument("--batch-only", action="store_true",
                    help="print only the 512-instance batched-solve section")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--batch-trials", type=int, default=0,
                    help="with --batch-only: time this many batch trials instead of solving")
    ap.add_argument("--serve", action="store_true",
                    help="print only the served-stream section")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-drain", type=float, default=60.0)
    ap.add_argument("--serve-pool", type=int, default=64)
    ap.add_argument("--serve-active-nnz", type=float, default=16e6,
                    help="work cap of the running batch (nonzeros)")
    ap.add_argument("--batch-m-hi", type=int, default=50000)
    ap.add_argument("--batch-sample", type=int, default=16)
    ap.add_argument("--batch-precision", default="fp64", choices=["fp64", "mixed"],
                    help="matrix precision of the batch")
    ap.add_argument("--serve-precision", default="mixed", choices=["fp64", "mixed"],
                    help="matrix precision of the served stream")
    ap.add_argument("--batch-cpu-sample", type=int, default=4,
                    help="smallest sampled instances also solved by the reference on the CPU")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the FP32-matrix forms of the power-law LP iteration rate")
    ap.add_argument("--block-angular", action="store_true",
                    help="print only the block-angular LP iteration-rate section")
    ap.add_argument("--block-angular-blocks", type=int, default=64)
    ap.add_argument("--no-ingest", action="store_true",
                    help="skip the model-file write/load timing in the default line")
    ap.add_argument("--ingest", action="store_true",
                    help="time model-file ingestion (and, with --impl reference, the "
                         "reference's JSON reader on the same model); CPU only")
    ap.add_argument("--kkt-curve", action="store_true",
                    help="print only the KKT reached at equal iteration counts (engine, "
                         "reference CPU, reference CUDA build) on the power-law LP")
    ap.add_argument("--kkt-curve-child", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--curve-device", default="cpu", choices=["cpu", "cuda"],
                    help=argparse.SUPPRESS)
    ap.add_argument("--curve-iters", type=int, nargs="+", default=[2000, 10000])
    ap.add_argument("--traffic", type=float, default=None,
                    help="DRAM bytes per launch of the top kernel from an ncu capture")
    args = ap.parse_args()
    if args.warmup < 3 and not (args.cpu_child or args.solve_child or args.kkt_curve_child):
        ap.error("--warmup must be at least 3")
    if args.cpu_child:
        return cpu_child(args)
    if args.ref_gpu_child:
        return ref_gpu_child(args)
    if args.solve_child:
        return solve_child(args)
    if args.kkt_curve_child:
        return kkt_curve_child(args)
    if args.kkt_curve:
        print(json.dumps({"kkt_curve": kkt_curve_section(args)}))
        return
    if args.batch_only:
        print(json.dumps({"batch": batch_throughput(args) if args.batch_trials
                          else batch_section(args)}))
        return
    if args.serve:
        print(json.dumps({"serve": serve_section(args)}))
        return
    if args.block_angular:
        print(json.dumps({"block_angular": block_angular_section(args)}))
        return
    if args.ingest:
        return ingest_section(args)
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return reference_arm(args, world, rank)
    return engine_arm(args, world, rank, local)


if __name__ == "__main__":
    main()
