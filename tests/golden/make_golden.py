"""Generate the golden fixtures in this folder from the reference itself.

Runs the reference's own CPU code (oracle/_ref/libvantage_ref.so, built from
the reference sources by oracle/Makefile) on small seeded instances and stores
inputs and outputs as .npz files.  The GPU box has no reference sources, so the
tests compare the engine (and the C oracle) against these files there.

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from niryukti_b200 import synth  # noqa: E402
from oracle.oracle import Reference  # noqa: E402


def model_arrays(m: synth.Model) -> dict:
    d = dict(m=m.m, n=m.n, ptr=m.ptr, idx=m.idx, val=m.val, c=m.c, q=m.q, lb=m.lb, ub=m.ub,
             rl=m.rl, ru=m.ru, offset=m.offset)
    if m.qnnz:
        d.update(qptr=m.qptr, qidx=m.qidx, qval=m.qval)
    return d


def model_from(d) -> synth.Model:
    q = {}
    if "qptr" in d:
        q = dict(qptr=d["qptr"], qidx=d["qidx"], qval=d["qval"])
    return synth.Model(m=int(d["m"]), n=int(d["n"]), ptr=d["ptr"], idx=d["idx"], val=d["val"],
                       c=d["c"], q=d["q"], lb=d["lb"], ub=d["ub"], rl=d["rl"], ru=d["ru"],
                       offset=float(d["offset"]), **q)


def small_lp(seed=11, m=60, n=150, per_col=3):
    return synth.random_lp(m=m, n=n, per_col=per_col, seed=seed)


def small_qp(seed=12, m=40):
    rng = np.random.default_rng(seed)
    return synth.batch_instance(rng, m, True, name="small_qp")


def skewed_lp(seed=13):
    # power-law rows up to 5000 entries: exercises warp- and CTA-per-row items
    return synth.power_law_lp(m=3000, n=6000, nnz=60000, seed=seed, len_hi=5000)


def record_steps(ref, model, name, chunks, count, tau, sigma, **kw):
    rm = ref.model(model)
    b = rm.backend(np.zeros(model.n), np.zeros(model.m), **kw)
    xs, ys, xas, yas, rej, prog = [], [], [], [], [], []
    for _ in range(chunks):
        prog.append(b.advance(count, tau, sigma))
        x, y, xa, ya = b.candidates()
        xs.append(x); ys.append(y); xas.append(xa); yas.append(ya)
        rej.append(b.rejected_steps())
    np.savez_compressed(HERE / f"{name}.npz", **model_arrays(model), x=np.array(xs),
                        y=np.array(ys), xa=np.array(xas), ya=np.array(yas),
                        rejected=np.array(rej), progress=np.array(prog), tau=tau, sigma=sigma,
                        count=count, options=json.dumps(kw))


def main():
    ref = Reference()
    lp = small_lp()
    record_steps(ref, lp, "steps_lp_adaptive", 6, 5, 0.5, 0.5, adaptive=True)
    record_steps(ref, lp, "steps_lp_fixed", 6, 5, 0.05, 0.05, adaptive=False)
    record_steps(ref, lp, "steps_lp_halpern", 6, 5, 0.05, 0.05, halpern=True, reflection=0.5,
                 restarts=True)
    record_steps(ref, small_qp(), "steps_qp", 6, 5, 0.05, 0.05, adaptive=False)
    record_steps(ref, skewed_lp(), "steps_skewed", 4, 5, 0.02, 0.02, adaptive=True)

    # a full reference solve of a small feasible LP
    sol = small_lp(seed=21, m=120, n=300, per_col=4)
    rm = ref.model(sol)
    r = rm.solve(method="pdhg", device="cpu", iteration_limit=200000)
    np.savez_compressed(HERE / "solve_small_lp.npz", **model_arrays(sol), x=r["x"], y=r["y"],
                        result=json.dumps({k: v for k, v in r.items() if k not in ("x", "y")}))

    # Verifier values on assorted points (LP and QP, safe and unsafe bound)
    rng = np.random.default_rng(5)
    cases = {}
    for tag, mod in (("lp", lp), ("qp", small_qp())):
        rmm = ref.model(mod)
        pts = []
        for k in range(4):
            x = np.clip(mod.x0 + 0.1 * k * rng.standard_normal(mod.n), mod.lb, mod.ub)
            y = rng.standard_normal(mod.m) * (0 if k == 0 else 1)
            for safe in (0, 1):
                acc = rmm.verify(x, y, safe)
                pts.append(np.concatenate([x, y, [safe], [acc[k2] for k2 in (
                    "objective", "primal", "dual", "gap", "kkt", "lower_bound")]]))
        cases[tag] = np.array(pts)
        np.savez_compressed(HERE / f"verify_{tag}.npz", **model_arrays(mod), points=cases[tag])
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
