"""The engine's KKT proxy (IterationBackend::monitor, src/cuda.cu:387-446,
661-738) against an FP64 host evaluation of the reference's formula
(oracle/monitor.py), on an LP and on a QP with a sparse Q, and that host
evaluation against the reference's own CUDA build where it is present.

Tolerance: 1e-12 relative.  The device and the host compute the same
per-entry terms; they differ only in the order of the SpMV sums (A x, A^T y,
Q x) and of the objective and complementarity sums, which the host adds
exactly (math.fsum)."""
import numpy as np
import pytest

from niryukti_b200 import synth
from oracle.monitor import monitor, monitor_point

pytestmark = pytest.mark.gpu

TOL = 1e-12


def close(got, expected, tol=TOL):
    assert np.isfinite(expected) and expected > 0
    assert abs(got - expected) <= tol * abs(expected), (got, expected)


def lp_with_diagonal_q():
    model = synth.random_lp(m=3000, n=7000, per_col=5, seed=13)
    model.q = np.where(np.arange(model.n) % 7 == 0, 0.5, 0.0)
    return model


def qp_with_sparse_q():
    model = synth.batch_instance(np.random.default_rng(21), 1500, qp=True, name="qp")
    assert model.qnnz > 0
    return model


@pytest.mark.parametrize("make", [lp_with_diagonal_q, qp_with_sparse_q], ids=["lp", "qp"])
@pytest.mark.parametrize("trials", [1, 300])
def test_engine_monitor_matches_host_formula(gpu, make, trials):
    model = make()
    g = gpu.PdhgBackend(model, adaptive=True, graphs=True)
    g.advance(trials, 0.05, 0.05)
    got = g.monitor()
    x, y, xa, ya = g.candidates()
    close(got, monitor(model, x, y, xa, ya))
    # both points separately: the current one and the average
    assert min(monitor_point(model, x, y), monitor_point(model, xa, ya)) == \
        monitor(model, x, y, xa, ya)


REF_CHILD = """
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from tests.test_monitor_gpu import lp_with_diagonal_q, qp_with_sparse_q
from oracle.oracle import REF_CUDA_SO, Reference
model = {"lp": lp_with_diagonal_q, "qp": qp_with_sparse_q}[sys.argv[2]]()
be = Reference(REF_CUDA_SO).model(model).backend(np.zeros(model.n), np.zeros(model.m),
                                                 adaptive=True, device="cuda")
be.advance(200, 0.05, 0.05)
mon = be.monitor()
x, y, xa, ya = be.candidates()
np.savez(sys.argv[3], monitor=mon, x=x, y=y, xa=xa, ya=ya)
"""


@pytest.mark.parametrize("kind", ["lp", "qp"])
def test_host_formula_matches_reference_cuda_monitor(kind, tmp_path):
    """Pins the host restatement to the reference itself: its CudaBackend
    (src/cuda.cu built for sm_100a, cuSPARSE SpMVs) monitors its own iterates,
    in a child process of its own."""
    import pathlib
    import subprocess
    import sys
    from oracle.oracle import REF_CUDA_SO
    if not REF_CUDA_SO.exists():
        pytest.skip("the reference's CUDA build is not present")
    root = pathlib.Path(__file__).resolve().parents[1]
    out = tmp_path / "ref.npz"
    r = subprocess.run([sys.executable, "-c", REF_CHILD, str(root), kind, str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    d = np.load(out)
    model = {"lp": lp_with_diagonal_q, "qp": qp_with_sparse_q}[kind]()
    close(float(d["monitor"]), monitor(model, d["x"], d["y"], d["xa"], d["ya"]))
