"""The C ABI boundary without a GPU: the library loads, exports every entry point
declared in include/*.h, validates arguments before touching a device, and
reports a missing device as a status instead of crashing."""
import ctypes as C
import pathlib
import re
import subprocess

import numpy as np
import pytest

from niryukti_b200 import engine, synth

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(nk_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def exported_symbols(lib):
    out = subprocess.check_output(["nm", "-D", "--defined-only", str(lib)], text=True)
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_symbol():
    lib = engine.LIB_PATH
    assert lib.exists(), "build the extension first (python -m niryukti_b200.build)"
    declared = declared_symbols()
    assert {"nk_pdhg_create", "nk_pdhg_advance", "nk_pdhg_candidates"} <= declared
    missing = declared - exported_symbols(lib)
    assert not missing, missing


def test_library_loads_and_reports_version():
    L = engine.library()
    assert L.nk_abi_version() == 1
    assert isinstance(engine.cuda_available(), bool)


def _bad_model():
    m = synth.random_lp(m=20, n=40, per_col=2, seed=3)
    return m


def test_invalid_csr_is_rejected_before_device_use():
    m = _bad_model()
    m.ptr = m.ptr.copy()
    m.ptr[5], m.ptr[6] = m.ptr[6], m.ptr[5] - 1  # decreasing offsets
    with pytest.raises(engine.EngineError) as e:
        engine.PdhgBackend(m)
    assert e.value.status == "INVALID"
    assert "CSR" in str(e.value)


def test_halpern_with_adaptive_is_refused():
    with pytest.raises(engine.EngineError) as e:
        engine.PdhgBackend(_bad_model(), adaptive=True, halpern=True)
    assert e.value.status == "UNSUPPORTED"
    assert "Halpern requires a fixed PDHG operator" in str(e.value)


def test_bad_reflection_is_refused():
    with pytest.raises(engine.EngineError) as e:
        engine.PdhgBackend(_bad_model(), halpern=True, reflection=1.5)
    assert "reflection" in str(e.value)


@pytest.mark.skipif(engine.cuda_available(), reason="checks the no-device path")
def test_missing_device_is_a_status():
    with pytest.raises(engine.EngineError) as e:
        engine.PdhgBackend(_bad_model())
    assert e.value.status == "NO_DEVICE"
    assert engine.hardware_info()["gpu_available"] is False
    assert engine.cuda_description() == "No CUDA device"


def test_side_entries_check_their_arguments_before_device_use():
    """The presolve and Newton entries refuse bad maps, bounds and shapes with a
    status before any device call (so these run without a GPU)."""
    m = _bad_model()
    cmap = np.arange(m.n)
    with pytest.raises(engine.EngineError, match="compaction row map"):
        engine.compact_csr(m.ptr, m.idx, m.val, m.n, [4, 4], cmap, m.n)
    with pytest.raises(engine.EngineError, match="compaction column map"):
        engine.compact_csr(m.ptr, m.idx, m.val, m.n, [0], cmap, m.n - 1)  # map beyond the output
    bad_lb = m.lb.copy()
    bad_lb[3] = m.ub[3] + 1  # crossed bounds
    with pytest.raises(engine.EngineError, match="invalid propagation bounds"):
        engine.propagate_bounds(m, np.zeros(m.n, dtype=np.int32), bad_lb, m.ub)
    with pytest.raises(engine.EngineError, match="invalid propagation arguments"):
        engine.propagate_bounds(m, np.zeros(m.n, dtype=np.int32), m.lb, m.ub, passes=101)
    rect = np.array([0, 1, 2]), np.array([0, 5]), np.array([1.0, 2.0])
    with pytest.raises(engine.EngineError, match="Newton column index out of range"):
        engine.linear_solve(*rect, np.ones(2))


@pytest.mark.skipif(engine.cuda_available(), reason="checks the no-device path")
def test_side_entries_report_a_missing_device():
    m = _bad_model()
    with pytest.raises(engine.EngineError) as e:
        engine.compact_csr(m.ptr, m.idx, m.val, m.n, [0, 1], np.arange(m.n), m.n)
    assert e.value.status == "NO_DEVICE"
    with pytest.raises(engine.EngineError) as e:
        engine.propagate_bounds(m, np.zeros(m.n, dtype=np.int32), m.lb, m.ub)
    assert e.value.status == "NO_DEVICE"


def test_null_pointers_are_argument_errors():
    """A null handle or a null required pointer is answered with NK_ERR_INVALID
    and a message, never a host crash; destroy, free and defaults accept null;
    the info entries skip null outputs.  Runs through the C ABI with no GPU."""
    L = C.CDLL(str(engine.LIB_PATH))
    L.nk_last_error.restype = C.c_char_p
    INVALID, P, d = 1, C.c_void_p(), C.c_double
    assert L.nk_pdhg_advance(P, 1, d(1.0), d(1.0), P) == INVALID
    assert L.nk_last_error() == b"null engine handle"
    for name in ("nk_pdhg_rejected_steps", "nk_pdhg_restart_requested", "nk_pdhg_monitor",
                 "nk_pdhg_snapshot", "nk_pdhg_stream"):
        assert getattr(L, name)(P, P) == INVALID, name
    assert L.nk_pdhg_candidates(P, P, P, P, P) == INVALID
    assert L.nk_pdhg_reset(P, P, P) == INVALID
    assert L.nk_pdhg_restore(P, P, P, 10) == INVALID
    assert L.nk_pdhg_create(P, P, P, P, P, P, P, P, P, P, P, P) == INVALID
    assert L.nk_prepare(P, 1, 0, 5, P) == INVALID
    assert L.nk_solve(P, P, P, P, P) == INVALID
    assert L.nk_verify(P, P, P, 0, P) == INVALID
    assert L.nk_batch_create(P, P) == INVALID
    assert L.nk_batch_estimate(P, P) == INVALID
    assert L.nk_batch_step(P, 1, P, 0, P) == INVALID
    assert L.nk_batch_result(P, C.c_int64(0), P, P, P) == INVALID
    assert L.nk_cuda_description(P, 0) == INVALID
    for name in ("nk_pdhg_destroy", "nk_batch_destroy", "nk_prepared_free",
                 "nk_batch_item_free", "nk_solve_defaults", "nk_batch_defaults"):
        getattr(L, name)(P)
    assert L.nk_hardware_info(P, P, P) == 0
    total = d(-1.0)
    assert L.nk_hardware_info(P, P, C.byref(total)) == 0 and total.value >= 0


def test_plain_c_caller(tmp_path):
    """include/nk_pdhg.h compiles as strict C99 and a C program linked against
    the library runs its host entries and gets the solve's missing-device
    status (tests/c/abi_host.c)."""
    exe = tmp_path / "abi_host"
    lib_dir = engine.LIB_PATH.parent
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                           f"-I{ROOT / 'include'}", str(ROOT / "tests" / "c" / "abi_host.c"),
                           f"-L{lib_dir}", "-lnkpdhg", f"-Wl,-rpath,{lib_dir}", "-lm",
                           "-o", str(exe)])
    out = subprocess.run([str(exe), str(tmp_path / "lp.nkm")], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    words = out.stdout.split()
    assert words[:4] == ["rows", "2", "cols", "2"]
    assert float(words[5]) == pytest.approx(-2.8, rel=1e-12)
    assert float(words[7]) < 1e-12


def test_model_entries_are_checked_like_the_reference():
    """The host entries (nk_prepare, nk_solve, nk_verify, nk_batch_*) refuse the
    entries Model::validate refuses (src/model.cpp:107-123), before any host
    array is indexed by them."""
    from niryukti_b200 import solver
    from tests.test_oracle import sparse_qp_model

    def refused(model, message):
        with pytest.raises(engine.EngineError, match=message) as e:
            solver.prepare(model)
        assert e.value.status == "INVALID"

    lp = synth.random_lp(m=20, n=40, per_col=2, seed=3)
    for k, bad in ((5, lp.n), (7, -1)):
        m = synth.Model(**{**lp.__dict__, "idx": lp.idx.copy()})
        m.idx[k] = bad
        refused(m, "Invalid matrix coefficient/index")
    for bad in (np.nan, np.inf):
        m = synth.Model(**{**lp.__dict__, "val": lp.val.copy()})
        m.val[3] = bad
        refused(m, "Invalid matrix coefficient/index")
    qp = sparse_qp_model()
    assert qp.qnnz >= 2
    m = synth.Model(**{**qp.__dict__, "qval": qp.qval.copy()})
    off = np.flatnonzero(np.repeat(np.arange(qp.n), np.diff(qp.qptr)) != qp.qidx)[0]
    m.qval[off] += 1.0  # one off-diagonal entry without its mirror
    refused(m, "exactly symmetric")
    m = synth.Model(**{**qp.__dict__, "qval": qp.qval.copy()})
    m.qval[0] = np.nan
    refused(m, "Invalid quadratic coefficient/index")
    solver.prepare(qp)  # the valid model still passes


def test_solve_decided_before_the_device(reference):
    """nk_solve's host stages (the verifier built beside prepare, the start-point
    checks of src/solver.cpp:268-287) run without a device: a model infeasible
    at presolve and one optimal at the start point are decided there, like the
    reference's solve; any other model then reports the missing device."""
    from niryukti_b200 import solver
    from tests.test_host import from_rows
    infeasible = from_rows(2, [[(0, 2.0)], [(1, 1.0)]], lb=[1, 0], ub=[1, 1], rl=[5, 0],
                           ru=[6, 1])
    assert solver.solve(infeasible)["status"] == "INFEASIBLE"
    assert reference.model(infeasible).solve(method="pdhg")["status"] == "INFEASIBLE"
    at_start = from_rows(2, [[(0, 1.0), (1, 1.0)]], c=[1, 1], lb=[0, 0], ub=[3, 3],
                         rl=[-np.inf], ru=[5])
    r = solver.solve(at_start)
    want = reference.model(at_start).solve(method="pdhg")
    assert r["status"] == want["status"] == "OPTIMAL"
    assert r["iterations"] == 0 and r["objective"] == want["objective"] == 0.0
    if not engine.cuda_available():
        with pytest.raises(engine.EngineError) as e:
            solver.solve(synth.random_lp(m=20, n=40, per_col=2, seed=3))
        assert e.value.status == "NO_DEVICE"
