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
