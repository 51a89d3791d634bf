import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def has_cuda() -> bool:
    try:
        from niryukti_b200 import engine
        return engine.cuda_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import REF_SO, Reference
    if not REF_SO.exists():
        pytest.skip("reference build oracle/_ref not present")
    return Reference()


def load_golden(name):
    from tests.golden.make_golden import model_from
    d = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    return model_from(d), d


@pytest.fixture(scope="session")
def gpu():
    if not has_cuda():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    from niryukti_b200 import engine
    return engine
