"""The drop-in build on the CPU: the reference's host code linked with this
engine at its cuda_backend() seam (oracle/_ref/libvantage_nk.so and the CLI
oracle/_ref/niryukti_nk, built by `make -C oracle bridge`).

Without a device it must answer the way the reference's own CUDA build does:
its driver reports UNSUPPORTED with cuda_description()'s "No CUDA device"
(src/cuda.cu:1283), through the library and through the CLI.  The CPU path of
the same build is the reference's own code, so its results are the plain
reference's bit for bit."""
import json
import subprocess

import numpy as np
import pytest

from niryukti_b200 import engine, serve, synth

pytestmark = pytest.mark.skipif(engine.cuda_available(), reason="checks the no-device answers")


@pytest.fixture(scope="module")
def bridged():
    from oracle.oracle import BRIDGE_SO, Reference
    if not BRIDGE_SO.exists():
        pytest.skip("bridged build oracle/_ref/libvantage_nk.so not present")
    return Reference(BRIDGE_SO)


def _lp():
    return synth.random_lp(m=30, n=60, per_col=2, seed=1)


def test_bridged_library_reports_no_device(bridged):
    assert not bridged.cuda_available()
    r = bridged.model(_lp()).solve(method="pdhg", device="cuda")
    assert r["status"] == "UNSUPPORTED" and r["message"] == "No CUDA device"


def test_bridged_cpu_path_is_the_reference(bridged, reference):
    model = _lp()
    a = bridged.model(model).solve(method="pdhg", device="cpu", threads=1)
    b = reference.model(model).solve(method="pdhg", device="cpu", threads=1)
    assert a["status"] == b["status"] == "OPTIMAL"
    assert a["objective"] == b["objective"] and a["iterations"] == b["iterations"]
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["y"], b["y"])


def test_bridged_cli(tmp_path, bridged, reference):
    from oracle.oracle import BRIDGE_SO
    cli = BRIDGE_SO.parent / "niryukti_nk"
    if not cli.exists():
        pytest.skip("bridged CLI not built")
    model = _lp()
    path = tmp_path / "lp.json"
    path.write_text(json.dumps(serve._finite(serve.model_to_json(model))))

    def run(device):
        out = subprocess.run([str(cli), "solve", str(path), "--method", "pdhg", "--device",
                              device, "--threads", "1"], capture_output=True, text=True,
                             timeout=300)
        return json.loads(out.stdout)

    cuda = run("cuda")
    assert cuda["status"] == "UNSUPPORTED" and cuda["message"] == "No CUDA device"
    cpu = run("cpu")
    want = reference.model(model).solve(method="pdhg", device="cpu", threads=1)
    assert cpu["status"] == "OPTIMAL"
    assert cpu["objective"] == pytest.approx(want["objective"], rel=1e-12)
