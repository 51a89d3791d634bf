"""The engine's host stages under AddressSanitizer and UndefinedBehaviorSanitizer.

tests/c/host_sanitize.cpp is built from the library's host sources (prepare and
scaling, the verifier, model files) with -fsanitize=address,undefined and run
over the host tests' models: hand-made presolve cases, infinite bounds,
subnormal coefficients, QPs, models infeasible at presolve, and one above the
size where the host loops go parallel.  A damaged model file must be refused
cleanly.  Any sanitizer report fails the run."""
import pathlib
import subprocess

import pytest

from niryukti_b200 import modelfile
from tests.test_host import MODELS, infeasible_models, random_presolve_model

ROOT = pathlib.Path(__file__).resolve().parents[1]
CSRC = ROOT / "niryukti_b200" / "csrc"


@pytest.fixture(scope="module")
def sanitized(tmp_path_factory):
    out = tmp_path_factory.mktemp("sanitize") / "host_sanitize"
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=all", "-fno-omit-frame-pointer", "-fopenmp",
           "-ffp-contract=off", f"-I{ROOT / 'include'}", f"-I{CSRC}", "-I/usr/local/cuda/include",
           str(CSRC / "nk_prepare.cpp"), str(CSRC / "nk_modelfile.cpp"),
           str(ROOT / "tests" / "c" / "host_sanitize.cpp"), "-o", str(out)]
    build = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if build.returncode != 0 and "sanitizer" in build.stderr.lower():
        pytest.skip("sanitizer runtime not available: " + build.stderr[-300:])
    assert build.returncode == 0, build.stderr[-3000:]
    return out


def _run(exe, paths):
    return subprocess.run([str(exe), *map(str, paths)], capture_output=True, text=True,
                          timeout=600, env={"ASAN_OPTIONS": "detect_leaks=1",
                                            "UBSAN_OPTIONS": "print_stacktrace=1",
                                            "OMP_NUM_THREADS": "4"})


def test_host_stages_are_clean(sanitized, tmp_path):
    models = {**{k: f() for k, f in MODELS.items()}, **infeasible_models(),
              "threaded": random_presolve_model(21, m=30000, n=70000, per_col=6, fixed=4000,
                                                dups=2500, redundant=1000)}
    assert models["threaded"].nnz > 200000
    paths = []
    for name, model in models.items():
        paths.append(tmp_path / f"{name}.nkm")
        modelfile.save(model, paths[-1])
    r = _run(sanitized, paths)
    assert "Sanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-4000:]
    assert r.returncode == 0, r.stderr[-4000:]
    assert r.stdout.count("prepared") == len(models)


def test_damaged_file_is_refused_cleanly(sanitized, tmp_path):
    from tests.test_oracle import sparse_qp_model
    good = tmp_path / "qp.nkm"
    modelfile.save(sparse_qp_model(), good)
    bad = tmp_path / "cut.nkm"
    bad.write_bytes(good.read_bytes()[:-64])
    r = _run(sanitized, [bad])
    assert "Sanitizer" not in r.stderr and "runtime error" not in r.stderr, r.stderr[-4000:]
    assert r.returncode == 1 and "size does not match" in r.stderr
