"""Build the engine's shared library in-tree for sm_100a.

    python -m niryukti_b200.build          # libnkpdhg.so next to this file

The library is plain nvcc output (no torch extension machinery): C ABI only,
CUDA runtime linked statically, FMA contraction disabled so the elementwise
step formulas round exactly like the reference's CPU backend.  The host C++
(presolve, scaling, verifier) is compiled by g++ with OpenMP and without FMA
contraction, the way the reference's host code is built.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
OUT = HERE / "libnkpdhg.so"
SOURCES = ["nk_engine.cu", "nk_modelfile.cpp"]  # nvcc: CUDA and the host code that shares its errors
HOST_SOURCES = ["nk_prepare.cpp"]  # plain C++: presolve, scaling, verifier
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def gxx() -> str:
    # the system g++ (its OpenMP runtime is installed); other toolchains on
    # PATH may lack libgomp
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("g++ not found")


def _stale(out: pathlib.Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    deps = ([CSRC / s for s in SOURCES + HOST_SOURCES] + list(CSRC.glob("*.cuh")) +
            list(CSRC.glob("*.hpp")) + [ROOT / "include" / "nk_pdhg.h"])
    if not force and not _stale(OUT, deps):
        return OUT
    objs = []
    build_dir = HERE / "_build"
    build_dir.mkdir(exist_ok=True)
    common = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "--fmad=false",
              f"-I{ROOT / 'include'}", f"-I{CSRC}"]
    for s in SOURCES:
        obj = build_dir / (pathlib.Path(s).stem + ".o")
        cmd = [nvcc(), *common, "-c", str(CSRC / s), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        objs.append(str(obj))
    for s in HOST_SOURCES:
        obj = build_dir / (pathlib.Path(s).stem + ".o")
        cmd = [gxx(), "-std=c++17", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off",
               f"-I{ROOT / 'include'}", f"-I{CSRC}", "-c", str(CSRC / s), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        objs.append(str(obj))
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-Xcompiler", "-fopenmp", "-lgomp"]
    subprocess.check_call(cmd)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
