"""nk_monitor_static: the KKT proxy for callers that may not allocate device memory.

Some callers of this library cannot call cudaMalloc: a host application that
gives all device memory to its own pool or admission budget, or a
latency-critical loop where an allocation would synchronise the device.  For
them nk_monitor_static runs the monitor kernel on a fixed array inside the
library.  This test feeds it the engine's own iterates (device vectors the test
allocates with torch), on an LP and on a QP with a sparse Q (so with a real
Q x), and checks each call against nk_pdhg_monitor, the existing entry point,
and against the FP64 host evaluation of the reference's formula
(oracle/monitor.py, 1e-12 relative), on calls in a row, plus its size limit.

The file name sorts last so that a run stopping at the first failure has run
every other test first; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from niryukti_b200 import synth
from oracle.monitor import cscale_of, monitor_point, products

pytestmark = pytest.mark.gpu

MAX = 4194304  # NK_MONITOR_STATIC_MAX
TOL = 1e-12


def bind(lib):
    f = lib.nk_monitor_static
    f.argtypes = [C.c_int64, C.c_int64] + [C.c_void_p] * 11 + [C.c_double, C.c_void_p,
                                                                C.c_void_p]
    f.restype = C.c_int
    return f


def lp_model():
    model = synth.random_lp(m=3000, n=7000, per_col=5, seed=13)
    model.q = np.where(np.arange(model.n) % 7 == 0, 0.5, 0.0)  # diagonal QP terms too
    return model


def qp_model():
    model = synth.batch_instance(np.random.default_rng(21), 1500, qp=True, name="qp")
    assert model.qnnz > 0
    return model


@pytest.mark.parametrize("make", [lp_model, qp_model], ids=["lp", "sparse_q"])
def test_static_monitor_matches_engine_monitor(gpu, make):
    import torch
    model = make()
    engine = gpu
    lib = engine.library()
    f = bind(lib)
    b = engine.PdhgBackend(model, adaptive=True)
    b.advance(300, 0.05, 0.05)
    expected = b.monitor()  # min over the current and averaged points
    x, y, xa, ya = b.candidates()
    dev = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    cscale = cscale_of(model.c)
    const = {k: t(getattr(model, k)) for k in ("c", "q", "lb", "ub", "rl", "ru")}
    stream = torch.cuda.current_stream(dev)
    outs, host = [], []
    for px, py in ((x, y), (xa, ya), (x, y)):
        ax, aty, qx = products(model, px, py)
        dx, dy, dax, daty = t(px), t(py), t(ax), t(aty)
        dqx = t(qx) if qx is not None else None
        res = torch.full((1,), np.nan, dtype=torch.float64, device=dev)
        status = f(model.n, model.m, dx.data_ptr(), dy.data_ptr(), dax.data_ptr(),
                   daty.data_ptr(), None if dqx is None else dqx.data_ptr(),
                   const["c"].data_ptr(), const["q"].data_ptr(), const["lb"].data_ptr(),
                   const["ub"].data_ptr(), const["rl"].data_ptr(), const["ru"].data_ptr(),
                   cscale, res.data_ptr(), C.c_void_p(stream.cuda_stream))
        assert status == 0, lib.nk_last_error().decode()
        stream.synchronize()
        outs.append(float(res.item()))
        host.append(monitor_point(model, px, py))
    assert all(np.isfinite(outs))
    assert outs[2] == outs[0]  # the shared scratch carries nothing from call to call
    for got, want in zip(outs, host):  # the reference's formula, evaluated on the host
        assert abs(got - want) <= TOL * abs(want), (got, want)
    got = min(outs[:2])
    assert abs(got - expected) <= TOL * abs(expected), (got, expected, outs)


def test_static_monitor_rejects_oversized_input(gpu):
    lib = gpu.library()
    f = bind(lib)
    status = f(MAX + 1, 10, *([None] * 11), 1.0, None, None)
    assert status == 1  # NK_ERR_INVALID
    assert "NK_MONITOR_STATIC_MAX" in lib.nk_last_error().decode()
