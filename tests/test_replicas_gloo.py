"""Multi-process path of bench.py on CPU (gloo, world size 2).

A single LP is not partitioned: with N GPUs the benchmark runs N independent
replicas, takes the slowest rank's CUDA-event time (max over ranks) and reports
the units all ranks processed over that time.  The reference arm runs on rank 0
only; the other ranks exit without work.  These are the host-side pieces of
that path, run here as two gloo ranks."""
import json
import os
import pathlib
import socket
import sys
import types

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms = bench.max_over_ranks(local_ms, dist, device="cpu")
        rate = bench.replica_rate(world, 100, ms)
        # the reference arm does its work on rank 0 only
        skipped = bench.reference_arm(types.SimpleNamespace(), world, rank) is None \
            if rank != 0 else None
        dist.barrier()
        pathlib.Path(out_dir, f"rank{rank}.json").write_text(
            json.dumps({"ms": ms, "rate": rate, "skipped": skipped}))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    got = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for g in got:
        assert g["ms"] == pytest.approx(15.0)           # max over ranks, on every rank
        assert g["rate"] == pytest.approx(2 * 100 / 0.015)  # both replicas' units / slowest time
    assert got[1]["skipped"] is True


def test_one_process_is_its_own_maximum():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.replica_rate(1, 100, 20.0) == pytest.approx(5000.0)
