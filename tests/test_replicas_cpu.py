"""Multi-GPU form on CPU: bench.py runs one independent replica per rank and reports the job
aggregate with the slowest rank's device time.  Two gloo ranks (spawned processes) check the
max-over-ranks reduction and the whole-job throughput that the N > 1 runs use."""

import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402

TIMES_MS = (12.5, 40.0)  # per-rank device time of the timed region
UNITS = 11_778_624       # ordered determinant pairs per step per rank
STEPS = 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(TIMES_MS[rank], "cpu")
        value = bench.job_throughput(UNITS, STEPS, world, ms)
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{ms!r} {value!r}\n")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    expect_ms = max(TIMES_MS)
    expect_value = UNITS * STEPS * world / (expect_ms * 1e-3)
    for rank in range(world):
        ms, value = (float(x) for x in open(tmp_path / f"rank{rank}.txt").read().split())
        assert ms == expect_ms
        assert value == pytest.approx(expect_value, rel=1e-15)


def test_single_process_keeps_its_own_time():
    assert bench.max_over_ranks(7.25, "cpu") == 7.25
    assert bench.job_throughput(100, 2, 1, 1000.0) == pytest.approx(200.0)
