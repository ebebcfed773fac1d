"""The multi-GPU path is replicas (independent windows / camera streams per rank, no collective on
the data path); what crosses ranks is the timing: a barrier and the max over ranks of the
device-timed region.  These run as world-size-2 gloo process groups on the CPU."""
import json
import os
import pathlib
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world)     # rank 1 is the slower replica
        rate = bench.aggregate_rate(world, steps=4, units_per_step=8, ms=ms)
        q.put((rank, ms, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, rate in got:
        assert ms == 15.0                       # every rank sees the slowest replica's time
        assert rate == pytest.approx(2 * 4 * 8 / 0.015)


def test_single_rank_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.aggregate_rate(1, 10, 8, 1000.0) == 80.0


def test_reference_arm_prints_on_rank_zero_only():
    """bench.py --impl reference under torchrun: ranks other than 0 exit 0 without output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
