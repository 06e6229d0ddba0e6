"""The multi-GPU path of bench.py is replicas (one full instance per rank, no
collective on the data path); its only exchange is the max of the ranks' times.
Run here as two gloo ranks on the CPU."""
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        kernel_ms, total_ms = 1000.0 + 250.0 * rank, 1500.0 - 100.0 * rank
        slow = bench.max_over_ranks([kernel_ms, total_ms], world, "cpu")
        out[rank] = (slow, bench.replica_throughput(10 ** 12, world, slow[0]))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_time():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        slow, value = res[r]
        assert slow == [1250.0, 1500.0]  # kernel time of rank 1, total time of rank 0
        assert value == pytest.approx(2 * 10 ** 12 / 1.25)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks([3.0, 4.0], 1, "cpu") == [3.0, 4.0]
    assert bench.replica_throughput(100, 1, 1000.0) == 100.0


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
