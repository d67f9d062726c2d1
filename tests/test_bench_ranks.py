"""The multi-rank bookkeeping of bench.py on CPU ranks (gloo, world size 2):
the time reported is the slowest rank's, the throughput counts every
replica's units, and the reference arm runs on rank 0 only."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        q.put((rank, ms, bench.replica_throughput(world, 1000, 4, ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_throughput_with_two_gloo_ranks():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, value in got:
        assert ms == 15.0                              # the slower rank's time on every rank
        assert value == pytest.approx(2 * 1000 * 4 / 15e-3)


def test_single_rank_helpers_need_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_throughput(1, 10, 2, 4.0) == pytest.approx(5000.0)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
