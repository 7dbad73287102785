"""The N > 1 plumbing of bench.py on CPU: world_size-2 gloo process groups.

Every rank of `bench.py --gpus N` runs its own replica of the workload (cells
are independent given the conditioning data: no collective on the data path);
the step time is the slowest rank's (rank_max) and the value is the whole
job's units per second (whole_job_rate). The reference arm runs on rank 0
alone; the other ranks exit 0 without work.
"""
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ms = bench.rank_max(dist, 10.0 + 5.0 * rank, "cpu")  # rank 1 is the slower replica
        value = bench.whole_job_rate(1000, world, ms)
        dist.barrier()
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_rank_max_and_whole_job_rate_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]  # both ranks time the job by its slowest rank
    assert all(abs(o[2] - 2 * 1000 / 0.015) < 1e-6 for o in out)


def test_rank_max_without_a_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.rank_max(None, 3.5, "cpu") == 3.5
    assert bench.whole_job_rate(500, 1, 250.0) == 2000.0


def test_reference_arm_is_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1", MASTER_PORT="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
