"""Host logic of the multi-GPU bench on CPU: world-size-2 gloo ranks reduce
the timed region by MAX and the work by SUM (replicas, weak scaling), and the
reference arm does its work on rank 0 only."""
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank
        res = bench.reduce_over_ranks(ms, 1000 * (rank + 1), 7 * (rank + 1))
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_max_time_sum_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    for r in range(2):
        assert res[r] == (15.0, 3000.0, 21.0)


def test_reference_arm_rank_nonzero_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == ""
