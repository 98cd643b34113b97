"""Host logic of the multi-GPU bench on CPU: world-size-2 gloo ranks reduce
the timed region by MAX and the work by SUM (replicas, weak scaling), merge
pixel-tile partitions into one frame (tile data parallelism), and the
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


def _partition_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    import bench
    import barney_b200 as bn
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        W, H = 97, 61
        owners = torch.from_numpy(bn.partition_owners(W, H, world))
        # this rank "renders" its own pixels (value rank+1); the rest is garbage
        frame = torch.full((H, W), -7, dtype=torch.int32)
        frame[owners == rank] = rank + 1
        full = bench.gather_partitions(frame, owners)
        q.put((rank, bool(torch.equal(full, owners + 1))))
    finally:
        dist.destroy_process_group()


def test_two_rank_pixel_partition_gather_assembles_the_frame():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000
    procs = [ctx.Process(target=_partition_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: True, 1: True}


def test_partition_owner_map_deals_whole_tiles_round_robin():
    import numpy as np
    import barney_b200 as bn
    W, H = 1920, 1080
    assert (bn.partition_owners(W, H, 1) == 0).all()
    for n in (2, 3, 8):
        o = bn.partition_owners(W, H, n)
        counts = np.bincount(o.ravel(), minlength=n)
        assert counts.sum() == W * H and counts.min() > 0
        assert counts.max() - counts.min() <= 1024  # whole 1024-pixel tiles
        # the first 4-row band is 4 * W pixels = 7.5 tiles, dealt in order
        band = o[:4].T.ravel()  # column-major inside the band
        assert (band[:1024] == 0).all() and (band[1024:2048] == 1 % n).all()
