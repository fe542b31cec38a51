"""The multi-GPU form of the path is replicas (no data-path collective): every rank runs the
whole step, the job's time is the slowest rank's, and the value is the units all ranks
processed over that time. The rank reduction of bench.py, run as two gloo processes on CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.5, 20.0][rank]
        slowest = bench.max_over_ranks(ms, torch.device("cpu"))
        dist.barrier()
        out[rank] = (slowest, bench.replica_value(1 << 20, slowest, world))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_sum_the_work():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        slowest, value = out[r]
        assert slowest == 20.0
        assert value == pytest.approx(world * (1 << 20) / 20e-3 / 1e9)


def test_single_process_needs_no_group():
    sys.path.insert(0, REPO)
    import bench
    import torch
    assert bench.max_over_ranks(3.5, torch.device("cpu")) == 3.5
    assert bench.replica_value(10 ** 9, 1000.0, 1) == pytest.approx(1.0)


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm (the reference's CPU path) runs and prints on rank 0;
    every other rank exits 0 without work or output."""
    import subprocess
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def _shard_rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "alias-table-gpu_b200"))
    import bench
    import numpy as np
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        def small_batch():
            sizes = bench.zipf_sizes(5000, 2.0, 2, 1 << 12, 11)
            w = np.random.default_rng(11).random(int(sizes.sum()), dtype=np.float32)
            return sizes, w, np.full(sizes.size, 64, np.int64), "small batch", [[np.arange(4), sizes.size]]
        sizes, w, counts, what, groups = bench.shard_of(small_batch, rank, world)()
        t0, t1 = [int(x) for x in what.split("tables [")[1].rstrip(")").split(", ")]
        mine = torch.tensor([t0, t1, int(sizes.sum()), w.size], dtype=torch.int64)
        every = [torch.zeros(4, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(every, mine)
        out[rank] = [e.tolist() for e in every]
        assert groups == []
    finally:
        dist.destroy_process_group()


def test_batch_shards_cover_the_batch_once_without_exchange():
    """Under a world of 2 gloo ranks every rank takes its own contiguous table range of the
    batch (the plan is computed identically on every rank, no exchange of data); together the
    ranges cover every table once and the items are split about evenly."""
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_shard_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert out[0] == out[1]
    ranges = out[0]
    assert ranges[0][0] == 0 and ranges[0][1] == ranges[1][0] and ranges[1][1] == 5000
    items = [r[2] for r in ranges]
    assert all(r[2] == r[3] for r in ranges)
    assert abs(items[0] - items[1]) <= 0.1 * sum(items)
