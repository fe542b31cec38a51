"""Table files and the sharding of a batch over devices.

CPU: the shard planner's ranges (contiguous, covering, balanced by items plus a per-table cost)
and the file reader's rejection of files that are not table files. GPU: a single table and a
CSR batch written, read back bit for bit (rows, offsets, W), and a corrupted file rejected by
its checksum."""
import os

import numpy as np
import pytest
import torch

import wrs
from gpu_util import gpu_build


def shard_cost(off, bounds, cost):
    return [int(off[bounds[s + 1]] - off[bounds[s]]) + cost * int(bounds[s + 1] - bounds[s])
            for s in range(len(bounds) - 1)]


@pytest.mark.parametrize("shards", [1, 2, 3, 8])
def test_shard_plan_covers_and_balances(shards):
    rng = np.random.default_rng(shards)
    sizes = np.minimum(rng.zipf(2.0, 20000), 1 << 16).astype(np.int64)
    off = np.zeros(sizes.size + 1, np.int64)
    np.cumsum(sizes, out=off[1:])
    st, b = wrs.shard_tables(off, shards, 16)
    assert st == wrs.WRS_SUCCESS
    assert b[0] == 0 and b[-1] == sizes.size and np.all(np.diff(b) >= 0)
    costs = shard_cost(off, b, 16)
    total = sum(costs)
    # each shard within one table (plus its cost) of an even share
    assert max(costs) <= total / shards + sizes.max() + 16


def test_shard_plan_edge_cases():
    off = np.array([0, 5, 5, 5, 100], np.int64)
    st, b = wrs.shard_tables(off, 8, 0)
    assert st == wrs.WRS_SUCCESS and b[0] == 0 and b[-1] == 4 and np.all(np.diff(b) >= 0)
    st, b = wrs.shard_tables(np.array([0], np.int64), 3, 16)
    assert st == wrs.WRS_SUCCESS and np.all(b == 0)
    assert wrs.shard_tables(np.array([0, 5, 3], np.int64), 2, 0)[0] == wrs.WRS_ERR_INVALID_ARGUMENT
    assert wrs.shard_tables(np.array([1, 5], np.int64), 2, 0)[0] == wrs.WRS_ERR_INVALID_ARGUMENT


def test_file_info_rejects_other_files(tmp_path):
    p = tmp_path / "x.bin"
    p.write_bytes(b"not a table" * 10)
    assert wrs.table_file_info(str(p))[0] == wrs.WRS_ERR_INVALID_ARGUMENT
    assert wrs.table_file_info(str(tmp_path / "missing"))[0] == wrs.WRS_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
def test_table_file_round_trip(cuda, tmp_path):
    w = np.random.default_rng(5).random(300_001, dtype=np.float32)
    st, rows, W = gpu_build(w)
    assert st == 0
    table = torch.from_numpy(rows.view(np.int64).reshape(-1)).cuda()
    path = str(tmp_path / "t.wrs")
    assert wrs.table_file_write(path, table, W) == wrs.WRS_SUCCESS
    st, n, t, W2 = wrs.table_file_info(path)
    assert (st, n, t, W2) == (wrs.WRS_SUCCESS, w.size, 1, W)
    back = torch.full_like(table, -1)
    st, off = wrs.table_file_read(path, back)
    assert st == wrs.WRS_SUCCESS and list(off) == [0, w.size]
    np.testing.assert_array_equal(back.cpu().numpy(), table.cpu().numpy())
    # a flipped byte in the rows fails the checksum
    data = bytearray(open(path, "rb").read())
    data[-5] ^= 0x40
    open(path, "wb").write(bytes(data))
    assert wrs.table_file_read(path, back)[0] == wrs.WRS_ERR_INVALID_ARGUMENT
    # the wrong size is refused before anything is read
    small = torch.empty(10, dtype=torch.int64, device="cuda")
    assert wrs.table_file_read(path, small)[0] == wrs.WRS_ERR_CAPACITY


@pytest.mark.gpu
def test_batched_table_file_round_trip(cuda, tmp_path):
    sizes = np.array([3, 0, 1000, 1, 70_000, 64], np.int64)
    off = np.zeros(sizes.size + 1, np.int64)
    np.cumsum(sizes, out=off[1:])
    rows = np.random.default_rng(6).integers(0, 2**31, size=(int(off[-1]), 2), dtype=np.uint32)
    table = torch.from_numpy(rows.view(np.int64).reshape(-1)).cuda()
    path = str(tmp_path / "b.wrs")
    assert wrs.batched_table_file_write(path, table, off) == wrs.WRS_SUCCESS
    st, n, t, W = wrs.table_file_info(path)
    assert (st, n, t, W) == (wrs.WRS_SUCCESS, int(off[-1]), sizes.size, 0.0)
    back = torch.zeros_like(table)
    st, off2 = wrs.table_file_read(path, back, num_tables=sizes.size)
    assert st == wrs.WRS_SUCCESS
    np.testing.assert_array_equal(off2, off)
    np.testing.assert_array_equal(back.cpu().numpy(), table.cpu().numpy())
