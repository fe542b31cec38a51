"""Batched (CSR) alias build and sampler vs the oracle.

Every table of a batch must get exactly the rows of a single-table build of its weights
(or_exact_build per table, table-local aliases), whatever launch shape builds it: the
one-warp-per-table kernel for small tables or the tiled passes run over all large tables.
Batched samples must equal the plain sampling contract over global output positions. The
reference has no batched form; its experiment drivers loop over AliasTableSplitGpu objects
(plots/PlotConstruction.cuh:36-48), so the per-table oracle is its per-table build."""
import numpy as np
import pytest
import torch

import py_oracle as po
import wrs
from gpu_util import alloc_scratch, gpu_build, to_dev

pytestmark = pytest.mark.gpu

# sizes around every class and tile boundary of the launch shapes, empty tables included
EDGE_SIZES = [0, 1, 2, 3, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 513, 1000, 1023, 1024,
              1025, 2047, 2048, 2049, 4095, 4096, 4097, 9000, 33333, 0, 1, 5]


def weights(kind, n, rng):
    if kind == "uniform":
        return rng.random(n, dtype=np.float32)
    if kind == "exp":  # with zero weights
        return (rng.exponential(1.0, n) * (rng.random(n) > 0.1)).astype(np.float32)
    if kind == "powerlaw":
        return ((np.arange(1, n + 1, dtype=np.float64) ** -1.1).astype(np.float32))[rng.permutation(n)]
    if kind == "equal":
        return np.full(n, 0.75, dtype=np.float32)
    raise ValueError(kind)


def make_batch(sizes, seed, kinds=("uniform", "exp", "powerlaw", "equal")):
    rng = np.random.default_rng(seed)
    off = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.cumsum(np.asarray(sizes, dtype=np.int64), out=off[1:])
    parts = []
    for i, n in enumerate(sizes):
        w = weights(kinds[i % len(kinds)], int(n), rng)
        if n > 0 and not np.any(w > 0):
            w[0] = 1.0
        parts.append(w)
    w = np.concatenate(parts) if parts else np.zeros(0, np.float32)
    return w, off


def run_build(w, off, small=0, tile=0, graph=False):
    opts = wrs.build_opts(tile_items=tile, sync=not graph, small_table_items=small)
    d_w, d_off = to_dev(w), to_dev(off)
    table = torch.full((max(1, w.size),), -1, dtype=torch.int64, device="cuda")
    W = torch.zeros(off.size - 1, dtype=torch.float64, device="cuda")
    scratch = alloc_scratch(wrs.batched_build_scratch_bytes(off, opts))
    if graph:
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            g.capture_begin()
            st = wrs.batched_build(d_w, d_off, off, table, scratch, opts, W, stream=s)
            g.capture_end()
        torch.cuda.current_stream().wait_stream(s)
        assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
        g.replay()
        torch.cuda.synchronize()
        st = wrs.scratch_status(scratch)
    else:
        st = wrs.batched_build(d_w, d_off, off, table, scratch, opts, W)
    torch.cuda.synchronize()
    rows = table.cpu().numpy().view(np.uint32).reshape(-1, 2)[:w.size].copy()
    return st, rows, W.cpu().numpy()


def check_batch(w, off, rows, W):
    ref, W_ref, bad = po.batched_build(w, off)
    assert bad == 0
    mism = np.nonzero(np.any(rows != ref, axis=1))[0]
    if mism.size:
        t = np.searchsorted(off, mism[0], side="right") - 1
        raise AssertionError(f"{mism.size} rows differ; first item {mism[0]} (table {t}, n={off[t + 1] - off[t]}): "
                             f"{rows[mism[:3]]} vs {ref[mism[:3]]}")
    nonempty = (off[1:] - off[:-1]) > 0
    assert np.array_equal(W[nonempty], W_ref[nonempty])


@pytest.mark.parametrize("small", [32, 128, 512])
@pytest.mark.parametrize("tile", [1024, 2048, 4096])
def test_batched_edges_bit_exact(cuda, small, tile):
    w, off = make_batch(EDGE_SIZES, seed=small + tile)
    st, rows, W = run_build(w, off, small, tile)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    check_batch(w, off, rows, W)


def zipf_sizes(num, s, lo, hi, seed):
    rng = np.random.default_rng(seed)
    k = np.arange(lo, hi + 1, dtype=np.float64)
    p = k ** -s
    p /= p.sum()
    return rng.choice(np.arange(lo, hi + 1), size=num, p=p)


@pytest.mark.parametrize("small", [64, 256])
def test_batched_zipf_bit_exact(cuda, small):
    sizes = zipf_sizes(4096, 2.0, 2, 1 << 16, seed=41)
    w, off = make_batch(sizes, seed=42, kinds=("uniform",))
    st, rows, W = run_build(w, off, small, 2048)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    check_batch(w, off, rows, W)


def test_batched_equals_single_builds(cuda):
    w, off = make_batch([5, 300, 3000, 70000], seed=7)
    st, rows, _ = run_build(w, off, 128, 2048)
    assert st == wrs.WRS_SUCCESS
    for t in range(4):
        a, b = off[t], off[t + 1]
        st1, rows1, _ = gpu_build(w[a:b])
        assert st1 == wrs.WRS_SUCCESS
        assert np.array_equal(rows[a:b], rows1), f"table {t}"


def test_batched_graph_capture(cuda):
    w, off = make_batch(EDGE_SIZES, seed=3)
    st, rows, W = run_build(w, off, 128, 2048, graph=True)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    check_batch(w, off, rows, W)


def test_batched_autotune(cuda):
    sizes = zipf_sizes(2048, 2.0, 2, 1 << 14, seed=5)
    w, off = make_batch(sizes, seed=6, kinds=("uniform",))
    d_w, d_off = to_dev(w), to_dev(off)
    table = torch.empty(w.size, dtype=torch.int64, device="cuda")
    scratch = alloc_scratch(wrs.batched_build_scratch_bytes(off, None))
    opts = wrs.build_opts()
    st = wrs.batched_autotune(d_w, d_off, off, table, scratch, opts)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    assert opts.small_table_items in (32, 64, 128, 256, 512) and opts.tile_items in (1024, 2048, 4096)
    st, rows, W = run_build(w, off, opts.small_table_items, opts.tile_items)
    assert st == wrs.WRS_SUCCESS
    check_batch(w, off, rows, W)


@pytest.mark.parametrize("counts_kind", ["fixed64", "mixed"])
def test_batched_sample_bit_exact(cuda, counts_kind):
    w, off = make_batch(EDGE_SIZES, seed=11)
    st, rows, W = run_build(w, off, 128, 2048)
    assert st == wrs.WRS_SUCCESS
    sizes = off[1:] - off[:-1]
    rng = np.random.default_rng(12)
    if counts_kind == "fixed64":
        counts = np.where(sizes > 0, 64, 0)
    else:
        counts = np.where(sizes > 0, rng.integers(0, 5000, sizes.size), 0)
    soff = np.zeros(sizes.size + 1, dtype=np.int64)
    np.cumsum(counts, out=soff[1:])
    total = int(soff[-1])
    seed, cbase = 0x1234_5678_9ABC, 777
    table = to_dev(rows.view(np.int64).reshape(-1))
    out = torch.full((total + 8,), -7, dtype=torch.int32, device="cuda")
    st = wrs.batched_sample(table, to_dev(off), sizes.size, to_dev(soff), total, seed, out[:total], cbase)
    torch.cuda.synchronize()
    assert st == wrs.WRS_SUCCESS
    got = out.cpu().numpy().view(np.uint32)
    assert np.all(got[total:] == np.uint32(0xFFFFFFF9)), "sampler wrote past its output"
    ref = po.batched_sample(rows, off, soff, seed, cbase)
    assert np.array_equal(got[:total], ref)
    tab = np.repeat(np.arange(sizes.size), counts)
    assert np.all(got[:total] < sizes[tab]), "a sample is not a row of its table"


def test_batched_reports_mismatched_offsets(cuda):
    w, off = make_batch([100, 5000, 7], seed=2)
    bad = off.copy()
    bad[1] = 120  # the host copy disagrees with the device copy
    opts = wrs.build_opts(sync=True)
    table = torch.empty(w.size, dtype=torch.int64, device="cuda")
    scratch = alloc_scratch(wrs.batched_build_scratch_bytes(bad, None))
    st = wrs.batched_build(to_dev(w), to_dev(off), bad, table, scratch, opts)
    assert st == wrs.WRS_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("where", ["small", "large"])
def test_batched_reports_invalid_weight(cuda, where):
    w, off = make_batch([100, 5000, 7], seed=2)
    w[off[0 if where == "small" else 1] + 17] = -1.0
    st, _, _ = run_build(w, off, 128, 2048)
    assert st == wrs.WRS_ERR_INVALID_WEIGHT
