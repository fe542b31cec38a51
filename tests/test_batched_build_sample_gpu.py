"""wrs_batched_build_sample: the batched build and sampler in one call.

The rows must equal those of wrs_batched_build_f32 and the samples those of the oracle's
replay of the plain contract (py_oracle.batched_sample), on batches that take every path: the
lane-group and CTA builds with their per-list samplers, tables with more samples than a list
sampler takes (spilled to the chunked sampler), tables above 8192 items (tiled build, chunked
sampler) and empty tables. The reference has no batched form: it builds and samples one
AliasTableSplitGpu object per table (AliasTableSplitGpu.cu:388-468, SamplerGpuBasic.cu:28-133)."""
import numpy as np
import pytest
import torch

import py_oracle as po
import wrs
from gpu_util import alloc_scratch, to_dev
from test_batched_gpu import EDGE_SIZES, make_batch, zipf_sizes

pytestmark = pytest.mark.gpu

SENT = 0xFFFFFFF9  # fill of the sample output before a call


def counts_for(sizes, kind, seed):
    rng = np.random.default_rng(seed)
    if kind == "fixed64":
        c = np.full(sizes.size, 64)
    elif kind == "spill":  # some tables above the per-list sampler's 2048
        c = rng.integers(0, 5000, sizes.size)
    else:
        c = rng.integers(0, 200, sizes.size)
    return np.where(sizes > 0, c, 0).astype(np.int64)


def run_both(w, off, counts, small, tile, graph=False, seed=0x1234_5678_9ABC, cbase=777):
    sizes = off[1:] - off[:-1]
    soff = np.zeros(sizes.size + 1, dtype=np.int64)
    np.cumsum(counts, out=soff[1:])
    total = int(soff[-1])
    d_w, d_off, d_soff = to_dev(w), to_dev(off), to_dev(soff)
    opts = wrs.build_opts(tile_items=tile, sync=not graph, small_table_items=small)
    table = torch.full((max(1, w.size),), -1, dtype=torch.int64, device="cuda")
    out = torch.full((total + 8,), np.int32(SENT - (1 << 32)), dtype=torch.int32, device="cuda")
    scratch = alloc_scratch(wrs.batched_build_sample_scratch_bytes(off, opts))
    if graph:
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            g.capture_begin()
            st = wrs.batched_build_sample(d_w, d_off, off, table, d_soff, total, seed, out[:total], scratch, opts,
                                          cbase, stream=s)
            g.capture_end()
        torch.cuda.current_stream().wait_stream(s)
        assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
        g.replay()
        torch.cuda.synchronize()
        st = wrs.scratch_status(scratch)
    else:
        st = wrs.batched_build_sample(d_w, d_off, off, table, d_soff, total, seed, out[:total], scratch, opts, cbase)
    torch.cuda.synchronize()
    rows = table.cpu().numpy().view(np.uint32).reshape(-1, 2)[:w.size].copy()
    got = out.cpu().numpy().view(np.uint32)
    assert np.all(got[total:] == np.uint32(SENT)), "sampler wrote past its output"
    # the separate calls on the same batch
    table2 = torch.full((max(1, w.size),), -1, dtype=torch.int64, device="cuda")
    scr2 = alloc_scratch(wrs.batched_build_scratch_bytes(off, opts))
    assert wrs.batched_build(d_w, d_off, off, table2, scr2, wrs.build_opts(tile_items=tile, sync=True,
                                                                           small_table_items=small)) == 0
    rows2 = table2.cpu().numpy().view(np.uint32).reshape(-1, 2)[:w.size]
    return st, rows, rows2, got[:total], soff, seed, cbase


@pytest.mark.parametrize("kind", ["fixed64", "spill", "few"])
@pytest.mark.parametrize("small", [32, 128, 512])
def test_build_sample_edges(cuda, kind, small):
    w, off = make_batch(EDGE_SIZES + [9000, 20000, 3], seed=31)
    counts = counts_for(off[1:] - off[:-1], kind, seed=32)
    st, rows, rows2, got, soff, seed, cbase = run_both(w, off, counts, small, 1024)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    assert np.array_equal(rows, rows2)
    assert np.array_equal(got, po.batched_sample(rows, off, soff, seed, cbase))


def test_build_sample_zipf_graph(cuda):
    sizes = zipf_sizes(4096, 2.0, 2, 1 << 15, seed=41)
    w, off = make_batch(sizes, seed=42, kinds=("uniform",))
    counts = counts_for(off[1:] - off[:-1], "fixed64", seed=43)
    st, rows, rows2, got, soff, seed, cbase = run_both(w, off, counts, 256, 2048, graph=True)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    assert np.array_equal(rows, rows2)
    assert np.array_equal(got, po.batched_sample(rows, off, soff, seed, cbase))


def test_build_sample_equals_separate_calls(cuda):
    """The same samples as wrs_batched_sample on the rows of wrs_batched_build_f32."""
    w, off = make_batch(EDGE_SIZES + [70000], seed=51)
    sizes = off[1:] - off[:-1]
    counts = counts_for(sizes, "spill", seed=52)
    st, rows, rows2, got, soff, seed, cbase = run_both(w, off, counts, 128, 2048)
    assert st == wrs.WRS_SUCCESS
    total = int(soff[-1])
    out = torch.empty(total, dtype=torch.int32, device="cuda")
    assert wrs.batched_sample(to_dev(rows2.view(np.int64).reshape(-1)), to_dev(off), sizes.size, to_dev(soff), total,
                              seed, out, cbase) == 0
    torch.cuda.synchronize()
    assert np.array_equal(got, out.cpu().numpy().view(np.uint32))


def test_build_sample_empty_table_with_samples(cuda):
    w, off = make_batch([10, 0, 300], seed=61)
    counts = np.array([5, 7, 9], dtype=np.int64)
    st, rows, rows2, got, soff, seed, cbase = run_both(w, off, counts, 128, 1024)
    assert st == wrs.WRS_ERR_INVALID_ARGUMENT
    assert np.all(got[5:12] == np.uint32(0xFFFFFFFF))
    ref = po.batched_sample(rows, off, soff, seed, cbase)
    assert np.array_equal(got[:5], ref[:5]) and np.array_equal(got[12:], ref[12:])


def test_build_sample_reports_bad_total(cuda):
    w, off = make_batch([100, 200], seed=71)
    soff = np.array([0, 10, 30], dtype=np.int64)
    out = torch.empty(40, dtype=torch.int32, device="cuda")
    table = torch.empty(w.size, dtype=torch.int64, device="cuda")
    opts = wrs.build_opts(sync=True)
    scratch = alloc_scratch(wrs.batched_build_sample_scratch_bytes(off, opts))
    st = wrs.batched_build_sample(to_dev(w), to_dev(off), off, table, to_dev(soff), 40, 5, out, scratch, opts)
    assert st == wrs.WRS_ERR_INVALID_ARGUMENT


def test_build_sample_autotune(cuda):
    sizes = zipf_sizes(2048, 2.0, 2, 1 << 14, seed=81)
    w, off = make_batch(sizes, seed=82, kinds=("uniform",))
    counts = counts_for(off[1:] - off[:-1], "fixed64", seed=83)
    soff = np.zeros(counts.size + 1, dtype=np.int64)
    np.cumsum(counts, out=soff[1:])
    total = int(soff[-1])
    table = torch.empty(w.size, dtype=torch.int64, device="cuda")
    out = torch.empty(total, dtype=torch.int32, device="cuda")
    scratch = alloc_scratch(wrs.batched_build_sample_scratch_bytes(off, None))
    opts = wrs.build_opts()
    st = wrs.batched_autotune_build_sample(to_dev(w), to_dev(off), off, table, to_dev(soff), total, out, scratch, opts)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    assert opts.small_table_items in (32, 64, 128, 256, 512) and opts.tile_items in (1024, 2048, 4096)
    st, rows, rows2, got, soff2, seed, cbase = run_both(w, off, counts, opts.small_table_items, opts.tile_items)
    assert st == wrs.WRS_SUCCESS
    assert np.array_equal(rows, rows2)
    assert np.array_equal(got, po.batched_sample(rows, off, soff2, seed, cbase))


# every size-class boundary of the lists: lane groups of 2/4/8/16 lanes, a warp with two items
# a lane, a warp up to small_max, CTAs of 256 / 1024 threads, the tiled passes
LIST_EDGES = [1, 2, 4, 5, 8, 9, 16, 17, 32, 33, 64, 65, 128, 129, 256, 257, 512, 513, 2047, 2048, 2049,
              8191, 8192, 8193, 16385]


@pytest.mark.parametrize("small", [32, 64, 256, 512])
def test_build_sample_list_boundaries(cuda, small):
    w, off = make_batch(LIST_EDGES + LIST_EDGES[::-1], seed=91)
    counts = counts_for(off[1:] - off[:-1], "few", seed=92)
    st, rows, rows2, got, soff, seed, cbase = run_both(w, off, counts, small, 1024)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    assert np.array_equal(rows, rows2)
    ref, _, _ = po.batched_build(w, off)
    assert np.array_equal(rows, ref)
    assert np.array_equal(got, po.batched_sample(rows, off, soff, seed, cbase))


def test_build_sample_single_table_and_all_spilled(cuda):
    """One table with many samples (spilled to the chunked sampler), and a batch whose every
    table has more samples than a list sampler takes."""
    for sizes, cnt in (([700], 100_000), ([3, 40, 500, 3000], 3000)):
        w, off = make_batch(sizes, seed=93)
        counts = np.full(len(sizes), cnt, dtype=np.int64)
        st, rows, rows2, got, soff, seed, cbase = run_both(w, off, counts, 128, 2048)
        assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
        assert np.array_equal(rows, rows2)
        assert np.array_equal(got, po.batched_sample(rows, off, soff, seed, cbase))
