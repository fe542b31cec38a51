"""Mixed batches (alias or rejection per table) vs the oracle.

Alias tables must get exactly the rows of the batched alias build, rejection tables exactly
the slots, acceptances and |A_t| of a single-table rejection build of their weights
(or_rejection_build with W the exact sum, at A[2 off[t]:]); skipped tables must be left
alone. The mixed sampler must equal the oracle's replay: the plain contract on alias
tables, the rejection contract over the global position on rejection tables. The reference
has no mixed form: it builds one RejectionSampling or AliasTableSplitGpu object per table
(RejectionSampling.cu:35-56, AliasTableSplitGpu.cu:388-468)."""
import numpy as np
import pytest
import torch

import py_oracle as po
import wrs
from gpu_util import alloc_scratch, to_dev
from test_batched_gpu import EDGE_SIZES, make_batch

pytestmark = pytest.mark.gpu

SENT = 0xFFFFFFF7  # fill of the slot array and of the sample output before a call


def mixed_sizes():
    # the edge sizes, plus tables above the one-warp rejection limit (4096 items)
    return EDGE_SIZES + [4097, 5000, 9000, 70000, 3, 64]


def random_kinds(num, seed):
    return np.random.default_rng(seed).integers(0, 3, num).astype(np.uint8)


def run_mixed_build(w, off, kinds, opts=None, graph=False):
    n = w.size
    d_w, d_off, d_kinds = to_dev(w), to_dev(off), to_dev(kinds)
    table = torch.full((max(1, n),), -1, dtype=torch.int64, device="cuda")
    A = torch.full((max(1, 2 * n),), SENT - (1 << 32), dtype=torch.int32, device="cuda")
    frac = torch.full((max(1, n),), -2.0, dtype=torch.float32, device="cuda")
    a_size = torch.full((kinds.size,), 12345, dtype=torch.int64, device="cuda")
    W = torch.zeros(kinds.size, dtype=torch.float64, device="cuda")
    scratch = alloc_scratch(wrs.batched_mixed_build_scratch_bytes(off, kinds, opts))
    if graph:
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            g.capture_begin()
            st = wrs.batched_mixed_build(d_w, d_off, off, d_kinds, kinds, table, A, frac, a_size, scratch, opts, W,
                                         stream=s)
            g.capture_end()
        torch.cuda.current_stream().wait_stream(s)
        assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
        g.replay()
    else:
        st = wrs.batched_mixed_build(d_w, d_off, off, d_kinds, kinds, table, A, frac, a_size, scratch, opts, W)
        assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    torch.cuda.synchronize()
    st = wrs.scratch_status(scratch)
    out = dict(rows=table.cpu().numpy().view(np.uint32).reshape(-1, 2)[:n].copy(),
               A=A.cpu().numpy().view(np.uint32)[:2 * n].copy(), frac=frac.cpu().numpy()[:n].copy(),
               a_size=a_size.cpu().numpy().astype(np.uint64), W=W.cpu().numpy(),
               dev=dict(table=table, A=A, frac=frac, a_size=a_size, off=d_off, kinds=d_kinds))
    return st, out


def check_mixed(w, off, kinds, got):
    rows, A, frac, a_size, W, bad = po.batched_mixed_build(w, off, kinds)
    assert bad == 0
    for t in range(kinds.size):
        a, b = int(off[t]), int(off[t + 1])
        n = b - a
        if n == 0:
            continue
        if kinds[t] == wrs.WRS_TABLE_ALIAS:
            assert np.array_equal(got["rows"][a:b], rows[a:b]), f"alias table {t} (n={n})"
            assert got["W"][t] == W[t]
        elif kinds[t] == wrs.WRS_TABLE_REJECTION:
            asz = int(a_size[t])
            assert int(got["a_size"][t]) == asz, f"rejection table {t} (n={n}): |A| {got['a_size'][t]} vs {asz}"
            assert np.array_equal(got["A"][2 * a:2 * a + asz], A[2 * a:2 * a + asz]), f"rejection table {t} slots"
            assert np.all(got["A"][2 * a + asz:2 * b] == SENT), f"rejection table {t} wrote past |A|"
            assert np.array_equal(got["frac"][a:b].view(np.uint32), frac[a:b].view(np.uint32)), f"table {t} frac"
            assert got["W"][t] == W[t]
            assert np.all(got["rows"][a:b] == 0xFFFFFFFF), f"rejection table {t} got alias rows"
        else:
            assert np.all(got["rows"][a:b] == 0xFFFFFFFF) and np.all(got["A"][2 * a:2 * b] == SENT), f"skipped {t}"
            assert int(got["a_size"][t]) == 12345


@pytest.mark.parametrize("seed", [1, 2])
def test_mixed_build_bit_exact(cuda, seed):
    w, off = make_batch(mixed_sizes(), seed=seed)
    kinds = random_kinds(off.size - 1, seed)
    st, got = run_mixed_build(w, off, kinds, wrs.build_opts(small_table_items=128, tile_items=2048))
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    check_mixed(w, off, kinds, got)


def test_mixed_all_rejection_skewed(cuda):
    # power-law weights: items with many slots (the cooperative fill) in both launch forms
    sizes = [10, 100, 1000, 4096, 4097, 20000, 100000]
    w, off = make_batch(sizes, seed=9, kinds=("powerlaw",))
    kinds = np.full(len(sizes), wrs.WRS_TABLE_REJECTION, dtype=np.uint8)
    st, got = run_mixed_build(w, off, kinds)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    check_mixed(w, off, kinds, got)


def test_mixed_all_alias_equals_batched(cuda):
    w, off = make_batch(mixed_sizes(), seed=4)
    kinds = np.zeros(off.size - 1, dtype=np.uint8)
    st, got = run_mixed_build(w, off, kinds)
    assert st == wrs.WRS_SUCCESS
    ref, _, _ = po.batched_build(w, off)
    assert np.array_equal(got["rows"], ref)


def test_mixed_graph_capture(cuda):
    w, off = make_batch(mixed_sizes(), seed=5)
    kinds = random_kinds(off.size - 1, 5)
    st, got = run_mixed_build(w, off, kinds, graph=True)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    check_mixed(w, off, kinds, got)


def sample_offsets(off, seed):
    sizes = off[1:] - off[:-1]
    rng = np.random.default_rng(seed)
    counts = np.where(sizes > 0, rng.integers(0, 3000, sizes.size), 0)
    soff = np.zeros(sizes.size + 1, dtype=np.int64)
    np.cumsum(counts, out=soff[1:])
    return soff


@pytest.mark.parametrize("seed", [3, 4])
def test_mixed_sample_bit_exact(cuda, seed):
    w, off = make_batch(mixed_sizes(), seed=seed)
    kinds = random_kinds(off.size - 1, seed)
    st, got = run_mixed_build(w, off, kinds)
    assert st == wrs.WRS_SUCCESS
    soff = sample_offsets(off, seed)
    total = int(soff[-1])
    d = got["dev"]
    out = torch.full((total + 8,), SENT - (1 << 32), dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    sd, cb = 0xABCDEF12345, 99
    st = wrs.batched_mixed_sample(d["table"], d["A"], d["frac"], d["a_size"], d["off"], d["kinds"], kinds.size,
                                  to_dev(soff), total, sd, out[:total], cb, 0, status)
    torch.cuda.synchronize()
    assert st == wrs.WRS_SUCCESS and int(status.item()) == 0
    g = out.cpu().numpy().view(np.uint32)
    assert np.all(g[total:] == SENT), "sampler wrote past its output"
    expect = np.full(max(total, 1), SENT, dtype=np.uint32)
    ref, failed = po.batched_mixed_sample(got["rows"], got["A"], got["frac"], got["a_size"], off, kinds, soff, sd, cb,
                                          0, expect)
    assert failed == 0
    assert np.array_equal(g[:total], ref), f"{np.count_nonzero(g[:total] != ref)} samples differ"
    tab = np.repeat(np.arange(kinds.size), soff[1:] - soff[:-1])
    live = kinds[tab] <= 1
    assert np.all(g[:total][live] < (off[1:] - off[:-1])[tab][live])


def test_autotune_kinds(cuda):
    # tiny tables and a few large ones, like the mixed-batch workload
    rng = np.random.default_rng(21)
    sizes = list(rng.integers(1, 65, 3000)) + [1 << 16] * 3
    w, off = make_batch(sizes, seed=22, kinds=("exp",))
    n = w.size
    counts = 4 * (off[1:] - off[:-1])
    soff = np.zeros(counts.size + 1, dtype=np.int64)
    np.cumsum(counts, out=soff[1:])
    d_w, d_off, d_soff = to_dev(w), to_dev(off), to_dev(soff)
    table = torch.empty(n, dtype=torch.int64, device="cuda")
    A = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    frac = torch.empty(n, dtype=torch.float32, device="cuda")
    a_size = torch.empty(off.size - 1, dtype=torch.int64, device="cuda")
    kt = torch.empty(off.size - 1, dtype=torch.uint8, device="cuda")
    out = torch.empty(int(soff[-1]), dtype=torch.int32, device="cuda")
    scratch = alloc_scratch(wrs.batched_mixed_build_scratch_bytes(off, None, None))
    st, kinds, cls, ms = wrs.batched_autotune_kinds(d_w, d_off, off, d_soff, soff, table, A, frac, a_size, kt,
                                                    out, scratch)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    sizes = off[1:] - off[:-1]
    c = np.where(sizes <= 1, 0, np.ceil(np.log2(np.maximum(sizes, 2))).astype(int))
    assert np.all(kinds == cls[c]), "a table's kind is not its class's"
    for k in np.unique(c):
        assert ms[k, 0] > 0 and ms[k, 1] > 0
        # rejection only where it takes under 0.95 of alias's time
        want = wrs.WRS_TABLE_REJECTION if np.float32(ms[k, 1]) < np.float32(0.95) * np.float32(ms[k, 0]) \
            else wrs.WRS_TABLE_ALIAS
        assert cls[k] == want
    assert set(np.unique(cls[c]).tolist()) <= {wrs.WRS_TABLE_ALIAS, wrs.WRS_TABLE_REJECTION}
    st, got = run_mixed_build(w, off, kinds)
    assert st == wrs.WRS_SUCCESS
    check_mixed(w, off, kinds, got)


def test_mixed_rejection_invalid_weight(cuda):
    w, off = make_batch([100, 5000, 7], seed=2)
    w[off[1] + 17] = -1.0
    kinds = np.array([0, 1, 1], dtype=np.uint8)
    st, _ = run_mixed_build(w, off, kinds)
    assert st == wrs.WRS_ERR_INVALID_WEIGHT
