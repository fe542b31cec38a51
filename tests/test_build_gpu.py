"""GPU alias build vs the oracle: bit-exact tables against the CPU restatement of the same
exact merge (or_exact_build), per-item probability error against w_i / W, edge cases and
failure reporting (UnitTests::testTableCorrectness, UnitTests.cu:10-94)."""
import os

import numpy as np
import pytest
import torch

import py_oracle as po
import wrs
from gpu_util import gpu_build
from test_oracle_precision import NAMES, gen

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_tables.npz")


def check_parity(w, rows, W):
    ref = po.exact_build(w, W)
    mism = np.nonzero(np.any(rows != ref, axis=1))[0]
    assert mism.size == 0, f"{mism.size} rows differ from the oracle, first {mism[:5]}: {rows[mism[:3]]} vs {ref[mism[:3]]}"
    chk = po.check_table(w, rows)
    assert chk["bad_rows"] == 0 and chk["zero_mass"] == 0, chk
    assert chk["max_rel"] <= 2.5e-7, chk
    return chk


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("n", [1, 2, 3, 17, 2047, 2048, 2049, 100_003, 1 << 20])
def test_build_parity(cuda, name, n):
    w = gen(name, n)
    st, rows, W = gpu_build(w)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    assert W == po.exact_sum(w)
    check_parity(w, rows, W)


@pytest.mark.parametrize("tile", [1024, 2048, 4096])
@pytest.mark.parametrize("name", ["uniform", "powerlaw_shuffled", "loguniform", "near_uniform"])
def test_build_tile_sizes_give_identical_tables(cuda, tile, name):
    w = gen(name, 300_001)
    st, rows, W = gpu_build(w, tile_items=tile)
    assert st == wrs.WRS_SUCCESS
    check_parity(w, rows, W)


@pytest.mark.parametrize("num_tiles", [591, 592, 1182, 1184, 4728, 4729])
def test_build_scan_group_boundaries(cuda, num_tiles):
    # the scan groups fewer tiles per look-back unit while a table has fewer than 592 units of
    # eight (1, 2, 4 or 8 tiles): tables on either side of each switch, with a ragged last tile
    tile = 1024
    n = num_tiles * tile - 7
    w = gen("powerlaw_shuffled", n)
    st, rows, W = gpu_build(w, tile_items=tile)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    check_parity(w, rows, W)


def test_build_reference_generators(cuda):
    g = np.load(GOLDEN)
    for case in ["sine", "bestworst", "ramp", "powerlaw1", "powerlaw2", "oneheavy", "onelight", "uniform_f32"]:
        w = g[f"{case}/w"].astype(np.float32)
        st, rows, W = gpu_build(w)
        assert st == wrs.WRS_SUCCESS
        check_parity(w, rows, W)


def test_build_regression_onelight_505711(cuda):
    w = np.ones(505711, np.float32)
    w[0] = 0.5
    st, rows, W = gpu_build(w)
    assert st == wrs.WRS_SUCCESS
    check_parity(w, rows, W)


def test_build_is_deterministic(cuda):
    w = gen("pareto", 1 << 20)
    a = gpu_build(w)[1]
    b = gpu_build(w)[1]
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("n", [1, 2, 17, 2047, 2049, 100_003, 1 << 20])
@pytest.mark.parametrize("tile", [1024, 2048, 4096])
def test_psa_plus_parity(cuda, name, n, tile):
    """WRS_METHOD_PSA_PLUS: bit-identical to the oracle's PSA+ restatement."""
    w = gen(name, n)
    st, rows, W = gpu_build(w, method=wrs.WRS_METHOD_PSA_PLUS, tile_items=tile)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    ref = po.psa_plus_build(w, W, tile)
    mism = np.nonzero(np.any(rows != ref, axis=1))[0]
    assert mism.size == 0, f"{mism.size} rows differ, first {mism[:5]}: {rows[mism[:3]]} vs {ref[mism[:3]]}"
    chk = po.check_table(w, rows)
    assert chk["bad_rows"] == 0 and chk["zero_mass"] == 0 and chk["max_rel"] <= 2.5e-7, chk


def test_psa_plus_rejects_invalid_weights(cuda):
    w = gen("uniform", 10_000)
    w[77] = np.nan
    st, _, _ = gpu_build(w, method=wrs.WRS_METHOD_PSA_PLUS)
    assert st == wrs.WRS_ERR_INVALID_WEIGHT


@pytest.mark.parametrize("bad", [np.nan, -1.0, np.inf, -np.inf])
def test_build_rejects_invalid_weights_and_recovers(cuda, bad):
    w = gen("uniform", 10_000)
    w[1234] = bad
    st, _, _ = gpu_build(w)
    assert st == wrs.WRS_ERR_INVALID_WEIGHT
    w[1234] = 0.5
    st, rows, W = gpu_build(w)
    assert st == wrs.WRS_SUCCESS
    check_parity(w, rows, W)


def test_build_rejects_all_zero(cuda):
    st, _, _ = gpu_build(np.zeros(5000, np.float32))
    assert st == wrs.WRS_ERR_ZERO_TOTAL


def test_build_unaligned_weights(cuda):
    w = gen("exp", 70_001)
    buf = torch.from_numpy(np.concatenate([[0.0], w]).astype(np.float32)).cuda()
    wv = buf[1:]
    n = wv.numel()
    opts = wrs.build_opts(sync=True)
    table = torch.empty(n, dtype=torch.int64, device="cuda")
    scratch = torch.empty(wrs.alias_build_scratch_bytes(n, opts), dtype=torch.uint8, device="cuda")
    assert wrs.alias_build(wv, table, scratch, opts) == wrs.WRS_SUCCESS
    rows = table.cpu().numpy().view(np.uint32).reshape(-1, 2)
    check_parity(w, rows, po.exact_sum(w))


def test_build_config_sizes_large(cuda):
    # n = 2^24: uniform and the permuted power law of the large-table workload
    n = 1 << 24
    rng = np.random.default_rng(42)
    for w in [rng.random(n, dtype=np.float32),
              (np.arange(1, n + 1, dtype=np.float64) ** -1.1).astype(np.float32)[rng.permutation(n)]]:
        st, rows, W = gpu_build(w)
        assert st == wrs.WRS_SUCCESS
        chk = po.check_table(w, rows)
        assert chk["max_rel"] <= 2.5e-7 and chk["bad_rows"] == 0 and chk["zero_mass"] == 0, chk


def test_reference_shaped_surface(cuda):
    w = gen("uniform", 10_000)
    t = wrs.AliasTableSplitGpu(w)
    assert t.fullBuild()
    assert t.name() == "AliasTableSplitGpu"
    prob, alias = t.aliasTable
    rows = np.stack([prob.view(np.uint32), alias], axis=1)
    check_parity(w, rows, t.W)


@pytest.mark.parametrize("method", [wrs.WRS_METHOD_SPLIT, wrs.WRS_METHOD_PSA_PLUS])
def test_export_reference_format(cuda, method):
    """The table in the reference's TableStorage format passes the reference-format check
    (the per-item restatement of AliasTable::verifyTableCorrectness, AliasTable.cu:24-65)."""
    w = gen("powerlaw_shuffled", 100_003)
    st, rows, W = gpu_build(w, method=method)
    assert st == wrs.WRS_SUCCESS
    table = torch.from_numpy(rows.view(np.int64).reshape(-1)).cuda()
    weight = torch.empty(w.size, dtype=torch.float64, device="cuda")
    alias = torch.empty(w.size, dtype=torch.int32, device="cuda")
    assert wrs.export_reference_table(table, W, weight, alias) == wrs.WRS_SUCCESS
    torch.cuda.synchronize()
    wt, al = weight.cpu().numpy(), alias.cpu().numpy()
    assert np.array_equal(wt, rows[:, 0].view(np.float32).astype(np.float64) * (W / w.size))
    chk = po.check_ref_table(w.astype(np.float64), wt, al, W)
    assert chk["bad_rows"] == 0 and chk["max_rel"] <= 2.5e-7, chk
