"""The exact merge build (CPU restatement) meets the 1e-6 per-item bar on adversarial
inputs: the bound is ~2^-23 + |D|/E_total whatever the distribution."""
import numpy as np
import pytest

import py_oracle as po

RNG = np.random.default_rng(1234)


def gen(name, n):
    if name == "uniform":
        return RNG.random(n, dtype=np.float32)
    if name == "powerlaw_shuffled":
        return (np.arange(1, n + 1, dtype=np.float64) ** -1.1).astype(np.float32)[RNG.permutation(n)]
    if name == "loguniform":
        return (10.0 ** RNG.uniform(-8, 8, n)).astype(np.float32)
    if name == "near_uniform":
        return (1.0 + 1e-6 * RNG.random(n)).astype(np.float32)
    if name == "one_heavy":
        w = np.ones(n, np.float32)
        w[0] = 2.0
        return w
    if name == "one_light":
        w = np.ones(n, np.float32)
        w[0] = 0.5
        return w
    if name == "zeros_mix":
        w = RNG.random(n, dtype=np.float32)
        w[RNG.random(n) < 0.3] = 0
        if not w.any():
            w[0] = 1.0
        return w
    if name == "exp":
        return RNG.exponential(1.0, n).astype(np.float32)
    if name == "pareto":
        return (RNG.pareto(1.5, n) + 1).astype(np.float32)
    if name == "all_equal":
        return np.full(n, 3.0, np.float32)
    if name == "tiny_and_huge":
        w = np.full(n, 1e-30, np.float32)
        w[::97] = 1e30
        return w
    raise ValueError(name)


NAMES = ["uniform", "powerlaw_shuffled", "loguniform", "near_uniform", "one_heavy", "one_light", "zeros_mix",
         "exp", "pareto", "all_equal"]


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("n", [1, 2, 3, 17, 1000, 100_003])
def test_exact_build_per_item_error(name, n):
    w = gen(name, n)
    rows = po.exact_build(w)
    chk = po.check_table(w, rows)
    assert chk["bad_rows"] == 0 and chk["zero_mass"] == 0
    assert chk["max_rel"] <= 2.5e-7, chk


def test_exact_build_zero_weight_items_get_no_mass():
    w = np.array([0, 1, 0, 3, 0, 0.5], np.float32)
    rows = po.exact_build(w)
    chk = po.check_table(w, rows)
    assert chk["zero_mass"] == 0 and chk["max_rel"] < 1e-7


def test_exact_build_regression_onelight_505711():
    # UnitTests.cu:47-49: n=505711 OneLight, "a group with 0 threads eligible for packing"
    w = np.ones(505711, np.float32)
    w[0] = 0.5
    chk = po.check_table(w, po.exact_build(w))
    assert chk["max_rel"] <= 2.5e-7


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("n", [1, 2, 3, 17, 1000, 2049, 100_003])
@pytest.mark.parametrize("tile", [1024, 2048])
def test_psa_plus_build_per_item_error(name, n, tile):
    """The PSA+ restatement (tile-local pre-pack, then the exact merge of the leftovers;
    AliasTableSplitGpu::psaPlus, AliasTableSplitGpu.cu:342-386) is a valid table with the
    split method's error bound."""
    w = gen(name, n)
    rows = po.psa_plus_build(w, tile=tile)
    chk = po.check_table(w, rows)
    assert chk["bad_rows"] == 0 and chk["zero_mass"] == 0
    assert chk["max_rel"] <= 2.5e-7, chk


def test_psa_plus_pairs_locally():
    """PSA+ resolves most items inside their own tile: the aliases of its light rows point
    into the same tile far more often than the split method's do."""
    w = gen("uniform", 1 << 16)
    W = po.exact_sum(w)
    n = w.size
    light = w <= W / n
    same = lambda rows: np.mean((rows[light, 1] // 2048) == (np.nonzero(light)[0] // 2048))
    local, split = same(po.psa_plus_build(w, W, 2048)), same(po.exact_build(w, W))
    assert local > 0.95 and local > split, (local, split)


@pytest.mark.skipif(not po.ref_available(debug=True), reason="the compiled reference (oracle/_ref) is not built")
@pytest.mark.parametrize("name,n", [("uniform", 10_000), ("powerlaw_shuffled", 100_003), ("loguniform", 50_000),
                                    ("one_heavy", 4097), ("one_light", 505_711), ("zeros_mix", 30_000),
                                    ("pareto", 65_536), ("all_equal", 1000)])
def test_reference_verifier_accepts_the_tables(name, n):
    """The reference's own AliasTable::verifyTableCorrectness (AliasTable.cu:24-65, compiled from
    its sources, debug build) accepts this library's tables in the reference's row format
    (weight = prob * W/N in FP64, as wrs_export_reference_table writes them). The tables are the
    oracle's, which the GPU build reproduces bit for bit. The reference's check is absolute
    (every item within max(N 1e-8, 1e-3) of its weight), so the log-uniform weights, which reach
    1e8, are scaled to mean 1 first: at their own scale no FP32-probability table passes it."""
    w = gen(name, n)
    if name == "loguniform":
        w = (w.astype(np.float64) / w.astype(np.float64).mean()).astype(np.float32)
    rows = po.exact_build(w)
    W = po.exact_sum(w)
    weight = rows[:, 0].view(np.float32).astype(np.float64) * (W / n)
    alias = rows[:, 1].astype(np.int32)
    assert po.ref_verify(w.astype(np.float64), weight, alias, W)
    # the verifier is live: a quarter of a donating row's mass moved to its alias fails it
    # (where W/N is large enough for the absolute tolerance to notice)
    donors = np.nonzero((alias != np.arange(n)) & (weight > 0.5 * W / n))[0]
    if W / n >= 0.1 and donors.size:
        j = int(donors[0])
        bad = weight.copy()
        bad[j] *= 0.75
        assert not po.ref_verify(w.astype(np.float64), bad, alias, W)


def test_precision_comparison_builds_in_the_oracle():
    """The oracle's all-FP64 / all-FP32 restatements give valid tables; the FP32 lines lose
    accuracy on spread weights, the FP64 lines stay near the stored FP32 rounding."""
    w = gen("loguniform", 1 << 16)
    r64, W64 = po.prec_build(w, True)
    r32, W32 = po.prec_build(w, False)
    assert r64 is not None and r32 is not None
    assert np.all(r64[:, 1] < w.size) and np.all(r32[:, 1] < w.size)
    e64 = po.check_table(w, r64)["max_rel"]
    e32 = po.check_table(w, r32)["max_rel"]
    assert e64 < 1e-6 < e32
    assert po.prec_build(np.zeros(10, np.float32), True)[0] is None
