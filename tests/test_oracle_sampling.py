"""CPU checks of the sampling oracle: the binomial tree behind sectioned sampling is an
exact binomial / multinomial, and the plain, sectioned and rejection samplers draw from
w_i / W (cf. UnitTests::testSamplingDistribution, UnitTests.cu:96-145, with a chi-square
test instead of the reference's |diff| < numSamples/tableSize)."""
import numpy as np
import pytest
from scipy import stats

import py_oracle as po

SEED = 0x5EED


def chi2_pvalue(counts, expected, min_expected=32.0):
    """Chi-square p-value with bins merged (in index order) until each expects >= 32."""
    counts = np.asarray(counts, dtype=np.float64)
    expected = np.asarray(expected, dtype=np.float64)
    oc, ec = [], []
    co = ce = 0.0
    for c, e in zip(counts, expected):
        co += c
        ce += e
        if ce >= min_expected:
            oc.append(co)
            ec.append(ce)
            co = ce = 0.0
    if ce > 0:
        if ec:
            oc[-1] += co
            ec[-1] += ce
        else:
            oc.append(co)
            ec.append(ce)
    oc, ec = np.array(oc), np.array(ec)
    if len(oc) < 2:
        return 1.0
    stat = ((oc - ec) ** 2 / ec).sum()
    return float(stats.chi2.sf(stat, len(oc) - 1))


@pytest.mark.parametrize("n,p", [(20, 0.3), (1000, 0.5), (5000, 0.01), (100, 0.9), (400, 0.02), (60, 0.25),
                                 (100_000, 0.37), (1_000_000, 1e-5)])
def test_binomial_matches_pmf(n, p):
    draws = np.array([po.binomial(n, p, SEED, 7, node) for node in range(1, 20001)])
    assert draws.min() >= 0 and draws.max() <= n
    ks = np.arange(n + 1)
    pmf = stats.binom.pmf(ks, n, p)
    counts = np.bincount(draws, minlength=n + 1)
    assert chi2_pvalue(counts, pmf * draws.size) > 1e-4


def test_binomial_large_n_moments():
    n, p = 1 << 30, 0.5
    draws = np.array([po.binomial(n, p, SEED, 11, node) for node in range(1, 20001)], dtype=np.float64)
    z_mean = (draws.mean() - n * p) / np.sqrt(n * p * (1 - p) / draws.size)
    assert abs(z_mean) < 5
    var_ratio = draws.var() / (n * p * (1 - p))
    assert 0.95 < var_ratio < 1.05


def test_binomial_deterministic_and_edge_cases():
    assert po.binomial(0, 0.5, SEED, 0, 1) == 0
    assert po.binomial(10, 0.0, SEED, 0, 1) == 0
    assert po.binomial(10, 1.0, SEED, 0, 1) == 10
    assert po.binomial(1 << 20, 0.5, SEED, 3, 5) == po.binomial(1 << 20, 0.5, SEED, 3, 5)


def test_section_counts_multinomial():
    n, S, m = 1000, 100, 2000
    tot = []
    for cb in range(400):
        c = po.section_counts(n, S, m, SEED, cb * 1000)
        assert int(c.sum()) == m
        tot.append(c)
    tot = np.array(tot, dtype=np.float64)
    # each section ~ Binomial(m, 1/10): per-section mean and variance
    z = (tot.mean(axis=0) - m / 10) / np.sqrt(m * 0.1 * 0.9 / tot.shape[0])
    assert np.all(np.abs(z) < 5)
    # ragged last section
    c = po.section_counts(1050, 100, 10_000, SEED)
    assert c.size == 11 and int(c.sum()) == 10_000


def _weights(n, seed=3):
    rng = np.random.default_rng(seed)
    return rng.random(n, dtype=np.float32)


def test_plain_sampler_distribution():
    w = _weights(1000)
    rows = po.exact_build(w)
    out = po.sample_plain(rows, 400_000, SEED, 0)
    assert out.max() < w.size
    counts = np.bincount(out, minlength=w.size)
    assert chi2_pvalue(counts, w / w.sum(dtype=np.float64) * out.size) > 1e-4


def test_plain_sampler_counter_continuation():
    w = _weights(333)
    rows = po.exact_build(w)
    a = po.sample_plain(rows, 1000, SEED, 0)
    b = po.sample_plain(rows, 600, SEED, 0)
    c = po.sample_plain(rows, 400, SEED, 600)
    np.testing.assert_array_equal(a, np.concatenate([b, c]))


def _contract_sample(rows, start, length, b, seed):
    """One output position of the sampling contract in include/wrs.h, in plain Python:
    Philox block b, row = floor((x1:x0) * length / 2^64) + start, coin = (x2 >> 8) 2^-24."""
    x = po.philox([b & 0xFFFFFFFF, b >> 32, 0, 0], [seed & 0xFFFFFFFF, seed >> 32])
    row = start + ((((int(x[1]) << 32) | int(x[0])) * length) >> 64)
    p = rows[row, 0].view(np.float32)
    coin = np.float32((int(x[2]) >> 8) * 2.0 ** -24)
    return row if coin < p else int(rows[row, 1])


@pytest.mark.parametrize("n", [1, 7, 5003])
def test_plain_and_sectioned_follow_the_written_contract(n):
    """The oracle's samplers against a plain-Python reading of the contract, on table sizes that
    are not powers of two (where a 32-bit row uniform would be biased)."""
    rng = np.random.default_rng(n)
    w = rng.random(n, dtype=np.float32) + np.float32(0.01)
    rows = po.exact_build(w)
    seed, cbase, m = 0x1234_5678_9ABC_DEF0, (1 << 32) - 5, 300
    out = po.sample_plain(rows, m, seed, cbase)
    assert [int(v) for v in out] == [_contract_sample(rows, 0, n, cbase + s, seed) for s in range(m)]
    S = 64
    sect, counts = po.sample_sectioned(rows, m, S, seed, cbase)
    assert int(counts.sum()) == m
    s = 0
    for k, c in enumerate(counts):
        start = k * S
        length = min(S, n - start)
        for _ in range(int(c)):
            assert int(sect[s]) == _contract_sample(rows, start, length, cbase + s, seed)
            s += 1


def test_sectioned_sampler_distribution():
    w = _weights(5000)
    rows = po.exact_build(w)
    out, counts_sec = po.sample_sectioned(rows, 300_000, 512, SEED)
    assert int(counts_sec.sum()) == out.size
    counts = np.bincount(out, minlength=w.size)
    assert chi2_pvalue(counts, w / w.sum(dtype=np.float64) * out.size) > 1e-4
    # samples of section k lie in section k's rows (or are aliases of them)
    np.testing.assert_array_equal(counts_sec, po.section_counts(5000, 512, 300_000, SEED))


def test_rejection_structure_and_distribution():
    rng = np.random.default_rng(9)
    w = (rng.pareto(1.5, 2000) + 0.01).astype(np.float32)
    w[::50] = 0.0
    A, frac = po.rejection_build(w)
    n = w.size
    assert A.size <= 2 * n
    items = A & 0x7FFFFFFF
    assert np.all(np.diff(items.astype(np.int64)) >= 0)
    first = (A >> 31).astype(bool)
    assert first.sum() == n
    slots = np.bincount(items, minlength=n)
    W = po.exact_sum(w)
    x = n * w.astype(np.float64) / W
    np.testing.assert_array_equal(slots, np.floor(x).astype(np.int64) + 1)
    np.testing.assert_allclose(slots - 1 + frac.astype(np.float64), x, rtol=1e-6, atol=1e-7)
    out, failed = po.rejection_sample(A, frac, 300_000, SEED)
    assert failed == 0
    counts = np.bincount(out, minlength=n)
    assert counts[w == 0].sum() == 0
    assert chi2_pvalue(counts, w / w.sum(dtype=np.float64) * out.size) > 1e-4


def test_philox_is_a_function_of_counter_and_key():
    a = po.philox([0, 0, 0, 0], [0, 0])
    b = po.philox([1, 0, 0, 0], [0, 0])
    c = po.philox([0, 0, 0, 0], [1, 0])
    assert not np.array_equal(a, b) and not np.array_equal(a, c)
    np.testing.assert_array_equal(a, po.philox([0, 0, 0, 0], [0, 0]))


def test_philox_matches_curand_golden():
    """The oracle's Philox4x32-10 against cuRAND's outputs (tests/golden/philox_curand.json,
    written on a GPU machine by tests/golden/make_philox_golden.py)."""
    import json
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "philox_curand.json")
    if not os.path.exists(path):
        pytest.skip("philox_curand.json not generated yet")
    cases = json.load(open(path))
    assert cases
    for c in cases:
        seed, sub, off = c["seed"], c["subsequence"], c["offset"]
        key = [seed & 0xFFFFFFFF, seed >> 32]
        for i, expect in enumerate(c["outputs"]):
            b = off // 4 + i
            ctr = [b & 0xFFFFFFFF, (b >> 32) & 0xFFFFFFFF, sub & 0xFFFFFFFF, sub >> 32]
            np.testing.assert_array_equal(po.philox(ctr, key), np.array(expect, dtype=np.uint32))


def test_batched_oracle_matches_per_table_oracle():
    """or_batched_build / or_batched_sample restate the per-table build and the plain
    contract over global output positions."""
    rng = np.random.default_rng(9)
    sizes = np.array([3, 0, 40, 1, 700, 5], dtype=np.int64)
    off = np.zeros(sizes.size + 1, dtype=np.int64)
    np.cumsum(sizes, out=off[1:])
    w = rng.random(int(off[-1]), dtype=np.float32)
    rows, W, bad = po.batched_build(w, off)
    assert bad == 0
    for t in range(sizes.size):
        a, b = off[t], off[t + 1]
        if b > a:
            assert W[t] == po.exact_sum(w[a:b])
            assert np.array_equal(rows[a:b], po.exact_build(w[a:b], W[t]))
    # one table alone: the batched sampler is the plain sampler
    r = rows[off[4]:off[5]]
    assert np.array_equal(po.batched_sample(r, np.array([0, 700]), np.array([0, 1001]), 99, 5),
                          po.sample_plain(r, 1001, 99, 5))
    # odd split points: position s draws Philox block s, whichever table it falls in
    counts = np.array([7, 0, 9, 1, 33, 2], dtype=np.int64)
    soff = np.zeros(sizes.size + 1, dtype=np.int64)
    np.cumsum(counts, out=soff[1:])
    out = po.batched_sample(rows, off, soff, 5, 0)
    for t in range(sizes.size):
        n = int(sizes[t])
        for s in range(soff[t], soff[t + 1]):
            x = po.philox([s & 0xffffffff, s >> 32, 0, 0], [5, 0])
            row = (((int(x[1]) << 32) | int(x[0])) * n) >> 64
            p = rows[off[t] + row, 0].view(np.float32)
            coin = np.float32((int(x[2]) >> 8) * 2.0 ** -24)
            assert out[s] == (row if coin < p else rows[off[t] + row, 1])


@pytest.mark.skipif(not po.ref_available(), reason="the compiled reference (oracle/_ref) is not built")
def test_reference_sampler_draws_from_the_tables():
    """The reference's own CPU sampler (SamplerCpu::sample, SamplerCpu.cu:12-18, compiled from its
    sources) driven by this library's table in the reference's row format draws from w_i / W."""
    rng = np.random.default_rng(31)
    n = 1000
    w = (rng.pareto(1.5, n) + 1.0).astype(np.float32)
    rows = po.exact_build(w)
    W = po.exact_sum(w)
    weight = rows[:, 0].view(np.float32).astype(np.float64) * (W / n)
    alias = rows[:, 1].astype(np.int32)
    _, out = po.ref_sampler_cpu(weight, alias, W, 1_000_000, want_out=True)
    assert out.min() >= 0 and out.max() < n
    counts = np.bincount(out, minlength=n)
    assert chi2_pvalue(counts, w.astype(np.float64) / W * out.size) > 1e-4
