"""GPU samplers vs the oracle: bit-exact sample streams given identical tables and Philox
counters (plain and sectioned), and the sampled distribution (chi-square)."""
import numpy as np
import pytest
import torch

import py_oracle as po
import wrs
from gpu_util import gpu_build, gpu_sample
from test_oracle_precision import gen
from test_oracle_sampling import chi2_pvalue

pytestmark = pytest.mark.gpu
SEED = 0x5EED


@pytest.fixture(scope="module")
def tables(cuda):
    out = {}
    for name, n in [("uniform", 1000), ("powerlaw_shuffled", 100_003), ("one_heavy", 4096), ("loguniform", 1 << 18)]:
        w = gen(name, n)
        st, rows, W = gpu_build(w)
        assert st == 0
        out[name] = (w, rows)
    return out


@pytest.mark.parametrize("name", ["uniform", "powerlaw_shuffled", "one_heavy", "loguniform"])
@pytest.mark.parametrize("m,cbase,off", [(1, 0, 0), (7, 3, 0), (8, 0, 1), (1001, 12345, 3), (1 << 20, 99, 0),
                                         ((1 << 20) + 5, (1 << 40) + 1, 2)])
def test_plain_sampler_bit_exact(tables, name, m, cbase, off):
    w, rows = tables[name]
    st, got, _ = gpu_sample(rows, m, SEED, cbase, out_offset=off)
    assert st == 0
    np.testing.assert_array_equal(got, po.sample_plain(rows, m, SEED, cbase))


@pytest.mark.parametrize("S", [512, 2048, 12288, 65536])
@pytest.mark.parametrize("name", ["uniform", "powerlaw_shuffled", "loguniform"])
def test_sectioned_sampler_bit_exact(tables, name, S):
    w, rows = tables[name]
    m = 1 << 20
    st, got, counts = gpu_sample(rows, m, SEED, 77, mode=wrs.WRS_SAMPLE_SECTIONED, section_items=S)
    assert st == 0
    ref, ref_counts = po.sample_sectioned(rows, m, S, SEED, 77)
    np.testing.assert_array_equal(counts, ref_counts)
    np.testing.assert_array_equal(got, ref)


def test_plain_sampler_distribution_chi2(cuda):
    w = gen("pareto", 1 << 16)
    st, rows, W = gpu_build(w)
    m = 1 << 26
    st, got, _ = gpu_sample(rows, m, 12345)
    counts = np.bincount(got, minlength=w.size)
    assert chi2_pvalue(counts, w.astype(np.float64) / w.sum(dtype=np.float64) * m) > 1e-6


def test_sectioned_sampler_distribution_chi2(cuda):
    w = gen("uniform", 1 << 16)
    st, rows, W = gpu_build(w)
    m = 1 << 26
    st, got, _ = gpu_sample(rows, m, 777, mode=wrs.WRS_SAMPLE_SECTIONED, section_items=4096)
    counts = np.bincount(got, minlength=w.size)
    assert chi2_pvalue(counts, w.astype(np.float64) / w.sum(dtype=np.float64) * m) > 1e-6


def test_reference_shaped_samplers(cuda):
    w = gen("uniform", 10_000)
    t = wrs.AliasTableSplitGpu(w)
    t.fullBuild()
    for s in [wrs.SamplerGpuBasic(t), wrs.SamplerGpuSectioned(t, 2500)]:
        dist = s.getSamplingDistribution(2_000_000)
        assert dist.sum() == 2_000_000
        assert chi2_pvalue(dist, w / w.sum(dtype=np.float64) * 2_000_000) > 1e-6
        assert s.benchmarkSampling(1 << 20) > 0


@pytest.mark.parametrize("m,chunk,cbase", [(1, 0, 0), (1001, 64, 7), (1001, 63, 8), ((1 << 20) + 5, 1 << 17, 99),
                                           (3 << 20, 0, (1 << 40) + 1)])
def test_sample_to_host_bit_exact(tables, m, chunk, cbase):
    # chunked sampling with overlapped copies gives the plain sampler's stream, in pinned memory;
    # two calls in a row on the same buffers (the second must wait for the first's copies)
    w, rows = tables["powerlaw_shuffled"]
    table = torch.from_numpy(np.ascontiguousarray(rows).view(np.int64).reshape(-1)).cuda()
    out = torch.empty(m, dtype=torch.int32, device="cuda")
    host = torch.full((m,), -1, dtype=torch.int32).pin_memory()
    for rep in range(2):
        c = cbase + rep * m
        st = wrs.alias_sample_to_host(table, rows.shape[0], m, SEED, out, host, c, chunk)
        assert st == 0
        torch.cuda.current_stream().synchronize()
        np.testing.assert_array_equal(host.numpy().view(np.uint32), po.sample_plain(rows, m, SEED, c))


@pytest.mark.parametrize("m,cbase", [(1, 0), (1001, 7), ((1 << 20) + 5, 99)])
def test_histogram_mode_counts_plain_samples(tables, m, cbase):
    # the counts of the histogram mode are the bin counts of the plain sampler's output
    w, rows = tables["powerlaw_shuffled"]
    n = rows.shape[0]
    table = torch.from_numpy(np.ascontiguousarray(rows).view(np.int64).reshape(-1)).cuda()
    counts = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert wrs.alias_histogram(table, n, m, SEED, counts, cbase) == 0
    torch.cuda.synchronize()
    ref = np.bincount(po.sample_plain(rows, m, SEED, cbase), minlength=n)
    np.testing.assert_array_equal(counts.cpu().numpy(), ref)


@pytest.mark.parametrize("m,cbase", [(1, 0), (1001, 7), ((1 << 20) + 5, 99)])
def test_discard_mode_folds_plain_samples(tables, m, cbase):
    # the discard mode draws the plain samples and keeps only their XOR (folded into out[0])
    w, rows = tables["uniform"]
    n = rows.shape[0]
    table = torch.from_numpy(np.ascontiguousarray(rows).view(np.int64).reshape(-1)).cuda()
    out = torch.full((2,), 0x1234, dtype=torch.int32, device="cuda")
    assert wrs.alias_sample(table, n, m, SEED, out[:1], cbase, mode=wrs.WRS_SAMPLE_DISCARD) == 0
    torch.cuda.synchronize()
    ref = np.bitwise_xor.reduce(po.sample_plain(rows, m, SEED, cbase).astype(np.uint32)) ^ np.uint32(0x1234)
    got = out.cpu().numpy().view(np.uint32)
    assert got[0] == ref and got[1] == 0x1234
