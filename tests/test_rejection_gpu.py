"""GPU rejection sampling vs the oracle: the slot array, acceptance fractions and |A| equal
the CPU restatement of RejectionSampling::build + fillA; samples equal the restatement of
SamplerRejection::sample under the same Philox counters, give-up outputs included."""
import numpy as np
import pytest
import torch

import py_oracle as po
import wrs
from gpu_util import to_dev, alloc_scratch
from test_oracle_precision import gen
from test_oracle_sampling import chi2_pvalue

pytestmark = pytest.mark.gpu
SEED = 0xFEED


def gpu_rej_build(w):
    n = w.size
    wd = to_dev(w)
    A = torch.full((2 * n + 2,), -1, dtype=torch.int32, device="cuda")
    frac = torch.empty(n, dtype=torch.float32, device="cuda")
    asz = torch.zeros(1, dtype=torch.int64, device="cuda")
    W = torch.zeros(1, dtype=torch.float64, device="cuda")
    scratch = alloc_scratch(wrs.rejection_build_scratch_bytes(n))
    st = wrs.rejection_build(wd, A, frac, asz, scratch, W, sync=True)
    return st, A, frac, asz, float(W.item())


def big_items(n):
    w = np.random.default_rng(5).random(n, dtype=np.float32)
    w[17] = 3e4          # thousands of slots: deferred, warp-filled
    w[n // 2] = 3e5      # more than 2^16 slots: filled by the whole grid
    return w


def many_huge_items(n):
    # several items of more than 2^16 slots (chunked over the grid) and of 2^16 or fewer
    w = np.random.default_rng(6).random(n, dtype=np.float32)
    for k, v in enumerate([4e5, 2e5, 1.5e5, 9e4, 7e4, 2e4, 5e3]):
        w[(k * 7919) % n] = v
    return w


@pytest.mark.parametrize("maker", [lambda: gen("uniform", 1000), lambda: many_huge_items(500_000), lambda: gen("pareto", 100_003),
                                   lambda: gen("zeros_mix", 50_000), lambda: gen("powerlaw_shuffled", 1 << 20),
                                   lambda: big_items(300_000), lambda: np.ones(1, np.float32)])
def test_rejection_build_bit_exact(cuda, maker):
    w = maker()
    st, A, frac, asz, W = gpu_rej_build(w)
    assert st == 0, wrs.status_string(st)
    A_ref, frac_ref = po.rejection_build(w, W)
    assert int(asz.item()) == A_ref.size
    np.testing.assert_array_equal(A[:A_ref.size].cpu().numpy().view(np.uint32), A_ref)
    np.testing.assert_array_equal(frac.cpu().numpy(), frac_ref)


@pytest.mark.parametrize("max_tries", [0, 1, 2])
def test_rejection_sample_bit_exact(cuda, max_tries):
    w = gen("pareto", 20_000)
    st, A, frac, asz, W = gpu_rej_build(w)
    m = 300_001
    out = torch.empty(m, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = wrs.rejection_sample(A, asz, frac, w.size, m, SEED, out, 5, max_tries, status, sync=True)
    A_ref, frac_ref = po.rejection_build(w, W)
    ref, failed = po.rejection_sample(A_ref, frac_ref, m, SEED, 5, max_tries)
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), ref)
    if failed:
        assert st == wrs.WRS_ERR_TOO_MANY_TRIES
    else:
        assert st == 0


def packed(A, asz, frac, n, capacity=None):
    slots = torch.full((capacity if capacity is not None else int(asz.item()),), -1, dtype=torch.int64, device="cuda")
    assert wrs.rejection_pack(A, asz, frac, n, slots) == wrs.WRS_SUCCESS
    torch.cuda.synchronize()
    return slots


@pytest.mark.parametrize("maker", [lambda: gen("pareto", 20_000), lambda: big_items(70_001)])
def test_rejection_pack_layout(cuda, maker):
    w = maker()
    st, A, frac, asz, W = gpu_rej_build(w)
    assert st == 0
    k = int(asz.item())
    slots = packed(A, asz, frac, w.size).cpu().numpy().view(np.uint32).reshape(-1, 2)
    a = A[:k].cpu().numpy().view(np.uint32)
    f = frac.cpu().numpy()
    np.testing.assert_array_equal(slots[:, 0], a)
    first = (a >> 31) != 0
    expect = np.where(first, f[a & 0x7FFFFFFF].view(np.uint32), 0).astype(np.uint32)
    np.testing.assert_array_equal(slots[:, 1], expect)


@pytest.mark.parametrize("m", [300_001, 4, 3, 1])
@pytest.mark.parametrize("max_tries", [0, 1, 2])
def test_rejection_sample_packed_equals_unpacked(cuda, max_tries, m):
    # the same tries and decisions: bit for bit the oracle's samples, give-ups and status included
    w = gen("pareto", 20_000)
    st, A, frac, asz, W = gpu_rej_build(w)
    slots = packed(A, asz, frac, w.size)
    out = torch.empty(m, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = wrs.rejection_sample_packed(slots, asz, w.size, m, SEED, out, 5, max_tries, status, sync=True)
    A_ref, frac_ref = po.rejection_build(w, W)
    ref, failed = po.rejection_sample(A_ref, frac_ref, m, SEED, 5, max_tries)
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), ref)
    assert st == (wrs.WRS_ERR_TOO_MANY_TRIES if failed else 0)


@pytest.mark.parametrize("maker", [lambda: big_items(70_001), lambda: many_huge_items(500_000)])
def test_rejection_sample_packed_huge_items(cuda, maker):
    # items of thousands and of more than 2^16 slots; more samples than one chunk per CTA
    w = maker()
    st, A, frac, asz, W = gpu_rej_build(w)
    assert st == 0
    slots = packed(A, asz, frac, w.size)
    m = 1_000_003
    out = torch.empty(m, dtype=torch.int32, device="cuda")
    ref_out = torch.empty(m, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert wrs.rejection_sample_packed(slots, asz, w.size, m, SEED, out, 11, 3, status, sync=True) in (0, wrs.WRS_ERR_TOO_MANY_TRIES)
    st_ref = wrs.rejection_sample(A, asz, frac, w.size, m, SEED, ref_out, 11, 3, None, sync=True)
    assert st_ref == 0
    assert torch.equal(out, ref_out)


def test_rejection_sample_packed_slot_capacity(cuda):
    w = gen("uniform", 5_000)
    st, A, frac, asz, W = gpu_rej_build(w)
    slots = packed(A, asz, frac, w.size, capacity=int(asz.item()) - 1)
    out = torch.zeros(1000, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = wrs.rejection_sample_packed(slots, asz, w.size, 1000, SEED, out, 0, 0, status, sync=True)
    assert st == wrs.WRS_ERR_CAPACITY
    assert (out.cpu().numpy().view(np.uint32) == 0xFFFFFFFF).all()


def test_rejection_distribution(cuda):
    w = gen("exp", 1 << 14)
    st, A, frac, asz, W = gpu_rej_build(w)
    m = 1 << 24
    out = torch.empty(m, dtype=torch.int32, device="cuda")
    assert wrs.rejection_sample(A, asz, frac, w.size, m, 3, out, sync=True) == 0
    counts = np.bincount(out.cpu().numpy(), minlength=w.size)
    assert chi2_pvalue(counts, w.astype(np.float64) / w.sum(dtype=np.float64) * m) > 1e-6


def test_rejection_capacity_error(cuda):
    w = gen("uniform", 10_000)
    wd = to_dev(w)
    A = torch.empty(100, dtype=torch.int32, device="cuda")
    frac = torch.empty(w.size, dtype=torch.float32, device="cuda")
    asz = torch.zeros(1, dtype=torch.int64, device="cuda")
    scratch = alloc_scratch(wrs.rejection_build_scratch_bytes(w.size))
    assert wrs.rejection_build(wd, A, frac, asz, scratch, sync=True) == wrs.WRS_ERR_CAPACITY


def test_reference_shaped_rejection(cuda):
    w = gen("uniform", 10_000)
    r = wrs.RejectionSamplingGpu(w)
    assert r.fullBuild()
    dist = wrs.SamplerRejection(r).getSamplingDistribution(2_000_000)
    assert chi2_pvalue(dist, w / w.sum(dtype=np.float64) * 2_000_000) > 1e-6
