"""The allocation-free build (wrs_alias_build_f32_static_scratch), for callers that cannot
allocate device memory, against the regular build with caller scratch.

Its scratch is a fixed array inside the library, shared by every call on a device and kept
between calls, so the test makes two calls in a row with different inputs and sizes and
checks each table bit for bit against the regular entry point's (the tolerance of the other
build tests: identical rows). This file is collected last so that a run stopping at the
first failure has run every other test; it also passes alone in a fresh process."""
import numpy as np
import pytest
import torch

import wrs

pytestmark = pytest.mark.gpu

MAX_ITEMS = 1 << 18


def weights(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        return rng.random(n, dtype=np.float32)
    return (np.arange(1, n + 1, dtype=np.float64) ** -1.1).astype(np.float32)[rng.permutation(n)]


def regular_build(w, opts):
    n = w.numel()
    table = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    W = torch.zeros(1, dtype=torch.float64, device="cuda")
    scratch = torch.empty(wrs.alias_build_scratch_bytes(n, opts), dtype=torch.uint8, device="cuda")
    assert wrs.alias_build(w, table, scratch, opts, W) == wrs.WRS_SUCCESS
    torch.cuda.synchronize()
    return table.cpu().numpy(), W.item()


def static_build(w, opts):
    n = w.numel()
    table = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    W = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = wrs.alias_build_static_scratch(w, table, opts, W)
    torch.cuda.synchronize()
    return st, table.cpu().numpy(), W.item()


@pytest.mark.parametrize("tile", [0, 1024, 4096])
def test_static_scratch_build_matches_regular_build_twice(cuda, tile):
    opts = wrs.build_opts(tile_items=tile, sync=True)
    cases = [("powerlaw", MAX_ITEMS, 11), ("uniform", 100_003, 12)]  # two calls in a row
    for kind, n, seed in cases:
        w = torch.from_numpy(weights(kind, n, seed)).cuda()
        st, got, W_got = static_build(w, opts)
        assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
        ref, W_ref = regular_build(w, opts)
        assert W_got == W_ref
        np.testing.assert_array_equal(got, ref)


def test_static_scratch_build_rejects_sizes_beyond_its_limit(cuda):
    w = torch.ones(MAX_ITEMS + 1, dtype=torch.float32, device="cuda")
    table = torch.empty(MAX_ITEMS + 1, dtype=torch.int64, device="cuda")
    assert wrs.alias_build_static_scratch(w, table) == wrs.WRS_ERR_INVALID_ARGUMENT


def test_static_scratch_build_reports_device_errors_with_sync(cuda):
    w = torch.ones(5000, dtype=torch.float32, device="cuda")
    w[10] = float("nan")
    table = torch.empty(5000, dtype=torch.int64, device="cuda")
    assert wrs.alias_build_static_scratch(w, table, wrs.build_opts(sync=True)) == wrs.WRS_ERR_INVALID_WEIGHT
    w[10] = 1.0
    st, got, _ = static_build(w, wrs.build_opts(sync=True))
    assert st == wrs.WRS_SUCCESS
    ref, _ = regular_build(w, wrs.build_opts(sync=True))
    np.testing.assert_array_equal(got, ref)


def test_static_scratch_psa_plus_matches_regular_build(cuda):
    """PSA+ through the allocation-free entry point, below its documented limit (about
    190,000 items): two calls in a row, each bit for bit the regular PSA+ build."""
    opts = wrs.build_opts(method=wrs.WRS_METHOD_PSA_PLUS, sync=True)
    for kind, n, seed in [("uniform", 150_000, 21), ("powerlaw", 65_537, 22)]:
        w = torch.from_numpy(weights(kind, n, seed)).cuda()
        st, got, W_got = static_build(w, opts)
        assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
        ref, W_ref = regular_build(w, opts)
        assert W_got == W_ref
        np.testing.assert_array_equal(got, ref)


def test_static_scratch_psa_plus_rejects_tables_whose_scratch_exceeds_the_array(cuda):
    """n = 2^18 is within the item limit, but PSA+ needs more than the 8 MiB array holds."""
    opts = wrs.build_opts(method=wrs.WRS_METHOD_PSA_PLUS, sync=True)
    assert wrs.alias_build_scratch_bytes(MAX_ITEMS, opts) > 8 << 20
    w = torch.ones(MAX_ITEMS, dtype=torch.float32, device="cuda")
    table = torch.empty(MAX_ITEMS, dtype=torch.int64, device="cuda")
    assert wrs.alias_build_static_scratch(w, table, opts) == wrs.WRS_ERR_INVALID_ARGUMENT


def test_static_scratch_status_reports_an_error_without_sync(cuda):
    """Without WRS_FLAG_SYNC the call returns at once; the device-side error of that build is
    read afterwards from the library's array, and the next build clears it."""
    w = torch.ones(5000, dtype=torch.float32, device="cuda")
    w[17] = float("nan")
    table = torch.empty(5000, dtype=torch.int64, device="cuda")
    assert wrs.alias_build_static_scratch(w, table) == wrs.WRS_SUCCESS
    assert wrs.static_scratch_status() == wrs.WRS_ERR_INVALID_WEIGHT
    w[17] = 2.0
    assert wrs.alias_build_static_scratch(w, table) == wrs.WRS_SUCCESS
    assert wrs.static_scratch_status() == wrs.WRS_SUCCESS
