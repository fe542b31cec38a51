"""Bounded device waits run out and report WRS_ERR_DEVICE_TIMEOUT, without faulting or hanging
the GPU: a look-back block (split build) or tile (rejection build) is held so that it publishes
nothing, the limit is cut to 1 ms, and the waits of the blocks after it give up. The next build,
with the hold lifted and the default limit back, is bit for bit the oracle's again."""
import time

import numpy as np
import pytest
import torch

import py_oracle as po
import wrs
from gpu_util import gpu_build

pytestmark = pytest.mark.gpu

LIMIT_NS = 1_000_000  # 1 ms


@pytest.fixture
def short_waits(cuda):
    assert wrs.set_device_wait_limit(LIMIT_NS) == wrs.WRS_SUCCESS
    yield
    assert wrs.debug_hold_lookback(-1) == wrs.WRS_SUCCESS
    assert wrs.set_device_wait_limit(0) == wrs.WRS_SUCCESS


def test_split_build_lookback_wait_times_out(short_waits):
    # 2^22 + 5 items: over a thousand tiles, each looking back over its predecessors; tile 0 is
    # held, so the tiles after it wait on a flag that nothing sets
    n = (1 << 22) + 5
    w = np.random.default_rng(3).random(n, dtype=np.float32)
    assert wrs.debug_hold_lookback(0) == wrs.WRS_SUCCESS
    t0 = time.time()
    st, _, _ = gpu_build(w)
    assert st == wrs.WRS_ERR_DEVICE_TIMEOUT, wrs.status_string(st)
    assert time.time() - t0 < 30
    wrs.debug_hold_lookback(-1)
    wrs.set_device_wait_limit(0)
    st, rows, W = gpu_build(w)
    assert st == wrs.WRS_SUCCESS
    np.testing.assert_array_equal(rows, po.exact_build(w, W))


def test_rejection_build_lookback_wait_times_out(short_waits):
    n = 50 * 2048 + 17  # tiles of 2048 items
    w = np.random.default_rng(4).random(n, dtype=np.float32)
    d_w = torch.from_numpy(w).cuda()
    A = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    frac = torch.zeros(n, dtype=torch.float32, device="cuda")
    a_size = torch.zeros(1, dtype=torch.int64, device="cuda")
    W = torch.zeros(1, dtype=torch.float64, device="cuda")
    scratch = torch.empty(wrs.rejection_build_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    assert wrs.debug_hold_lookback(7) == wrs.WRS_SUCCESS
    st = wrs.rejection_build(d_w, A, frac, a_size, scratch, W, sync=True)
    assert st == wrs.WRS_ERR_DEVICE_TIMEOUT, wrs.status_string(st)
    wrs.debug_hold_lookback(-1)
    wrs.set_device_wait_limit(0)
    assert wrs.rejection_build(d_w, A, frac, a_size, scratch, W, sync=True) == wrs.WRS_SUCCESS
    k = int(a_size.item())
    A_ref, frac_ref = po.rejection_build(w, W.item())
    np.testing.assert_array_equal(A[:k].cpu().numpy().view(np.uint32), A_ref)
    np.testing.assert_array_equal(frac.cpu().numpy(), frac_ref)
