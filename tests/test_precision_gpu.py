"""The all-FP64 and all-FP32 comparison builds (WRS_PRECISION_FP64 / _FP32) on the GPU, bit
for bit against the oracle's restatement of them (the same merge and the same summation
order), and their place in the precision comparison: on the precision stress weights the
FP32 lines lose accuracy that the default (exact-line) build keeps."""
import numpy as np
import pytest
import torch

import py_oracle as po
import wrs
from gpu_util import alloc_scratch, to_dev
from test_oracle_precision import gen

pytestmark = pytest.mark.gpu


def gpu_build_prec(w_np, precision):
    w = to_dev(np.asarray(w_np, dtype=np.float32))
    n = w.numel()
    opts = wrs.build_opts(precision=precision, sync=True)
    table = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    scratch = alloc_scratch(wrs.alias_build_scratch_bytes(n, opts))
    W = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = wrs.alias_build(w, table, scratch, opts, W)
    torch.cuda.synchronize()
    return st, table.cpu().numpy().view(np.uint32).reshape(-1, 2).copy(), float(W.item())


NAMES = ["uniform", "powerlaw_shuffled", "loguniform", "near_uniform", "one_heavy", "one_light", "zeros_mix", "exp",
         "pareto", "all_equal", "tiny_and_huge"]


@pytest.mark.parametrize("precision", [wrs.WRS_PRECISION_FP64, wrs.WRS_PRECISION_FP32])
@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("n", [1, 7, 2048, 2049, 100_003])
def test_precision_build_matches_oracle(cuda, precision, name, n):
    w = gen(name, n)
    if not np.any(w > 0):
        w[0] = 1.0
    st, rows, W = gpu_build_prec(w, precision)
    ref, W_ref = po.prec_build(w, precision == wrs.WRS_PRECISION_FP64)
    assert st == wrs.WRS_SUCCESS, wrs.status_string(st)
    assert W == W_ref
    np.testing.assert_array_equal(rows, ref)


@pytest.mark.parametrize("precision", [wrs.WRS_PRECISION_FP64, wrs.WRS_PRECISION_FP32])
def test_precision_build_large_matches_oracle(cuda, precision):
    n = (1 << 22) + 3  # more than 1024 tiles: the chunked tile order
    w = gen("loguniform", n)
    st, rows, W = gpu_build_prec(w, precision)
    ref, W_ref = po.prec_build(w, precision == wrs.WRS_PRECISION_FP64)
    assert st == wrs.WRS_SUCCESS
    assert W == W_ref
    np.testing.assert_array_equal(rows, ref)


def test_precision_comparison_orders_the_modes(cuda):
    """On log-uniform weights over 16 decades the FP32 lines lose accuracy by orders of
    magnitude; the FP64 lines and the exact lines stay near the FP32 rounding of the stored
    probabilities."""
    w = gen("loguniform", 1 << 20)
    errs = {}
    for p in (wrs.WRS_PRECISION_MIXED, wrs.WRS_PRECISION_FP64, wrs.WRS_PRECISION_FP32):
        st, rows, _ = gpu_build_prec(w, p)
        assert st == wrs.WRS_SUCCESS
        errs[p] = po.check_table(w, rows)["max_rel"]
    assert errs[wrs.WRS_PRECISION_MIXED] < 2.5e-7
    assert errs[wrs.WRS_PRECISION_FP64] < 1e-6
    assert errs[wrs.WRS_PRECISION_FP32] > 100 * errs[wrs.WRS_PRECISION_MIXED]


def test_precision_build_rejects_bad_input(cuda):
    w = np.ones(5000, dtype=np.float32)
    w[3] = np.nan
    st, _, _ = gpu_build_prec(w, wrs.WRS_PRECISION_FP64)
    assert st == wrs.WRS_ERR_INVALID_WEIGHT
    st, _, _ = gpu_build_prec(np.zeros(100, np.float32), wrs.WRS_PRECISION_FP32)
    assert st == wrs.WRS_ERR_ZERO_TOTAL
