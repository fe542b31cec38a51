"""Precision comparison of the precision-stress weights (CPU): this library's mixed build
against the reference's FP64 sweep and an all-FP32 sweep, per item against n w_i / W with
W the exact sum. The mixed build's rows are or_exact_build's (equal to the GPU build's, bit
for bit, by the parity tests)."""
import numpy as np

import py_oracle as po
from precision_report import report


def test_report_small():
    r = report(16)
    assert r["mixed"]["max_rel"] <= 1e-6 and r["mixed"]["bad_rows"] == 0
    assert r["all_fp64"]["bad_rows"] == 0
    # the all-FP32 running residual drifts: far above the mixed build's error
    assert r["all_fp32"]["max_rel"] > 100 * r["mixed"]["max_rel"]


def test_fp32_sweep_matches_fp64_on_exact_inputs():
    # small integer weights over a power-of-two count: every sum, W / N and every residual
    # is exact in FP32, so both sweeps build the same table
    rng = np.random.default_rng(3)
    w = rng.integers(1, 16, 1024).astype(np.float32)
    wt32, al32, WN32 = po.sweep_build_f32(w)
    wt64, al64, W64 = po.sweep_build(w.astype(np.float64))
    assert WN32 == W64 / w.size
    assert np.array_equal(al32, al64)
    assert np.array_equal(wt32, wt64)
    c = po.check_ref_table_w(w, wt32, al32, WN32, float(w.astype(np.float64).sum()))
    assert c["bad_rows"] == 0 and c["max_rel"] < 1e-12
