"""The bench's reference arm (ReferenceCpuPath) on a small table, on the CPU: the reference's
build gives a correct table, the all-core sampler draws exactly the oracle's samples of that
table (the plain contract's Philox stream), and the step reports both timings."""
import os
import sys

import numpy as np
import pytest

import py_oracle as po

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
import bench  # noqa: E402


@pytest.mark.skipif(not po.ref_available(), reason="compiled reference absent")
def test_reference_cpu_path_builds_and_samples_the_contract():
    n, m = 1 << 16, 1 << 16
    w = bench.make_weights(n, seed=3)
    ref = bench.ReferenceCpuPath(w, m, threads=4)
    assert ref.kind == "reference"
    tb, ts = ref.step()
    assert tb > 0 and ts > 0
    chk = po.check_ref_table(w.astype(np.float64), ref.weight, ref.alias, ref.W)
    assert chk["max_rel"] < 1e-6
    np.testing.assert_array_equal(ref.out[:m], po.sample_plain(ref.rows, m, bench.SEED_SAMPLES, 0))


def test_cpu_baseline_line_shape():
    w = bench.make_weights(1 << 15, seed=4)
    c = bench.cpu_baseline(w, m_total=1 << 20, m_sample=1 << 14)
    assert c["kind"] in ("reference", "port") and c["cores"] >= 1
    assert c["value"] > 0 and c["step_s"] > 0
