"""The reference's own test harness against this library: oracle/_ref/ref_harness (built from
oracle/ref_harness.cu with the reference's headers and sources) drives wrs_alias_build_f32 and
wrs_alias_sample through subclasses of the reference's AliasTable and Sampler classes, on the
case list of the reference's UnitTests (every weight distribution, both build methods and both
row formats, the 505711-item OneLight regression case, 20 random cases from a fixed seed) with
the reference's verifyTableCorrectness as the check, and the sampled distribution against the
reference's expected counts (SamplerCpu and the library's plain and sectioned samplers). Where
the reference's absolute tolerance is below what an FP32 probability can hold at the weights'
own scale, the harness checks the same weights scaled to mean 1 and counts those cases."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HARNESS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_harness")


def test_reference_harness_passes_every_case(cuda):
    if not os.path.exists(HARNESS):
        pytest.skip("oracle/_ref/ref_harness not built (it needs the reference checkout at build time)")
    r = subprocess.run([HARNESS], capture_output=True, text=True, timeout=600)
    failed = [l for l in r.stdout.splitlines() if l.startswith("FAILED")]
    assert r.returncode == 0 and not failed, (failed, r.stderr[-2000:])
    summary = [l for l in r.stdout.splitlines() if l.startswith("cases=")]
    assert summary
    fields = dict(f.split("=") for f in summary[-1].split())
    assert fields["failures"] == "0"
    assert int(fields["cases"]) >= 80
    # only large tables of large weights need the mean-1 scale (the reference's absolute
    # tolerance is finer than an FP32 probability there)
    assert int(fields["scaled"]) <= 12
