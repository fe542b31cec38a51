"""The CPU oracle against the reference's own outputs (golden fixtures from the compiled
reference, tests/golden/make_golden.py) and known answers.

Mirrors the reference's self-checks: UnitTests::testTableCorrectness (UnitTests.cu:10-94,
all generators x Sweep/Split/Stack) and Adder::unitTest (utils/Adder.cu:159-171)."""
import os

import numpy as np
import pytest

import py_oracle as po

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_tables.npz")
CASES = ["sine", "bestworst", "ramp", "powerlaw1", "powerlaw2", "oneheavy", "onelight", "uniform_f32"]


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("case", CASES)
def test_sweep_restatement_matches_reference(golden, case):
    w = golden[f"{case}/w"]
    wt, al, W = po.sweep_build(w)
    assert W == golden[f"{case}/sweep_W"]
    np.testing.assert_array_equal(wt, golden[f"{case}/sweep_weight"])
    np.testing.assert_array_equal(al, golden[f"{case}/sweep_alias"])


@pytest.mark.parametrize("case", [c for c in CASES if c != "bestworst"])
def test_split_restatement_matches_reference(golden, case):
    w = golden[f"{case}/w"]
    wt, al, W, rc = po.split_build(w, 16)
    assert rc == 0
    assert W == golden[f"{case}/split_W"]
    np.testing.assert_array_equal(wt, golden[f"{case}/split_weight"])
    np.testing.assert_array_equal(al, golden[f"{case}/split_alias"])


def test_split_restatement_flags_nonterminating_reference_case(golden):
    # BestWorstCase: the reference's split search cannot find a split (it loops forever in a
    # Release build); the restatement bounds the search and reports it.
    _, _, _, rc = po.split_build(golden["bestworst/w"], 16)
    assert rc != 0


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("kind", ["sweep", "split", "stack"])
def test_reference_tables_reconstruct_weights(golden, case, kind):
    if kind == "split" and case == "bestworst":
        pytest.skip("reference split build does not terminate on BestWorstCase")
    w = golden[f"{case}/w"]
    chk = po.check_ref_table(w, golden[f"{case}/{kind}_weight"], golden[f"{case}/{kind}_alias"],
                             float(golden[f"{case}/{kind}_W"]))
    # the reference works in FP64 with an absolute pack tolerance (EPSILON 1e-10): its tables
    # reconstruct every item far inside the library's 1e-6 relative bar
    assert chk["max_rel"] < 1e-6, chk
    assert chk["zero_mass"] == 0


@pytest.mark.parametrize("case", CASES)
def test_reference_verifier_accepted_its_tables(golden, case):
    assert int(golden[f"{case}/sweep_verify"]) == 1
    if case != "bestworst":
        assert int(golden[f"{case}/split_verify"]) == 1


@pytest.mark.parametrize("best", [True, False])
def test_np_tables_known_answer(golden, best):
    key = "np_best" if best else "np_worst"
    chk = po.check_ref_table(golden[f"{key}/w"], golden[f"{key}/weight"], golden[f"{key}/alias"],
                             float(golden[f"{key}/W"]))
    assert chk["max_rel"] < 1e-12


@pytest.mark.parametrize("case", CASES)
def test_exact_build_on_reference_generators(golden, case):
    w = golden[f"{case}/w"].astype(np.float32)
    rows = po.exact_build(w)
    chk = po.check_table(w, rows)
    assert chk["max_rel"] <= 2.5e-7, chk
    assert chk["zero_mass"] == 0 and chk["bad_rows"] == 0


def test_exact_sum_known_answer():
    # Adder::unitTest: sum_{0..999} i == 499500 exactly
    assert po.exact_sum(np.arange(1000, dtype=np.float32)) == 499500.0
    # correctly rounded where naive FP32 / FP64 accumulation is not
    w = np.array([1.0, 2.0 ** -30, 2.0 ** -30, -0.0] * 3, dtype=np.float32)
    assert po.exact_sum(w) == 3.0 + 6 * 2.0 ** -30
