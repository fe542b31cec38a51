"""Generates the golden fixtures in this directory from the compiled reference.

Run in a checkout where the reference sources exist (the compiled reference is built from
them by `make -C oracle ref`):

    python tests/golden/make_golden.py

Writes ref_tables.npz: for the reference's deterministic weight generators
(SamplingAlgorithm.cu:21-71: Sine=1, Ramp=4, PowerLaw1=5, PowerLaw2=6, OneHeavy=7,
OneLight=8) at n=1000 and a seeded Uniform(0,1) FP32 case at n=4096, the weights and the
reference's own CPU tables (AliasTableSweep::build, AliasTableSplit::build with p=16,
AliasTableStack::build) as (weight, alias, W); the AliasTableNp best/worst-case tables; and
the reference's verifyTableCorrectness verdict on each table (debug build).
BestWorstCase (=2) is generated and swept but not split: the reference's split build does
not terminate on it in a Release build (its binary search relies on compiled-out asserts).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import py_oracle as po  # noqa: E402

N = 1000
P = 16
DISTS = {1: "sine", 2: "bestworst", 4: "ramp", 5: "powerlaw1", 6: "powerlaw2", 7: "oneheavy", 8: "onelight"}


def main():
    assert po.ref_available() and po.ref_available(debug=True), "build the reference first: make -C oracle ref"
    out = {}
    cases = {}
    for d, name in DISTS.items():
        cases[name] = po.ref_generate(N, d)
    rng = np.random.default_rng(0x5EED)
    cases["uniform_f32"] = rng.random(4096, dtype=np.float32).astype(np.float64)
    for name, w in cases.items():
        out[f"{name}/w"] = w
        wt, al, W, _ = po.ref_sweep_build(w)
        out[f"{name}/sweep_weight"], out[f"{name}/sweep_alias"], out[f"{name}/sweep_W"] = wt, al, np.float64(W)
        out[f"{name}/sweep_verify"] = np.int32(po.ref_verify(w, wt, al, W))
        if name != "bestworst":
            wt, al, W, _ = po.ref_split_build(w, P)
            out[f"{name}/split_weight"], out[f"{name}/split_alias"], out[f"{name}/split_W"] = wt, al, np.float64(W)
            out[f"{name}/split_verify"] = np.int32(po.ref_verify(w, wt, al, W))
        wt, al, W, _ = po.ref_stack_build(w)
        out[f"{name}/stack_weight"], out[f"{name}/stack_alias"], out[f"{name}/stack_W"] = wt, al, np.float64(W)
    for best in (True, False):
        w, wt, al, W = po.ref_np_table(N, best)
        key = "np_best" if best else "np_worst"
        out[f"{key}/w"], out[f"{key}/weight"], out[f"{key}/alias"], out[f"{key}/W"] = w, wt, al, np.float64(W)
    np.savez_compressed(os.path.join(HERE, "ref_tables.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
