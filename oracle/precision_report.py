"""Precision comparison of the precision-stress workload (test infrastructure, CPU only).

Weights w = 10^U(-8, 8) (numpy PCG64, seed 0x5EED + 3, FP32), the same generator as the
benchmark's precision-stress configuration. Three builds of the same weights, each checked
per item against n w_i / W with W the exact sum (or_check_* in wrs_oracle.c):
  * mixed: this library's build (FP32 stored probabilities, exact fixed-point prefixes and a
    compensated W); the oracle's or_exact_build gives the GPU's rows bit for bit;
  * all-FP64: the reference's sweep (AliasTableSweep.cu:12-60) with its FP64 running sums;
  * all-FP32: the same sweep with every quantity in FP32.

    python oracle/precision_report.py [log2n]      (default 28; about 20 GB of host memory at 2^28)

Prints one JSON line.
"""
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import py_oracle as po  # noqa: E402


def loguniform_weights(n: int, seed: int = 0x5EED + 3) -> np.ndarray:
    return (10.0 ** np.random.default_rng(seed).uniform(-8.0, 8.0, n)).astype(np.float32)


def report(log2n: int) -> dict:
    n = 1 << log2n
    w = loguniform_weights(n)
    out = {"workload": f"n=2^{log2n} w=10^U(-8,8) FP32 (seed 0x5EED+3)"}
    t = time.time()
    rows = po.exact_build(w)
    chk = po.check_table(w, rows)
    W = chk["W"]
    out["mixed"] = {k: chk[k] for k in ("max_rel", "p9999_rel", "zero_mass", "bad_rows")}
    del rows
    wt, al, W64 = po.sweep_build(w.astype(np.float64))
    c = po.check_ref_table_w(w, wt, al, W64 / n, W)
    out["all_fp64"] = {k: c[k] for k in ("max_rel", "p9999_rel", "zero_mass", "bad_rows")}
    del wt, al
    wt, al, WN32 = po.sweep_build_f32(w)
    c = po.check_ref_table_w(w, wt, al, WN32, W)
    out["all_fp32"] = {k: c[k] for k in ("max_rel", "p9999_rel", "zero_mass", "bad_rows")}
    out["seconds"] = round(time.time() - t, 1)
    return out


if __name__ == "__main__":
    print(json.dumps(report(int(sys.argv[1]) if len(sys.argv) > 1 else 28)))
