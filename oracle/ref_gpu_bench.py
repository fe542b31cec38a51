"""Times the reference's plain GPU sampling on this B200 (test infrastructure; run on a GPU box
after `make -C oracle ref` was run where the reference checkout exists).

The table is this library's split build of the large configuration's weights (n = 2^26,
w_i = (i+1)^-1.1 permuted; bench.make_weights), exported in the reference's row format
(FP64 absolute weight, int alias; wrs_export_reference_table). The reference's sampling
decision doSample<ArrayOfStructs> and its XORWOW generator (SamplerGpuBasic.cu:28-101,
utils/Prng.cuh:58-94) draw the samples in a harness loop (ref_gpu_shim.cu), at the reference's
default launch shape (46 x 160 threads) and at a full-GPU shape, next to this library's
wrs_alias_sample (PLAIN) on the same table and the same number of samples. Prints one JSON
line.

    python oracle/ref_gpu_bench.py [log2_samples]
"""
import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, ".."))
sys.path.insert(0, os.path.join(HERE, "..", "alias-table-gpu_b200"))
import bench  # noqa: E402
import py_oracle as po  # noqa: E402
import wrs  # noqa: E402


def main():
    log2m = int(sys.argv[1]) if len(sys.argv) > 1 else 30
    n = bench.N_ITEMS
    m = 1 << log2m
    w = torch.from_numpy(bench.make_weights()).cuda()
    table = torch.empty(n, dtype=torch.int64, device="cuda")
    scratch = torch.empty(wrs.alias_build_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    W = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert wrs.alias_build(w, table, scratch, wrs.build_opts(sync=True), W) == wrs.WRS_SUCCESS
    Wv = float(W.item())
    weight = torch.empty(n, dtype=torch.float64, device="cuda")
    alias = torch.empty(n, dtype=torch.int32, device="cuda")
    assert wrs.export_reference_table(table, Wv, weight, alias) == wrs.WRS_SUCCESS
    torch.cuda.synchronize()
    del scratch
    ref = po.ref_gpu()
    res = {"workload": f"plain sampling, n=2^26 bench table, 2^{log2m} samples", "n": n, "samples": m}
    for name, blocks, threads in [("reference_default_46x160", 46, 160),
                                  ("reference_full_gpu", torch.cuda.get_device_properties(0).multi_processor_count * 8,
                                   256)]:
        per = m // (blocks * threads)
        ms, chk = np.zeros(1, np.float32), np.zeros(1, np.uint32)
        rc = ref.ref_gpu_sample_timed(weight.data_ptr(), alias.data_ptr(), n, Wv / n, blocks, threads, per,
                                      0x5EED, ms.ctypes.data, chk.ctypes.data)
        assert rc == 0, f"reference sampling: CUDA error {rc}"
        drawn = per * blocks * threads
        res[name] = {"threads": blocks * threads, "samples": drawn, "ms": round(float(ms[0]), 3),
                     "gsamples_s": round(drawn / float(ms[0]) / 1e6, 3)}
    out = torch.empty(m, dtype=torch.int32, device="cuda")
    assert wrs.alias_sample(table, n, m, 7, out, 0) == 0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    assert wrs.alias_sample(table, n, m, 7, out, m) == 0
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    res["library_plain"] = {"samples": m, "ms": round(ms, 3), "gsamples_s": round(m / ms / 1e6, 3),
                            "writes": "4 B per sample (the reference's harness keeps an XOR only)"}
    print(json.dumps(res))


if __name__ == "__main__":
    main()
