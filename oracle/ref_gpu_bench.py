"""Times the reference's plain GPU sampling on this B200 (test infrastructure; run on a GPU box
after `make -C oracle ref` was run where the reference checkout exists).

The table is this library's split build of the large configuration's weights (n = 2^26,
w_i = (i+1)^-1.1 permuted; bench.make_weights), exported in the reference's row format
(FP64 absolute weight, int alias; wrs_export_reference_table). The reference's sampling
decision doSample<ArrayOfStructs> and its XORWOW generator (SamplerGpuBasic.cu:28-101,
utils/Prng.cuh:58-94) draw the samples in a harness loop (ref_gpu_shim.cu), at the reference's
default launch shape (46 x 160 threads) and at a full-GPU shape, next to this library's
wrs_alias_sample (PLAIN) on the same table and the same number of samples; and the reference's
rejection build (slot-count scan and slot fill) next to wrs_rejection_build_f32. Prints one JSON
line.

    python oracle/ref_gpu_bench.py [log2_samples]
"""
import json
import os
import sys
import time

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
    # the rejection build on the same weights: the reference's slot-count scan and slot fill
    # (RejectionSampling.cu:26-56, RejectionSamplingBinarySearch.cu:12-37; its own cub scan and
    # temporary allocation included, as in its build), against wrs_rejection_build_f32
    w64 = w.to(torch.float64)
    A_ref = torch.empty(2 * n + 1, dtype=torch.int32, device="cuda")
    size = np.zeros(1, dtype=np.int64)
    t_ref = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = ref.ref_gpu_rejection_build(w64.data_ptr(), n, Wv, A_ref.data_ptr(), A_ref.numel(), size.ctypes.data)
        t_ref.append(time.perf_counter() - t0)
        assert rc == 0, f"reference rejection build: CUDA error {rc}"
    del A_ref, w64
    A = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    frac = torch.empty(n, dtype=torch.float32, device="cuda")
    a_size = torch.zeros(1, dtype=torch.int64, device="cuda")
    rscr = torch.empty(wrs.rejection_build_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    assert wrs.rejection_build(w, A, frac, a_size, rscr, sync=True) == 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        wrs.rejection_build(w, A, frac, a_size, rscr)
    e1.record()
    torch.cuda.synchronize()
    res["rejection_build"] = {"slots": int(size[0]), "reference_ms_host_timed": round(min(t_ref) * 1e3, 3),
                              "library_ms": round(e0.elapsed_time(e1) / 3, 3)}
    del A, frac, rscr
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
