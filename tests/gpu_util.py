"""Helpers shared by the GPU tests: run the library through its C ABI on torch memory."""
import numpy as np
import torch

import wrs


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def alloc_scratch(nbytes):
    return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device="cuda")


def gpu_build(w_np, method=wrs.WRS_METHOD_SPLIT, tile_items=0):
    """Returns (status, rows uint32 (n, 2), W)."""
    w = to_dev(np.asarray(w_np, dtype=np.float32))
    n = w.numel()
    opts = wrs.build_opts(method, tile_items, sync=True)
    table = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    scratch = alloc_scratch(wrs.alias_build_scratch_bytes(n, opts))
    W = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = wrs.alias_build(w, table, scratch, opts, W)
    torch.cuda.synchronize()
    rows = table.cpu().numpy().view(np.uint32).reshape(-1, 2).copy()
    return st, rows, float(W.item())


def table_from_rows(rows):
    return to_dev(np.ascontiguousarray(rows, dtype=np.uint32).view(np.int64).reshape(-1))


def gpu_sample(rows, m, seed, cbase=0, mode=wrs.WRS_SAMPLE_PLAIN, section_items=0, out_offset=0):
    n = rows.shape[0]
    table = table_from_rows(rows)
    buf = torch.full((m + out_offset + 4,), -7, dtype=torch.int32, device="cuda")
    out = buf[out_offset:out_offset + m]
    K = (n + (section_items or 65536) - 1) // (section_items or 65536)
    counts = torch.zeros(K, dtype=torch.int64, device="cuda") if mode == wrs.WRS_SAMPLE_SECTIONED else None
    st = wrs.alias_sample(table, n, m, seed, out, cbase, mode=mode, section_items=section_items,
                          section_counts=counts, sync=True)
    torch.cuda.synchronize()
    res = out.cpu().numpy().view(np.uint32).copy()
    tail = buf[out_offset + m:].cpu().numpy()
    assert np.all(tail == -7), "sampler wrote past the end of its output"
    if out_offset:
        assert np.all(buf[:out_offset].cpu().numpy() == -7), "sampler wrote before its output"
    return st, res, (counts.cpu().numpy().astype(np.uint64) if counts is not None else None)
