#!/usr/bin/env python
"""bench.py — throughput of the weighted-random-sampling hot path on B200.

Workload (the large single-table configuration): n = 2^26 FP32 weights w_i = (i+1)^-1.1
(computed in FP64, rounded to FP32) under a seeded random permutation; one step = one
split-method alias build of the whole table followed by 2^30 plain samples (uint32 indices
written to HBM). `value` = (items built + samples drawn) per second over all GPUs, from CUDA
events around K steps with every input already resident in HBM (weights 256 MB, output
4 GB: larger than L2, so no flush is needed between steps). `e2e` measures the same step
through the public API from pinned host memory: weights copied in and all samples copied
out inside the timed region (wrs_alias_sample_to_host: the copy of each finished chunk of
samples overlaps the drawing of the next).

The JSON line also carries the per-phase numbers of the workload (split build Gitems/s,
plain and sectioned Gsamples/s), the per-item probability error of the built table, the
roofline of the dominant kernel (the plain sampler), the SM clocks seen while timing, and
the reference's CPU path timed on this host (`cpu_baseline`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one replica per GPU (the path does not need a collective:
"replicas only"); value is the sum over replicas, time the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "alias-table-gpu_b200"))

N_ITEMS = 1 << 26
N_SAMPLES = 1 << 30
SECTION_ITEMS = 1 << 16
SEED_WEIGHTS = 0x5EED + 2
SEED_SAMPLES = 0xC0FFEE
METRIC = "build Gitems/s + Gsamples/s, batched vs per-table, %HBM peak, at ≤1e-6 prob err"
UNIT = "G(items+samples)/s"
WORKLOAD = "single large table: n=2^26 w=(i+1)^-1.1 permuted; split build + 2^30 plain samples per step"
FALLBACK_HBM_GBS = 6650.0
# kernels one step launches: wsum, scan, tile_prefix, link, pack_walk, split_pack (the chunked
# form over the tiles pack_walk listed; an empty list costs one short launch) and the sampler
KERNELS_PER_STEP = 7

def batched_kernels_per_replay(sizes, small_max: int, fused: bool, kinds=None) -> int:
    """Kernels one replay of a batched graph launches: table_lists and lists_check, one build
    launch per non-empty list (size classes n <= 4, 8, 16, 32, 64, <= small_max by lane groups;
    n <= 2048 and <= 8192 by CTAs), with `fused` one list sampler per such list plus
    chunks_plan and chunk_sample, else batch_sample; the ten tiled passes (plan_count,
    plan_scan, plan_fill, batch_wsum, tile_reduce, batch_prefix, heavy_list, tile_link,
    split_pack, batch_status) when tables above 8192 items are present; a mixed batch (kinds)
    adds one or two rejection kernels."""
    sizes = np.asarray(sizes)
    alias = sizes[(sizes > 0) & ((np.asarray(kinds) == 0) if kinds is not None else True)]
    lists = 0
    for lo, hi in [(1, 4), (5, 8), (9, 16), (17, 32), (33, 64), (65, small_max)]:
        hi = min(hi, small_max)
        if lo <= hi:
            lists += int(np.any((alias >= lo) & (alias <= hi)))
    lists += int(np.any((alias > small_max) & (alias <= 2048))) + int(np.any((alias > 2048) & (alias <= 8192)))
    k = 2 + lists * (2 if fused else 1) + (2 if fused else 1)
    if np.any(alias > 8192):
        k += 10
    if kinds is not None:
        rej = sizes[(sizes > 0) & (np.asarray(kinds) == 1)]
        k += int(np.any(rej <= 4096)) + int(np.any(rej > 4096))
    return k
BATCH_TABLES = 1 << 17
BATCH_SAMPLES_PER_TABLE = 64
BATCH_PER_TABLE_SAMPLE = 4096  # tables timed one call at a time (the per-table baseline)


def make_weights(n: int = N_ITEMS, seed: int = SEED_WEIGHTS) -> np.ndarray:
    w = (np.arange(1, n + 1, dtype=np.float64) ** -1.1).astype(np.float32)
    return w[np.random.default_rng(seed).permutation(n)]


def uniform_weights(n: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).random(n, dtype=np.float32)


def loguniform_weights(n: int, seed: int) -> np.ndarray:
    return (10.0 ** np.random.default_rng(seed).uniform(-8.0, 8.0, n)).astype(np.float32)


# Single-table configurations (--config); "2" is the default and the headline. Each is seeded
# synthetic data of the configuration's shape and distribution.
CONFIGS = {
    "1": dict(log2n=20, log2m=24, make=lambda n: uniform_weights(n, 0x5EED + 1),
              workload="plain single table: n=2^20 w~U(0,1) FP32; split build + 2^24 plain samples per step "
                       "(L2-resident)", weights="U(0,1) FP32 (numpy PCG64, seed 0x5EED+1)"),
    "2": dict(log2n=26, log2m=30, make=lambda n: make_weights(n),
              workload=WORKLOAD, weights="w_i=(i+1)^-1.1 FP64->FP32, seeded permutation"),
    "3": dict(log2n=28, log2m=28, make=lambda n: loguniform_weights(n, 0x5EED + 3),
              workload="precision stress: n=2^28 w=10^U(-8,8) log-uniform FP32; split build + 2^28 plain samples "
                       "per step", weights="10^U(-8,8) FP32 (numpy PCG64, seed 0x5EED+3)"),
}


def measured_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(n, m):
    """DRAM bytes of one plain-sampler launch of m samples from an n-row table, from the
    committed ncu summary (bytes per sample of a capture on a table of the same size; the
    gathers are random, so the bytes grow in proportion to the samples), if there is one."""
    path = os.path.join(REPO, "profiles", "traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        if int(d["table_rows"]) != n:
            return None
        return int(round(d["sample_plain_kernel_bytes_per_sample"] * m))
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_uuid: str | None):
        self.uuid = gpu_uuid
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "power_w_max": max(power),
                "samples": len(sm), "reasons": sorted(reasons)}


def table_error_gpu(w, table) -> dict:
    """Per-item relative error of a device table against w_i / W, on the device in FP64:
    P_i = prob_i + sum over rows r aliasing i of (1 - prob_r), against n w_i / W."""
    import torch
    n = w.numel()
    rows = table.view(torch.int32).view(-1, 2)
    p = rows[:, 0].contiguous().view(torch.float32).double()
    a = rows[:, 1].long()
    got = p.clone()
    got.scatter_add_(0, a, 1.0 - p)
    del a
    wd = w.double()
    W = wd.sum()
    nz = wd > 0
    exp = wd[nz] * (n / W)
    rel = (got[nz] - exp).abs_() / exp
    k = max(1, int(math.ceil(rel.numel() * 1e-4)))
    top = torch.topk(rel, k).values
    zm = float(got[~nz].sum().item()) if bool((~nz).any()) else 0.0
    return {"max_rel": float(top[0].item()), "p9999_rel": float(top[-1].item()), "zero_weight_mass": zm}


def chi2_gpu(w, samples, min_expected: float = 32.0) -> dict:
    """Chi-square goodness of fit of the samples against w_i / W, on the device. Items are
    grouped, in index order, into bins of at least `min_expected` expected samples (the
    cumulative expected count cut every `min_expected`); the p-value of the statistic with
    bins - 1 degrees of freedom uses the Wilson-Hilferty normal approximation."""
    import torch
    m = samples.numel()
    wd = w.double()
    expected = wd * (m / wd.sum())
    cum = torch.cumsum(expected, 0)
    bin_of = torch.clamp((cum - expected * 0.5) / min_expected, min=0).long()
    nbins = int(bin_of[-1].item()) + 1
    del cum
    counts = torch.bincount(samples, minlength=w.numel()).double()
    obs = torch.zeros(nbins, dtype=torch.float64, device=w.device).index_add_(0, bin_of, counts)
    exp_b = torch.zeros(nbins, dtype=torch.float64, device=w.device).index_add_(0, bin_of, expected)
    del counts, bin_of, expected
    keep = exp_b > 0
    stat = float((((obs - exp_b) ** 2)[keep] / exp_b[keep]).sum().item())
    df = int(keep.sum().item()) - 1
    z = ((stat / df) ** (1.0 / 3.0) - (1.0 - 2.0 / (9.0 * df))) / math.sqrt(2.0 / (9.0 * df))
    return {"samples": m, "bins": df + 1, "min_expected_per_bin": min_expected, "stat": round(stat, 1), "df": df,
            "stat_over_df": round(stat / df, 6), "p_value": 0.5 * math.erfc(z / math.sqrt(2.0))}


def table_error(w: np.ndarray, rows_u32: np.ndarray) -> dict:
    """Per-item relative error of the table against w_i / W (W summed in FP64 pairwise)."""
    n = w.size
    p = rows_u32[:, 0].view(np.float32).astype(np.float64)
    a = rows_u32[:, 1].astype(np.int64)
    got = p + np.bincount(a, weights=1.0 - p, minlength=n)
    wd = w.astype(np.float64)
    W = math.fsum(wd.tolist()) if n <= (1 << 20) else float(np.sum(wd))
    exp = n * wd / W
    nz = wd > 0
    rel = np.abs(got[nz] - exp[nz]) / exp[nz]
    return {"max_rel": float(rel.max()), "p9999_rel": float(np.quantile(rel, 0.9999)),
            "zero_weight_mass": float(got[~nz].sum()) if (~nz).any() else 0.0}


# ---------------------------------------------------------------- multi-GPU replicas

def max_over_ranks(x: float, device) -> float:
    """The largest value over all ranks (time-like numbers: the job takes the slowest rank);
    x itself without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: int, ms: float, world: int) -> float:
    """Whole-job throughput in G units/s of `world` replicas that each process
    `units_per_rank` units, from the slowest rank's time."""
    return world * units_per_rank / (ms * 1e-3) / 1e9


# ---------------------------------------------------------------- our arm

def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import wrs

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if wrs.lib().wrs_check_device() != 0:
        raise RuntimeError("not an sm_100 device")
    cfg = CONFIGS[args.config]
    n, m = 1 << cfg["log2n"], 1 << (args.log2_samples if args.log2_samples else cfg["log2m"])
    w_np = cfg["make"](n)
    w_host = torch.from_numpy(w_np).pin_memory()
    w = w_host.to(dev)
    opts = wrs.build_opts(wrs.WRS_METHOD_SPLIT)
    table = torch.empty(n, dtype=torch.int64, device=dev)
    scratch = torch.empty(wrs.alias_build_scratch_bytes(n, opts), dtype=torch.uint8, device=dev)
    out = torch.empty(m, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    def build():
        st = wrs.alias_build(w, table, scratch, opts, None, sp)
        if st:
            raise wrs.WrsError(st, "build")

    def sample(counter_base, mode=wrs.WRS_SAMPLE_PLAIN, section_items=0):
        st = wrs.alias_sample(table, n, m, SEED_SAMPLES, out, counter_base, mode=mode, section_items=section_items,
                              stream=sp)
        if st:
            raise wrs.WrsError(st, "sample")

    # correctness of this exact table (before timing)
    build()
    st = wrs.scratch_status(scratch, sp)
    if st:
        raise wrs.WrsError(st, "build (device)")
    err = table_error_gpu(w, table) if rank == 0 else None

    for i in range(args.warmup):
        build()
        sample(i * m)
    torch.cuda.synchronize()

    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    smi_uuid = None
    try:
        smi_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(smi_uuid if rank == 0 else None)
    if rank == 0:
        clocks.start()
        time.sleep(0.3)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    for k in range(K):
        ev[k][0].record(stream)
        build()
        ev[k][1].record(stream)
        sample((args.warmup + k) * m)
        ev[k][2].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop() if rank == 0 else None
    total_ms = ev[0][0].elapsed_time(ev[K - 1][2])
    build_ms = statistics.median([e[0].elapsed_time(e[1]) for e in ev])
    sample_ms = statistics.median([e[1].elapsed_time(e[2]) for e in ev])
    total_ms = max_over_ranks(total_ms, dev)

    # sectioned sampling on the same table (reported beside the headline)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sample(0, wrs.WRS_SAMPLE_SECTIONED, SECTION_ITEMS)
    torch.cuda.synchronize()
    reps = 5
    s0.record(stream)
    for r in range(reps):
        sample((r + 1) * m, wrs.WRS_SAMPLE_SECTIONED, SECTION_ITEMS)
    s1.record(stream)
    torch.cuda.synchronize()
    sect_ms = s0.elapsed_time(s1) / reps

    # histogram mode: the same plain samples counted per row instead of written (the
    # reference's GPU samplers write no samples); the counts are zeroed inside the timed loop
    counts = torch.empty(n, dtype=torch.int32, device=dev)
    st = wrs.alias_histogram(table, n, m, SEED_SAMPLES, counts.zero_(), 0, stream=sp)
    torch.cuda.synchronize()
    s0.record(stream)
    for r in range(reps):
        counts.zero_()
        st |= wrs.alias_histogram(table, n, m, SEED_SAMPLES, counts, (r + 1) * m, stream=sp)
    s1.record(stream)
    torch.cuda.synchronize()
    if st:
        raise wrs.WrsError(st, "histogram")
    hist_ms = s0.elapsed_time(s1) / reps
    del counts
    # discard mode: the same plain samples drawn and folded into one word (the reference's GPU
    # samplers keep no samples: the like-for-like timing)
    fold = torch.zeros(1, dtype=torch.int32, device=dev)
    s0.record(stream)
    for r in range(reps):
        st |= wrs.alias_sample(table, n, m, SEED_SAMPLES, fold, (r + 1) * m, mode=wrs.WRS_SAMPLE_DISCARD,
                               stream=sp)
    s1.record(stream)
    torch.cuda.synchronize()
    if st:
        raise wrs.WrsError(st, "discard")
    discard_ms = s0.elapsed_time(s1) / reps
    # rejection sampling on the same weights (build: W, slot counts, slot fill; then samples)
    A = torch.empty(2 * n, dtype=torch.int32, device=dev)
    frac = torch.empty(n, dtype=torch.float32, device=dev)
    a_size = torch.zeros(1, dtype=torch.int64, device=dev)
    rscr = torch.empty(wrs.rejection_build_scratch_bytes(n), dtype=torch.uint8, device=dev)
    rstat = torch.zeros(1, dtype=torch.int32, device=dev)
    st = wrs.rejection_build(w, A, frac, a_size, rscr, sync=True, stream=sp)
    rm = min(m, 1 << 28)
    rout = torch.empty(rm, dtype=torch.int32, device=dev)
    st |= wrs.rejection_sample(A, a_size, frac, n, rm, SEED_SAMPLES, rout, 0, 0, rstat, stream=sp)
    torch.cuda.synchronize()
    s0.record(stream)
    for r in range(reps):
        st |= wrs.rejection_build(w, A, frac, a_size, rscr, stream=sp)
    s1.record(stream)
    torch.cuda.synchronize()
    rej_build_ms = s0.elapsed_time(s1) / reps
    s0.record(stream)
    for r in range(reps):
        st |= wrs.rejection_sample(A, a_size, frac, n, rm, SEED_SAMPLES, rout, (r + 1) * rm, 0, rstat, stream=sp)
    s1.record(stream)
    torch.cuda.synchronize()
    rej_sample_ms = s0.elapsed_time(s1) / reps
    if st or int(rstat.item()) or wrs.scratch_status(rscr, sp):
        raise wrs.WrsError(st or int(rstat.item()) or 1, "rejection")
    rej_slots = int(a_size.item())
    # the same samples from packed slots (slot and fraction in one 8-byte gather per try)
    slots = torch.empty(rej_slots, dtype=torch.int64, device=dev)
    rout2 = torch.empty(rm, dtype=torch.int32, device=dev)
    st = wrs.rejection_pack(A, a_size, frac, n, slots, stream=sp)
    st |= wrs.rejection_sample_packed(slots, a_size, n, rm, SEED_SAMPLES, rout2, 0, 0, rstat, stream=sp)
    torch.cuda.synchronize()
    s0.record(stream)
    for r in range(reps):
        st |= wrs.rejection_pack(A, a_size, frac, n, slots, stream=sp)
    s1.record(stream)
    torch.cuda.synchronize()
    rej_pack_ms = s0.elapsed_time(s1) / reps
    s0.record(stream)
    for r in range(reps):
        st |= wrs.rejection_sample_packed(slots, a_size, n, rm, SEED_SAMPLES, rout2, (r + 1) * rm, 0, rstat, stream=sp)
    s1.record(stream)
    torch.cuda.synchronize()
    rej_packed_ms = s0.elapsed_time(s1) / reps
    if st or int(rstat.item()):
        raise wrs.WrsError(st or int(rstat.item()), "packed rejection")
    if not torch.equal(rout, rout2):
        raise RuntimeError("packed rejection samples differ from the unpacked sampler's")
    del A, frac, rscr, slots, rout2
    # the PSA+ build on the same weights (a table of its own; the headline table is the split one)
    popts = wrs.build_opts(wrs.WRS_METHOD_PSA_PLUS)
    ptable = torch.empty(n, dtype=torch.int64, device=dev)
    pscr = torch.empty(wrs.alias_build_scratch_bytes(n, popts), dtype=torch.uint8, device=dev)
    st = wrs.alias_build(w, ptable, pscr, popts, stream=sp)
    torch.cuda.synchronize()
    s0.record(stream)
    for r in range(reps):
        st |= wrs.alias_build(w, ptable, pscr, popts, stream=sp)
    s1.record(stream)
    torch.cuda.synchronize()
    psa_build_ms = s0.elapsed_time(s1) / reps
    if st or wrs.scratch_status(pscr, sp):
        raise wrs.WrsError(st or 1, "psa+ build")
    del ptable, pscr
    rej_chi2 = chi2_gpu(w, rout) if rank == 0 else None
    del rout

    # the random-access bound of the plain sampler: a library gather (torch index_select) of
    # random 8-byte rows from the same table, with precomputed uniform row indices
    g_n = 1 << 27
    gidx = torch.randint(0, n, (g_n,), dtype=torch.int64, device=dev)
    gout = torch.index_select(table, 0, gidx)
    torch.cuda.synchronize()
    s0.record(stream)
    for r in range(reps):
        torch.index_select(table, 0, gidx, out=gout)
    s1.record(stream)
    torch.cuda.synchronize()
    gather_ms = s0.elapsed_time(s1) / reps
    del gidx, gout
    # ... and the library's own probe: the sampler's row gathers (same load form, eight in
    # flight per thread) at hashed rows, nothing written: the table's random-access ceiling
    sink = torch.zeros(1, dtype=torch.int32, device=dev)
    assert wrs.random_gather_probe(table, n, m, 7, sink, sp) == 0
    s0.record(stream)
    for r in range(reps):
        assert wrs.random_gather_probe(table, n, m, 8 + r, sink, sp) == 0
    s1.record(stream)
    torch.cuda.synchronize()
    probe_ms = s0.elapsed_time(s1) / reps

    # goodness of fit of the last timed step's samples (outside every timed region)
    chi2 = chi2_gpu(w, out) if rank == 0 else None

    # end to end through the API with host buffers: H2D weights, build, sample, D2H samples
    out_host = torch.empty(m, dtype=torch.int32).pin_memory()
    e2e_steps = max(3, min(K, 10))
    def sample_to_host(counter_base):
        st = wrs.alias_sample_to_host(table, n, m, SEED_SAMPLES, out, out_host, counter_base, 0, sp)
        if st:
            raise wrs.WrsError(st, "sample to host")

    # the next step's weights go up on a second stream as soon as this step's build has read
    # them, so that their transfer overlaps the samples' transfer down
    h2d = torch.cuda.Stream(dev)
    loaded = torch.cuda.Event()
    built = torch.cuda.Event()

    def load_weights():
        with torch.cuda.stream(h2d):
            w.copy_(w_host, non_blocking=True)
        loaded.record(h2d)

    def e2e_steps_run(steps, cbase0):
        h2d.wait_stream(stream)
        load_weights()
        for i in range(steps):
            stream.wait_event(loaded)
            build()
            built.record(stream)
            if i + 1 < steps:
                h2d.wait_event(built)
                load_weights()
            sample_to_host(cbase0 + i * m)  # chunks copied down while the next ones are drawn

    e2e_steps_run(2, 0)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_steps_run(e2e_steps, 0)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, dev)

    if rank != 0:
        return None
    peak, peak_kind = measured_peak()
    achieved = 12.0 * m / (sample_ms * 1e-3) / 1e9  # GB/s, 12 B per sample (8 B gather + 4 B write)
    build_gbs = 12.0 * n / (build_ms * 1e-3) / 1e9  # 12 B per item (4 B read + 8 B write)
    step_ms = total_ms / K
    value = replica_value(n + m, step_ms, world)
    cpu = cpu_baseline(w_np, m) if not args.no_cpu_baseline else None
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(step_ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["workload"], "n_items": n, "n_samples_per_step": m, "build": "split",
                   "sampling": "plain", "weights": cfg["weights"],
                   "l2": ("inputs larger than L2; no flush" if 12 * n + 4 * m > (256 << 20)
                          else "L2-resident table and samples (126 MB L2)"),
                   "parallelism": f"replicas x{world}"},
        "phases": {"build_ms": round(build_ms, 4), "build_gitems_s": round(n / build_ms / 1e6, 3),
                   "build_hbm_gbs": round(build_gbs, 1), "build_hbm_frac": round(build_gbs / peak, 4),
                   "sample_ms": round(sample_ms, 4), "sample_gsamples_s": round(m / sample_ms / 1e6, 3),
                   "sectioned_sample_ms": round(sect_ms, 4),
                   "sectioned_gsamples_s": round(m / sect_ms / 1e6, 3),
                   "histogram_sample_ms": round(hist_ms, 4), "histogram_gsamples_s": round(m / hist_ms / 1e6, 3),
                   "discard_sample_ms": round(discard_ms, 4), "discard_gsamples_s": round(m / discard_ms / 1e6, 3),
                   "psa_plus_build_ms": round(psa_build_ms, 4),
                   "rejection_build_ms": round(rej_build_ms, 4), "rejection_slots": rej_slots,
                   "rejection_build_gitems_s": round(n / rej_build_ms / 1e6, 3),
                   "rejection_samples": rm, "rejection_sample_ms": round(rej_sample_ms, 4),
                   "rejection_gsamples_s": round(rm / rej_sample_ms / 1e6, 3),
                   "rejection_pack_ms": round(rej_pack_ms, 4),
                   "rejection_packed_sample_ms": round(rej_packed_ms, 4),
                   "rejection_packed_gsamples_s": round(rm / rej_packed_ms / 1e6, 3),
                   "section_items": SECTION_ITEMS},
        "prob_error": err,
        "chi_square": chi2,
        "rejection_chi_square": rej_chi2,
        "roofline": {"kernel": "sample_plain_kernel", "bound": "hbm", "achieved": round(achieved, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": ncu_traffic(n, m),
                     "algorithmic_bytes": "12 B/sample x 2^%d samples per launch (8 B row gather + 4 B write)"
                                          % (m.bit_length() - 1),
                     "random_access_bound": {
                         "probe": "wrs_random_gather_probe: the sampler's 8-byte row gathers (.L2::64B, 8 in "
                                  "flight per thread) at hashed rows of the same table, nothing written, "
                                  "%d gathers" % m,
                         "gathers_per_s_g": round(m / probe_ms / 1e6, 2),
                         "sampler_over_probe": round((m / sample_ms) / (m / probe_ms), 3),
                         "torch_index_select_gathers_per_s_g": round(g_n / gather_ms / 1e6, 2)}},
        "cpu_baseline": cpu,
        "clocks": clk,
        "e2e": {"value": round(replica_value(n + m, e2e_ms, world), 4), "unit": UNIT,
                "ms_per_step": round(e2e_ms, 3), "h2d_bytes_per_step": 4 * n, "d2h_bytes_per_step": 4 * m},
        "gpu_launches": KERNELS_PER_STEP * K,
    }
    if not args.no_batched and args.config == "2":
        line["batched"] = batched_phase(dev)
    if not args.no_side and args.config == "2" and world == 1:
        del w, table, scratch, out
        torch.cuda.empty_cache()
        line["side_configs"] = side_configs(dev)
    return line


def single_table_summary(dev, cfg: dict, steps: int = 20) -> dict:
    """Split build and plain sampling of one configuration's table (median of `steps` CUDA-event
    timings each, after warm-up), with the table's per-item error."""
    import torch
    import wrs

    n, m = 1 << cfg["log2n"], 1 << cfg["log2m"]
    w = torch.from_numpy(cfg["make"](n)).to(dev)
    opts = wrs.build_opts()
    table = torch.empty(n, dtype=torch.int64, device=dev)
    scratch = torch.empty(wrs.alias_build_scratch_bytes(n, opts), dtype=torch.uint8, device=dev)
    out = torch.empty(m, dtype=torch.int32, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3 * steps)]
    for r in range(3):
        assert wrs.alias_build(w, table, scratch, opts) == 0
        assert wrs.alias_sample(table, n, m, SEED_SAMPLES, out, r * m) == 0
    torch.cuda.synchronize()
    for r in range(steps):
        ev[3 * r].record()
        assert wrs.alias_build(w, table, scratch, opts) == 0
        ev[3 * r + 1].record()
        assert wrs.alias_sample(table, n, m, SEED_SAMPLES, out, (3 + r) * m) == 0
        ev[3 * r + 2].record()
    torch.cuda.synchronize()
    if wrs.scratch_status(scratch) != 0:
        raise RuntimeError("build failed on the device")
    b = statistics.median([ev[3 * r].elapsed_time(ev[3 * r + 1]) for r in range(steps)])
    smp = statistics.median([ev[3 * r + 1].elapsed_time(ev[3 * r + 2]) for r in range(steps)])
    # sectioned sampling with the section size the autotuner picks for this table
    st, S = wrs.autotune_sections(table, n, m, out)
    if st:
        raise wrs.WrsError(st, "autotune_sections")
    for r in range(steps):
        ev[3 * r].record()
        assert wrs.alias_sample(table, n, m, SEED_SAMPLES, out, r * m, mode=wrs.WRS_SAMPLE_SECTIONED,
                                section_items=S) == 0
        ev[3 * r + 1].record()
    torch.cuda.synchronize()
    sec = statistics.median([ev[3 * r].elapsed_time(ev[3 * r + 1]) for r in range(steps)])
    return {"workload": cfg["workload"], "build_ms": round(b, 4), "build_gitems_s": round(n / b / 1e6, 2),
            "sample_ms": round(smp, 4), "sample_gsamples_s": round(m / smp / 1e6, 2),
            "sectioned_sample_ms": round(sec, 4), "sectioned_section_items": S,
            "value": round((n + m) / (b + smp) / 1e6, 3), "unit": UNIT, "prob_error": table_error_gpu(w, table)}


def precision_summary(dev, reps: int = 3) -> dict:
    """The precision stress configuration (n = 2^28 log-uniform weights over 16 decades): the
    default build (exact fixed-point lines, compensated W, FP32 stored probabilities) against
    the all-FP64 and all-FP32 builds, each timed (median of `reps`) with its per-item error
    against n w_i / W on the device; then 2^28 plain samples of the default table."""
    import torch
    import wrs

    cfg = CONFIGS["3"]
    n, m = 1 << cfg["log2n"], 1 << cfg["log2m"]
    w = torch.from_numpy(cfg["make"](n)).to(dev)
    table = torch.empty(n, dtype=torch.int64, device=dev)
    modes = [("mixed", wrs.WRS_PRECISION_MIXED), ("fp64", wrs.WRS_PRECISION_FP64), ("fp32", wrs.WRS_PRECISION_FP32)]
    need = max(wrs.alias_build_scratch_bytes(n, wrs.build_opts(precision=p)) for _, p in modes)
    scratch = torch.empty(need, dtype=torch.uint8, device=dev)
    res = {"workload": cfg["workload"] + "; builds in the three precisions"}
    for name, p in modes:
        opts = wrs.build_opts(precision=p)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * reps)]
        assert wrs.alias_build(w, table, scratch, opts) == 0
        torch.cuda.synchronize()
        for r in range(reps):
            ev[2 * r].record()
            assert wrs.alias_build(w, table, scratch, opts) == 0
            ev[2 * r + 1].record()
        torch.cuda.synchronize()
        if wrs.scratch_status(scratch) != 0:
            raise RuntimeError(f"{name} build failed on the device")
        ms = statistics.median([ev[2 * r].elapsed_time(ev[2 * r + 1]) for r in range(reps)])
        res[name] = {"build_ms": round(ms, 3), "build_gitems_s": round(n / ms / 1e6, 2),
                     **table_error_gpu(w, table)}
        torch.cuda.empty_cache()
    assert wrs.alias_build(w, table, scratch, wrs.build_opts()) == 0
    del scratch
    torch.cuda.empty_cache()
    out = torch.empty(m, dtype=torch.int32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    assert wrs.alias_sample(table, n, m, SEED_SAMPLES, out, 0) == 0
    e0.record()
    assert wrs.alias_sample(table, n, m, SEED_SAMPLES, out, m) == 0
    e1.record()
    torch.cuda.synchronize()
    res["sample_ms"] = round(e0.elapsed_time(e1), 3)
    return res


def side_configs(dev) -> dict:
    """Compact summaries of the other configurations, measured in the same run: the plain
    single table (n = 2^20, L2-resident), the precision comparison at n = 2^28, and the mixed
    batch (alias or rejection per size class, autotuned)."""
    import torch

    out = {"config1": single_table_summary(dev, CONFIGS["1"])}
    torch.cuda.empty_cache()
    out["config3"] = precision_summary(dev)
    torch.cuda.empty_cache()
    b = batched_phase(dev, batch_config5, mixed=True)
    out["config5"] = {k: b[k] for k in ("workload", "items", "samples", "batched_ms", "batched_g_items_plus_samples_s",
                                        "per_table_ms", "speedup", "e2e") if k in b}
    if "mixed" in b:
        out["config5"]["mixed"] = b["mixed"]
    return out


def zipf_sizes(num: int, s: float, lo: int, hi: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    k = np.arange(lo, hi + 1, dtype=np.float64)
    p = k ** -s
    p /= p.sum()
    return rng.choice(np.arange(lo, hi + 1), size=num, p=p).astype(np.int64)


def batch_config4():
    """2^17 tables, sizes Zipf(2) on [2, 2^16], w~U(0,1), 64 samples per table."""
    sizes = zipf_sizes(BATCH_TABLES, 2.0, 2, 1 << 16, 0x5EED + 4)
    w = np.random.default_rng(0x5EED + 4).random(int(sizes.sum()), dtype=np.float32)
    counts = np.full(sizes.size, BATCH_SAMPLES_PER_TABLE, dtype=np.int64)
    what = (f"2^17 tables, sizes Zipf(2) on [2, 2^16] ({int(sizes.sum())} items), w~U(0,1) FP32, int64 CSR "
            f"offsets; build + {BATCH_SAMPLES_PER_TABLE} samples per table")
    return sizes, w, counts, what, [(np.arange(BATCH_PER_TABLE_SAMPLE), np.ones(sizes.size, bool))]


def batch_config5():
    """10^6 tables of U{1..64} items with Exp(1) weights, then 100 tables of 2^20 items with
    Pareto(1.5) weights; 4 x size samples per table."""
    rng = np.random.default_rng(0x5EED + 5)
    small = rng.integers(1, 65, 1_000_000)
    sizes = np.concatenate([small, np.full(100, 1 << 20)]).astype(np.int64)
    w_small = rng.exponential(1.0, int(small.sum())).astype(np.float32)
    w_large = (rng.pareto(1.5, 100 << 20) + 1.0).astype(np.float32)
    w = np.concatenate([w_small, w_large])
    counts = 4 * sizes
    what = (f"10^6 tables of U{{1..64}} items, w~Exp(1), and 100 tables of 2^20 items, w~Pareto(1.5) "
            f"({int(sizes.sum())} items); build + 4 x size samples per table; alias or rejection per size "
            f"class (ceil(log2 n)), chosen by the autotuner on this batch")
    return sizes, w, counts, what, [(np.arange(BATCH_PER_TABLE_SAMPLE), sizes <= 64),
                                    (np.arange(1_000_000, 1_000_004), sizes > 64)]


def batched_phase(dev, make=batch_config4, mixed: bool = False, shape: str = "") -> dict:
    """A batched-tables configuration: the batched build and sample (autotuned launch shape,
    captured in one CUDA graph) against the plain single-table entry points called once per
    table, timed on samples of each size class and scaled to all tables of the class by count
    (each call pays the same launch sequence). With `mixed`, the autotuner also picks alias or
    rejection per size class, and the timed graph is the mixed build and sampler with those
    kinds (the all-alias graph is timed beside it)."""
    import torch
    import wrs

    sizes, w_np, counts, what, per_table_groups = make()
    nt = sizes.size
    off = np.zeros(nt + 1, dtype=np.int64)
    np.cumsum(sizes, out=off[1:])
    items = int(off[-1])
    w = torch.from_numpy(w_np).to(dev)
    d_off = torch.from_numpy(off).to(dev)
    table = torch.empty(items, dtype=torch.int64, device=dev)
    scratch = torch.empty(max(wrs.batched_build_scratch_bytes(off), wrs.batched_build_sample_scratch_bytes(off)),
                          dtype=torch.uint8, device=dev)
    soff = np.zeros(nt + 1, dtype=np.int64)
    np.cumsum(counts, out=soff[1:])
    total = int(soff[-1])
    d_soff = torch.from_numpy(soff).to(dev)
    out = torch.empty(total, dtype=torch.int32, device=dev)
    if shape:
        small, tile = (int(x) for x in shape.split(","))
        opts = wrs.build_opts(0, tile, False, small)
    else:
        opts = wrs.build_opts()
        st = (wrs.batched_autotune(w, d_off, off, table, scratch, opts) if mixed else
              wrs.batched_autotune_build_sample(w, d_off, off, table, d_soff, total, out, scratch, opts))
        if st:
            raise wrs.WrsError(st, "batched autotune")
    # the batch's rows equal single-table builds of the same weights (a sample of tables,
    # the largest ones included; the tests check every table against the oracle)
    st = wrs.batched_build(w, d_off, off, table, scratch, wrs.build_opts(0, opts.tile_items, True,
                                                                        opts.small_table_items))
    if st:
        raise wrs.WrsError(st, "batched build")
    rows = table.cpu().numpy().view(np.uint32).reshape(-1, 2)
    check = np.r_[0:64, np.argsort(sizes, kind="stable")[-8:]]
    exact = True
    for t in check:
        n_t = int(sizes[t])
        t1 = torch.empty(n_t, dtype=torch.int64, device=dev)
        sc1 = torch.empty(wrs.alias_build_scratch_bytes(n_t), dtype=torch.uint8, device=dev)
        if wrs.alias_build(w[int(off[t]):int(off[t + 1])], t1, sc1, wrs.build_opts(sync=True)):
            raise RuntimeError("single-table build failed")
        exact &= bool(np.array_equal(rows[off[t]:off[t + 1]], t1.cpu().numpy().view(np.uint32).reshape(-1, 2)))

    # the step: wrs_batched_build_sample (each size class sampled as soon as it is built); the
    # separate build and sample calls are timed beside it, and must give the same samples
    s = torch.cuda.Stream(dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        wrs.batched_build_sample(w, d_off, off, table, d_soff, total, SEED_SAMPLES, out, scratch, opts, stream=s)
        g.capture_end()
    g_sep = torch.cuda.CUDAGraph()
    out_sep = torch.empty_like(out)
    with torch.cuda.stream(s):
        g_sep.capture_begin()
        wrs.batched_build(w, d_off, off, table, scratch, opts, stream=s)
        wrs.batched_sample(table, d_off, nt, d_soff, total, SEED_SAMPLES, out_sep, 0, stream=s)
        g_sep.capture_end()
    torch.cuda.current_stream(dev).wait_stream(s)
    for _ in range(3):
        g.replay()
        g_sep.replay()
    torch.cuda.synchronize()
    if wrs.scratch_status(scratch) or not torch.equal(out, out_sep):
        raise RuntimeError("build and sample differs from the separate build and sample calls")
    reps = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the batch (weights, offsets, rows, samples) fits in L2: every replay is timed on its own
    # after a write of 256 MiB (twice the L2) evicted the previous one
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * reps)]
    t0 = time.perf_counter()
    for i in range(reps):
        flush.zero_()
        ev[2 * i].record()
        g.replay()
        ev[2 * i + 1].record()
    torch.cuda.synchronize()
    batched_ms = sum(ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(reps)) / reps
    batched_wall_ms = (time.perf_counter() - t0) * 1e3 / reps
    for i in range(reps):
        flush.zero_()
        ev[2 * i].record()
        g_sep.replay()
        ev[2 * i + 1].record()
    torch.cuda.synchronize()
    separate_ms = sum(ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(reps)) / reps
    # end to end: the weights and both offset arrays copied up from pinned host memory, the
    # graph replayed, the samples copied down
    w_h = torch.from_numpy(w_np).pin_memory()
    off_h, soff_h = torch.from_numpy(off).pin_memory(), torch.from_numpy(soff).pin_memory()
    out_h = torch.empty(total, dtype=torch.int32).pin_memory()

    def e2e_once():
        w.copy_(w_h, non_blocking=True)
        d_off.copy_(off_h, non_blocking=True)
        d_soff.copy_(soff_h, non_blocking=True)
        g.replay()
        out_h.copy_(out, non_blocking=True)

    e2e_once()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        e2e_once()
    e1.record()
    torch.cuda.synchronize()
    batched_e2e_ms = e0.elapsed_time(e1) / reps
    h2d_bytes = 4 * items + 8 * (nt + 1) * 2
    mixed_info = None
    if mixed:
        A = torch.empty(2 * items, dtype=torch.int32, device=dev)
        frac = torch.empty(items, dtype=torch.float32, device=dev)
        a_size = torch.empty(nt, dtype=torch.int64, device=dev)
        kt = torch.empty(nt, dtype=torch.uint8, device=dev)
        scr_m = torch.empty(wrs.batched_mixed_build_scratch_bytes(off, None, opts), dtype=torch.uint8, device=dev)
        st, kinds, cls, cms = wrs.batched_autotune_kinds(w, d_off, off, d_soff, soff, table, A, frac, a_size, kt,
                                                         out, scr_m, opts)
        if st:
            raise wrs.WrsError(st, "kinds autotune")
        d_kinds = torch.from_numpy(kinds).to(dev)
        st = wrs.batched_mixed_build(w, d_off, off, d_kinds, kinds, table, A, frac, a_size, scr_m,
                                     wrs.build_opts(0, opts.tile_items, True, opts.small_table_items))
        if st:
            raise wrs.WrsError(st, "mixed build")
        gm = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            gm.capture_begin()
            wrs.batched_mixed_build(w, d_off, off, d_kinds, kinds, table, A, frac, a_size, scr_m, opts, stream=s)
            wrs.batched_mixed_sample(table, A, frac, a_size, d_off, d_kinds, nt, d_soff, total, SEED_SAMPLES, out, 0,
                                     stream=s)
            gm.capture_end()
        torch.cuda.current_stream(dev).wait_stream(s)
        for _ in range(3):
            gm.replay()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record()
        for _ in range(reps):
            gm.replay()
        e1.record()
        torch.cuda.synchronize()
        present = sorted(set(int(c) for c in np.where(sizes <= 1, 0, np.ceil(np.log2(np.maximum(sizes, 2))))))
        names = {wrs.WRS_TABLE_ALIAS: "alias", wrs.WRS_TABLE_REJECTION: "rejection"}
        mixed_info = {"all_alias_ms": round(batched_ms, 4),
                      "kinds_by_size_class": {f"n<=2^{c}": names.get(int(cls[c]), "skip") for c in present},
                      "class_ms_alias_vs_rejection": {f"n<=2^{c}": [round(float(cms[c, 0]), 3),
                                                                     round(float(cms[c, 1]), 3)] for c in present},
                      "rejection_tables": int((kinds == wrs.WRS_TABLE_REJECTION).sum()),
                      "kernels_per_replay": batched_kernels_per_replay(sizes, int(opts.small_table_items), False,
                                                                       kinds)}
        mixed_ms = e0.elapsed_time(e1) / reps
        mixed_info["mixed_graph_ms"] = round(mixed_ms, 4)
        if mixed_info["rejection_tables"]:
            batched_ms = mixed_ms
            batched_wall_ms = (time.perf_counter() - t0) * 1e3 / reps
        else:
            # every class chosen alias: the mixed call computes what wrs_batched_build_sample does,
            # and the step is that call (timed above, L2 flushed before each replay)
            mixed_info["step"] = "all kinds alias: wrs_batched_build_sample (the mixed graph timed beside it)"
            mixed_info["kernels_per_replay"] = batched_kernels_per_replay(sizes, int(opts.small_table_items), True)

    # per-table launches: build + the table's samples, one call each, per size class
    per_ms = per_wall_ms = 0.0
    timed = []
    per_equal = True
    for grp, cls in per_table_groups:
        big = int(sizes[grp].max())
        scr1 = torch.empty(wrs.alias_build_scratch_bytes(big), dtype=torch.uint8, device=dev)
        tbl_p = torch.zeros_like(table)
        out_p = torch.zeros_like(out)

        def per_table(ts):  # wrs_batched_per_table: a native loop of one build and one sample call per table
            st = wrs.batched_per_table(w, off, soff, ts, tbl_p, SEED_SAMPLES, out_p, scr1)
            if st:
                raise wrs.WrsError(st, "per-table loop")

        per_table(grp[:8])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record()
        per_table(grp)
        e1.record()
        torch.cuda.synchronize()
        # the per-table launches give the batch's rows and samples for these tables
        if not mixed:
            rows_p = tbl_p.cpu().numpy().view(np.uint32).reshape(-1, 2)
            out_pn, out_bn = out_p.cpu().numpy(), out.cpu().numpy()
            for t in grp[:256]:
                per_equal &= bool(np.array_equal(rows_p[off[t]:off[t + 1]], rows[off[t]:off[t + 1]]))
                per_equal &= bool(np.array_equal(out_pn[soff[t]:soff[t + 1]], out_bn[soff[t]:soff[t + 1]]))
        scale = int(cls.sum()) / grp.size
        per_ms += e0.elapsed_time(e1) * scale
        per_wall_ms += (time.perf_counter() - t0) * 1e3 * scale
        timed.append(f"{grp.size} tables of {int(cls.sum())}")
    return {
        "workload": what, "items": items, "samples": total,
        "autotuned": {"small_table_items": int(opts.small_table_items), "tile_items": int(opts.tile_items)},
        "batched_ms": round(batched_ms, 4), "batched_wall_ms": round(batched_wall_ms, 4),
        "step": "wrs_batched_build_sample (one call, captured in a CUDA graph)",
        "kernels_per_replay": (mixed_info["kernels_per_replay"] if mixed_info else
                               batched_kernels_per_replay(sizes, int(opts.small_table_items), True)),
        "separate_build_then_sample_ms": round(separate_ms, 4),
        "l2": ("mixed graph: inputs larger than L2, replays back to back; all-alias graph: L2 flushed "
               "before every replay" if mixed else "L2 flushed (256 MiB write) before every replay"),
        "e2e": {"value": round((items + total) / (batched_e2e_ms * 1e-3) / 1e9, 3), "unit": UNIT,
                "ms_per_step": round(batched_e2e_ms, 4), "h2d_bytes_per_step": h2d_bytes,
                "d2h_bytes_per_step": 4 * total, "path": "all-alias graph"},
        "batched_g_items_plus_samples_s": round((items + total) / (batched_ms * 1e-3) / 1e9, 3),
        "per_table_ms": round(per_ms, 2), "per_table_wall_ms": round(per_wall_ms, 2),
        "per_table_sample": "timed on " + ", ".join(timed) + " per size class, scaled by table count",
        "per_table_path": "wrs_batched_per_table (native loop: wrs_alias_build_f32 + wrs_alias_sample per table)",
        **({} if mixed else {"per_table_equal_to_batched": per_equal}),
        "speedup": round(per_ms / batched_ms, 1) if per_ms else None,
        "tables_equal_to_single_builds": f"{int(check.size) if exact else 0} of {int(check.size)} checked",
        **({"mixed": mixed_info} if mixed_info else {}),
    }


def batched_once(args, dev) -> dict:
    """One wrs_batched_build_sample call (the config 4 step) of configuration 4 or 5 with a
    fixed launch shape (alias tables only), for profiler captures."""
    import torch
    import wrs
    sizes, w_np, counts, what, _ = (batch_config5 if args.config == "5" else batch_config4)()
    nt = sizes.size
    off = np.zeros(nt + 1, dtype=np.int64)
    np.cumsum(sizes, out=off[1:])
    soff = np.zeros(nt + 1, dtype=np.int64)
    np.cumsum(counts, out=soff[1:])
    small, tile = (int(x) for x in (args.shape or "128,1024").split(","))
    opts = wrs.build_opts(0, tile, True, small)
    w = torch.from_numpy(w_np).to(dev)
    d_off, d_soff = torch.from_numpy(off).to(dev), torch.from_numpy(soff).to(dev)
    table = torch.empty(int(off[-1]), dtype=torch.int64, device=dev)
    out = torch.empty(int(soff[-1]), dtype=torch.int32, device=dev)
    scratch = torch.empty(wrs.batched_build_sample_scratch_bytes(off, opts), dtype=torch.uint8, device=dev)
    st = wrs.batched_build_sample(w, d_off, off, table, d_soff, int(soff[-1]), SEED_SAMPLES, out, scratch, opts)
    torch.cuda.synchronize()
    if st:
        raise wrs.WrsError(st, "batched once")
    return {"workload": what, "shape": [small, tile], "items": int(off[-1]), "samples": int(soff[-1])}


def shard_of(make, rank: int, world: int):
    """The tables of shard `rank` of `world` as a batch of their own: contiguous table ranges
    balanced by items plus 16 per table (wrs_shard_tables), no exchange between shards; no
    per-table baseline."""
    def make_shard():
        import wrs
        sizes, w_np, counts, what, _ = make()
        off = np.zeros(sizes.size + 1, np.int64)
        np.cumsum(sizes, out=off[1:])
        st, b = wrs.shard_tables(off, world, 16)
        if st:
            raise wrs.WrsError(st, "shard_tables")
        t0, t1 = int(b[rank]), int(b[rank + 1])
        return (sizes[t0:t1], w_np[off[t0]:off[t1]], counts[t0:t1],
                what + f"; shard {rank} of {world}: tables [{t0}, {t1})", [])
    return make_shard


def run_batched_only(args, rank: int, world: int, local_rank: int):
    """Configurations 4 and 5 alone. With N > 1 processes the batch is sharded over the devices
    by table ranges (strong scaling: the batch is fixed, each device builds and samples its
    shard, no exchange); the time is the slowest rank's."""
    import torch
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    make = batch_config5 if args.config == "5" else batch_config4
    if world == 1:
        if args.once:
            return {"once": batched_once(args, dev)}
        b = batched_phase(dev, make, mixed=args.config == "5", shape=args.shape)
        items_samples = b["items"] + b["samples"]
        return {"metric": METRIC, "value": b["batched_g_items_plus_samples_s"], "unit": UNIT, "n_gpus": 1,
                "steps": 20, "warmup": 3, "ms_per_step": b["batched_ms"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": b["workload"], "items": b["items"], "samples": b["samples"]},
                "batched": b,
                "gpu_launches": b["kernels_per_replay"] * 20,
                "e2e": b["e2e"], "note": f"{items_samples} items+samples per graph replay"}
    b = batched_phase(dev, shard_of(make, rank, world), mixed=args.config == "5", shape=args.shape)
    slowest = max_over_ranks(b["batched_ms"], dev)
    units = torch.tensor([float(b["items"] + b["samples"])], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(units)
    if rank != 0:
        return None
    total = int(units.item())
    return {"metric": METRIC, "value": round(total / (slowest * 1e-3) / 1e9, 4), "unit": UNIT, "n_gpus": world,
            "steps": 20, "warmup": 3, "ms_per_step": round(slowest, 4), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": b["workload"].split("; shard")[0] + f"; sharded over {world} devices by table ranges",
                       "items_plus_samples": total, "parallelism": f"table shards x{world}"},
            "batched_rank0": b,
            "gpu_launches": b["kernels_per_replay"] * 20,
            "e2e": b["e2e"]}


# ---------------------------------------------------------------- reference CPU

class ReferenceCpuPath:
    """The reference's CPU path of the single-table workload on this host's cores, one full step
    at a time: AliasTableSplit::build (AliasTableSplit.cu:24-80) with its split and pack loops
    (the reference's own SplitMethodBasic::split and PackMethodSweep::pack, compiled from its
    sources) spread over all threads, then the step's samples drawn by the doSample decision
    (SamplerGpuBasic.cu:28-69) restated on all threads over the contract's Philox stream, every
    sample written to host memory. Without the compiled reference, the oracle's restatement of
    the split build stands in (kind "port"). The reference's own SamplerCpu::sample (one thread,
    rand()) is timed once on a bounded sample as a side figure."""

    def __init__(self, w_np: np.ndarray, m: int, threads: int | None = None):
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import py_oracle  # the reference arm and the CPU-baseline leg are where bench.py runs the oracle

        self.po = py_oracle
        self.threads = threads or os.cpu_count() or 1
        self.w64 = np.ascontiguousarray(w_np, dtype=np.float64)
        self.n, self.m = self.w64.size, m
        self.p = 64 * self.threads
        self.kind = "reference" if py_oracle.ref_available() else "port"
        self.out = np.zeros(m, dtype=np.uint32)
        self.out[::1024] = 1  # fault the pages in before the first timed step
        self.rows = None

    def build(self) -> float:
        po = self.po
        if self.kind == "reference":
            wt, al, W, t = po.ref_split_build_parallel(self.w64, self.p, self.threads)
        else:
            t0 = time.perf_counter()
            wt, al, W, _ = po.split_build(self.w64, self.p, self.threads)
            t = time.perf_counter() - t0
        # the table in the sampler's row format (a format change, outside the timing)
        rows = np.zeros((self.n, 2), dtype=np.uint32)
        rows[:, 0] = (wt / (W / self.n)).astype(np.float32).view(np.uint32)
        rows[:, 1] = np.clip(al, 0, self.n - 1).astype(np.uint32)
        self.rows, self.weight, self.alias, self.W = rows, wt, al, W
        return t

    def sample(self, m: int | None = None, seed: int = SEED_SAMPLES) -> float:
        m = self.m if m is None else m
        rate = self.po.oracle().or_sample_plain_timed(self.po._p(self.rows), self.n, m, seed, self.threads,
                                                      self.po._p(self.out))
        return m / rate

    def step(self) -> tuple[float, float]:
        return self.build(), self.sample()

    def sampler_cpu_side(self, m: int = 1 << 21) -> dict:
        if self.kind != "reference":
            return {}
        t, _ = self.po.ref_sampler_cpu(self.weight, self.alias, self.W, m)
        return {"sampler_cpu_1thread_gsamples_s": round(m / t / 1e9, 5), "sampler_cpu_samples": m}

    def describe(self, m: int | None = None) -> str:
        m = self.m if m is None else m
        b = (f"reference AliasTableSplit split+pack loops on {self.threads} threads (p={self.p})"
             if self.kind == "reference" else f"oracle restatement of AliasTableSplit::build on {self.threads} threads")
        return (f"{b} over all {self.n} weights; doSample restated with Philox on {self.threads} threads for "
                f"{m} samples written to host memory")


def cpu_baseline(w_np: np.ndarray, m_total: int = N_SAMPLES, m_sample: int = 1 << 26) -> dict:
    """The reference's CPU path on this host's cores (ReferenceCpuPath), on a bounded sample of
    the workload: one full build, and m_sample of the step's m_total samples; the step time is
    t_build + m_total / sample_rate."""
    ref = ReferenceCpuPath(w_np, min(m_sample, m_total))
    t_build = ref.build()
    t_samp = ref.sample()
    sample_rate = ref.m / t_samp
    t_step = t_build + m_total / sample_rate
    n = w_np.size
    return {"value": round((n + m_total) / t_step / 1e9, 6), "unit": UNIT, "cores": ref.threads, "kind": ref.kind,
            "sample": ref.describe() + f"; step time = t_build + m/sample_rate (m={m_total})",
            "build_gitems_s": round(n / t_build / 1e9, 5), "sample_gsamples_s": round(sample_rate / 1e9, 5),
            "step_s": round(t_step, 2), **ref.sampler_cpu_side()}


REF_BUDGET_S = 150.0  # timed seconds of the reference arm's steps


def run_reference(args, rank: int):
    """The reference arm: the reference's CPU path (ReferenceCpuPath) on this host's cores,
    rank 0 only, timing the full configured step (the n = 2^26 build and all 2^30 samples)
    every step; one untimed warm-up step."""
    if rank != 0:
        return None
    w_np = make_weights()
    ref = ReferenceCpuPath(w_np, N_SAMPLES)
    est = 0.0
    for _ in range(min(args.warmup, 1)):
        tb, ts = ref.step()
        est = tb + ts
    # every timed step is the full configured step; so that the run ends within a few minutes,
    # at most as many steps as fit in REF_BUDGET_S (at least 3) are timed, and the line says so
    steps = args.steps if est <= 0 else min(args.steps, max(3, int(REF_BUDGET_S // est)))
    t_builds, t_samps = [], []
    t0 = time.time()
    for _ in range(steps):
        tb, ts = ref.step()
        t_builds.append(tb)
        t_samps.append(ts)
    wall = time.time() - t0
    steps_s = [b + s for b, s in zip(t_builds, t_samps)]
    step_s = statistics.median(steps_s)
    value = round((N_ITEMS + N_SAMPLES) / step_s / 1e9, 6)
    side = ref.sampler_cpu_side()
    cpu = {"value": value, "unit": UNIT, "cores": ref.threads, "kind": ref.kind,
           "legs": {"build": ref.kind, "sample": "port (doSample restated over the contract's Philox stream)"},
           "sample": ref.describe() + "; every step the full configured step",
           "build_s_median": round(statistics.median(t_builds), 3),
           "sample_s_median": round(statistics.median(t_samps), 3),
           "build_gitems_s": round(N_ITEMS / statistics.median(t_builds) / 1e9, 5),
           "sample_gsamples_s": round(N_SAMPLES / statistics.median(t_samps) / 1e9, 5),
           "timed_s_total": round(sum(steps_s), 1), "wall_s": round(wall, 1), **side}
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "steps_requested": args.steps, "warmup": min(args.warmup, 1), "ms_per_step": round(step_s * 1e3, 1),
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_items": N_ITEMS, "n_samples_per_step": N_SAMPLES},
            "impl": "reference", "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-tables measurement")
    ap.add_argument("--no-side", action="store_true",
                    help="skip the summaries of configurations 1, 3 and 5 in the default line")
    ap.add_argument("--log2-samples", type=int, default=0,
                    help="samples per step (2^k, 0 = the configuration's); for profiler captures only")
    ap.add_argument("--config", default="2", choices=sorted(CONFIGS) + ["4", "5"],
                    help="workload: 2 (default, headline: n=2^26 table; includes the batched phase), 1 (n=2^20), 3 (n=2^28), "
                         "or 4 / 5 (the batched-tables workloads only)")
    ap.add_argument("--shape", default="",
                    help="batched configurations: small_table_items,tile_items instead of the autotuner's")
    ap.add_argument("--once", action="store_true",
                    help="batched configurations: one build and one sampling call, no timing (profiler captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank)
    else:
        if world > 1:
            import datetime

            import torch
            torch.cuda.set_device(local_rank)
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        if args.config in ("4", "5"):
            line = run_batched_only(args, rank, world, local_rank)
        else:
            line = run_ours(args, rank, world, local_rank)
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
