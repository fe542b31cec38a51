"""Parity pinned to the reference's own GPU code (compiled from its sources for sm_100a into
oracle/_ref/libref_gpu.so; test infrastructure only).

* Sampling: the reference's doSample<ArrayOfStructs> and doSample<StructOfArrays>
  (sampling/aliasTable/SamplerGpuBasic.cu:28-69) run on this library's table, exported in the
  reference's row format with W_N = 1 (W = n, so each row's weight is its FP32 probability
  exactly), and on the uniforms u = (row + coin) / n of the library's Philox contract. For
  power-of-two n, u * n recovers (row, coin) exactly, and every sample must equal the library
  sampler's. For other n the FP64 round trip can move a sample across a row or coin boundary;
  every mismatch must be one of those.
* Rejection build: the reference's slot-count scan and fillABinarySearch
  (construction/rejectionSampling/RejectionSampling.cu:26-56,
  RejectionSamplingBinarySearch.cu:12-37) on the same weights (FP32 -> FP64 exactly) with the
  library's weight total W: |A| and every slot's item must match, and the library's first-slot
  bits must mark the reference's first slots.
* Rejection acceptance: the reference forms N * weight in FP32 before dividing by W
  (SamplerRejection.cu:27); the library forms it in FP64 (wrs_common.cuh, rej_item). The
  fractions are compared with that rounding difference as the stated bound.
The reference's rejection sampler itself (an unbounded retry loop) is never run.
"""
import numpy as np
import pytest
import torch

import py_oracle as po
import wrs
from gpu_util import gpu_build
from test_oracle_precision import gen

pytestmark = pytest.mark.gpu
SEED = 0xD05A


@pytest.fixture(scope="module")
def ref_gpu(cuda):
    if not po.ref_gpu_available():
        pytest.skip("oracle/_ref/libref_gpu.so not built (it needs the reference checkout at build time)")
    return po.ref_gpu()


def bench_weights(n, seed=7):
    rng = np.random.default_rng(seed)
    return ((np.arange(1, n + 1, dtype=np.float64) ** -1.1).astype(np.float32))[rng.permutation(n)]


def reference_samples(ref_gpu, rows, u, layout):
    """The reference's doSample on the table `rows` (n x {f32 prob, u32 alias}) exported with
    W = n, over the uniforms u."""
    n = rows.shape[0]
    table = torch.from_numpy(rows.view(np.int64).reshape(-1)).cuda()
    weight = torch.zeros(n, dtype=torch.float64, device="cuda")
    alias = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert wrs.export_reference_table(table, float(n), weight, alias) == wrs.WRS_SUCCESS
    torch.cuda.synchronize()
    # W_N = 1: the exported weight is the stored probability itself
    assert np.array_equal(weight.cpu().numpy(), rows[:, 0].view(np.float32).astype(np.float64))
    d_u = torch.from_numpy(u).cuda()
    out = torch.full((u.size,), -1, dtype=torch.int32, device="cuda")
    fn = ref_gpu.ref_gpu_do_sample_aos if layout == "aos" else ref_gpu.ref_gpu_do_sample_soa
    rc = fn(weight.data_ptr(), alias.data_ptr(), n, 1.0, d_u.data_ptr(), out.data_ptr(), u.size)
    assert rc == 0, f"reference doSample: CUDA error {rc}"
    return out.cpu().numpy().view(np.uint32)


def library_samples(rows, m, seed, cbase):
    n = rows.shape[0]
    table = torch.from_numpy(rows.view(np.int64).reshape(-1)).cuda()
    out = torch.empty(m, dtype=torch.int32, device="cuda")
    assert wrs.alias_sample(table, n, m, seed, out, cbase, sync=True) == wrs.WRS_SUCCESS
    return out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("layout", ["aos", "soa"])
@pytest.mark.parametrize("name,log2n,log2m", [
    ("uniform", 20, 24),            # the plain single-table configuration's shape (2^20 items, 2^24 samples)
    ("bench", 22, 22),              # the large configuration's weights, smaller
    ("loguniform", 16, 20),
    ("one_heavy", 12, 20),
])
def test_reference_do_sample_equals_library_sampler(ref_gpu, layout, name, log2n, log2m):
    n, m, cbase = 1 << log2n, 1 << log2m, 1234567
    w = bench_weights(n) if name == "bench" else gen(name, n)
    st, rows, _ = gpu_build(w)
    assert st == 0
    u, r, c = po.plain_replay_uniforms(n, m, SEED, cbase)
    assert np.array_equal(np.floor(u * n).astype(np.int64), r) and np.array_equal(u * n - r, c.astype(np.float64))
    got = library_samples(rows, m, SEED, cbase)
    ref = reference_samples(ref_gpu, rows, u, layout)
    mismatches = int(np.count_nonzero(got != ref))
    assert mismatches == 0, f"{mismatches} of {m} samples differ from the reference's doSample"


def test_reference_do_sample_on_the_large_configuration(ref_gpu):
    """n = 2^26 permuted power law (the bench table), 2^24 samples, AoS rows."""
    n, m = 1 << 26, 1 << 24
    st, rows, _ = gpu_build(bench_weights(n, seed=0x5EED + 2))
    assert st == 0
    u, _, _ = po.plain_replay_uniforms(n, m, SEED, 99)
    got = library_samples(rows, m, SEED, 99)
    ref = reference_samples(ref_gpu, rows, u, "aos")
    assert int(np.count_nonzero(got != ref)) == 0


@pytest.mark.parametrize("n", [1000, 100_003, 3 * (1 << 18) + 1])
def test_reference_do_sample_non_power_of_two_mismatches_are_round_trip_losses(ref_gpu, n):
    """For other n, u = (row + coin) / n is rounded; a sample may differ from the library's
    only where u * n no longer gives back the same row or the same coin."""
    m = 1 << 20
    st, rows, _ = gpu_build(gen("uniform", n))
    assert st == 0
    u, r, c = po.plain_replay_uniforms(n, m, SEED, 5)
    un = u * n
    row_back = np.floor(un).astype(np.int64)
    lost = (row_back != r) | (un - np.floor(un) != c.astype(np.float64))
    got = library_samples(rows, m, SEED, 5)
    ref = reference_samples(ref_gpu, rows, u, "aos")
    diff = got != ref
    assert not np.any(diff & ~lost), "a mismatch where the round trip was exact"
    assert diff.sum() <= lost.sum()


def library_rejection(w):
    n = w.size
    d_w = torch.from_numpy(w).cuda()
    A = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    frac = torch.zeros(n, dtype=torch.float32, device="cuda")
    a_size = torch.zeros(1, dtype=torch.int64, device="cuda")
    W = torch.zeros(1, dtype=torch.float64, device="cuda")
    scratch = torch.empty(wrs.rejection_build_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    assert wrs.rejection_build(d_w, A, frac, a_size, scratch, W, sync=True) == wrs.WRS_SUCCESS
    k = int(a_size.item())
    return A[:k].cpu().numpy().view(np.uint32), frac.cpu().numpy(), W.item()


def reference_rejection(ref_gpu, w, W):
    n = w.size
    d_w = torch.from_numpy(w.astype(np.float64)).cuda()
    A = torch.full((2 * n + 1,), -1, dtype=torch.int32, device="cuda")
    size = np.zeros(1, dtype=np.int64)
    rc = ref_gpu.ref_gpu_rejection_build(d_w.data_ptr(), n, W, A.data_ptr(), A.numel(), size.ctypes.data)
    assert rc == 0, f"reference rejection build: CUDA error {rc}"
    frac = torch.zeros(n, dtype=torch.float32, device="cuda")
    rc = ref_gpu.ref_gpu_rejection_fraction(d_w.data_ptr(), n, W, frac.data_ptr())
    assert rc == 0
    return A[:int(size[0])].cpu().numpy(), frac.cpu().numpy()


@pytest.mark.parametrize("name,n", [("uniform", 1 << 20), ("bench", 1 << 22), ("loguniform", 100_003),
                                    ("exp", 65_536), ("one_heavy", 4096), ("zeros_mix", 10_007), ("tiny_and_huge", 9973)])
def test_reference_rejection_build_equals_library(ref_gpu, name, n):
    w = bench_weights(n) if name == "bench" else gen(name, n)
    A, frac, W = library_rejection(w)
    A_ref, frac_ref = reference_rejection(ref_gpu, w, W)
    assert A.size == A_ref.size, f"|A| {A.size} vs the reference's {A_ref.size}"
    items = (A & 0x7FFFFFFF).astype(np.int64)
    assert np.array_equal(items, A_ref.astype(np.int64))
    first_ref = np.ones(A_ref.size, dtype=bool)
    first_ref[1:] = A_ref[1:] != A_ref[:-1]
    assert np.array_equal((A >> 31).astype(bool), first_ref)
    check_fractions(w, W, frac, frac_ref)


def test_reference_rejection_build_on_the_large_configuration(ref_gpu):
    w = bench_weights(1 << 26, seed=0x5EED + 2)
    A, frac, W = library_rejection(w)
    A_ref, frac_ref = reference_rejection(ref_gpu, w, W)
    assert A.size == A_ref.size
    assert np.array_equal((A & 0x7FFFFFFF).astype(np.int64), A_ref.astype(np.int64))
    check_fractions(w, W, frac, frac_ref)


def check_fractions(w, W, frac, frac_ref):
    """The library's FP64 n*w/W against the reference's FP32 N*weight: equal up to the FP32
    rounding of N*weight (relative 2^-24) and of the fractions themselves (2^-24 each), except
    where x = n*w/W lies that close to an integer and the two sides floor differently."""
    n = w.size
    x = n * w.astype(np.float64) / W
    tol = x * 2.0 ** -22 + 2.0 ** -22
    d = np.abs(frac.astype(np.float64) - frac_ref.astype(np.float64))
    wrapped = d > 0.5  # one side floored to the next integer
    near_int = np.abs(x - np.round(x)) <= tol
    assert np.all(d[~wrapped] <= tol[~wrapped]), f"max excess {np.max(d[~wrapped] - tol[~wrapped]):.3g}"
    assert np.all(near_int[wrapped])


def test_reference_sampling_harness_runs(ref_gpu):
    """The timing harness over the reference's XORWOW generator and doSample (used by
    oracle/ref_gpu_bench.py) runs on an exported table and returns only row indices (their XOR
    stays below n = 2^12)."""
    n = 1 << 12
    st, rows, W = gpu_build(gen("uniform", n))
    assert st == 0
    table = torch.from_numpy(rows.view(np.int64).reshape(-1)).cuda()
    weight = torch.zeros(n, dtype=torch.float64, device="cuda")
    alias = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert wrs.export_reference_table(table, float(n), weight, alias) == wrs.WRS_SUCCESS
    torch.cuda.synchronize()
    ms, chk = np.zeros(1, np.float32), np.zeros(1, np.uint32)
    rc = ref_gpu.ref_gpu_sample_timed(weight.data_ptr(), alias.data_ptr(), n, 1.0, 4, 64, 16, 7,
                                      ms.ctypes.data, chk.ctypes.data)
    assert rc == 0 and ms[0] > 0
    assert int(chk[0]) < (1 << 12)  # an XOR of row indices below 2^12
