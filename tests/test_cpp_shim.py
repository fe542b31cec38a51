"""The C++ shim of the reference's object surface (include/wrs.hpp).

tests/cpp/shim_check.cpp uses it as code written against the reference's classes would:
AliasTableSplitGpu / RejectionSamplingGpu with fullBuild(), SamplerGpuBasic (sample,
getSamplingDistribution, benchmarkSampling), SamplerGpuSectioned, SamplerRejection, and the
batched form (BatchedAliasTablesGpu, SamplerBatched). On the
CPU the program must compile and link against the library; on the GPU its tables and samples
must equal the oracle's (the same contracts as the C ABI tests)."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import py_oracle as po

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "cpp", "shim_check.cpp")
LIB_DIR = os.path.join(REPO, "alias-table-gpu_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def compile_shim(tmp_path, src=SRC):
    cxx = shutil.which("g++")
    if cxx is None or not os.path.exists(os.path.join(CUDA, "include", "cuda_runtime.h")):
        pytest.skip("needs g++ and the CUDA headers")
    exe = str(tmp_path / os.path.splitext(os.path.basename(src))[0])
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"),
           "-I", os.path.join(CUDA, "include"), src, "-o", exe, "-L", LIB_DIR, "-lwrs",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{LIB_DIR}:{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_compiles_and_links(tmp_path):
    compile_shim(tmp_path)


def test_shim_reference_named_variants_compile_and_link(tmp_path):
    """SamplerGpuSectionedShared and SamplerRejectionGiveUp, the reference's other sampler names."""
    exe = compile_shim(tmp_path, os.path.join(REPO, "tests", "cpp", "shim_names.cpp"))
    assert subprocess.run([exe], timeout=60).returncode == 0  # no arguments: touches no device


@pytest.mark.gpu
@pytest.mark.parametrize("kind,n", [("uniform", 5000), ("powerlaw", 100_003)])
def test_shim_matches_oracle(cuda, tmp_path, kind, n):
    exe = compile_shim(tmp_path)
    rng = np.random.default_rng(13)
    if kind == "uniform":
        w = rng.random(n, dtype=np.float32)
    else:
        w = ((np.arange(1, n + 1, dtype=np.float64) ** -1.1).astype(np.float32))[rng.permutation(n)]
    wf = tmp_path / "w.f32"
    w.tofile(wf)
    prefix = str(tmp_path / "out")
    m, seed = 100_001, 987654321
    r = subprocess.run([exe, str(wf), prefix, str(m), str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["alias"] == "AliasTableSplitGpu" and info["sampler"] == "SamplerGpuBasic"
    assert info["gsamples_per_s"] > 0
    W = info["W"]
    rows = np.fromfile(prefix + "_rows.bin", dtype=np.uint32).reshape(-1, 2)
    assert np.array_equal(rows, po.exact_build(w, W))
    assert np.array_equal(np.fromfile(prefix + "_plain.bin", dtype=np.uint32), po.sample_plain(rows, m, seed, 0))
    hist = np.fromfile(prefix + "_hist.bin", dtype=np.int64)
    assert np.array_equal(hist, np.bincount(po.sample_plain(rows, m, seed, m), minlength=n))
    sect, _ = po.sample_sectioned(rows, m, 4096, seed, 0)
    assert np.array_equal(np.fromfile(prefix + "_sect.bin", dtype=np.uint32), sect)
    A, frac = po.rejection_build(w, W)
    assert info["slots"] == A.size
    rej, failed = po.rejection_sample(A, frac, m, seed, 0)
    assert failed == 0
    assert np.array_equal(np.fromfile(prefix + "_rej.bin", dtype=np.uint32), rej)
    off = np.array([0, n // 3, n // 2, n], dtype=np.int64)
    brows = np.fromfile(prefix + "_batch_rows.bin", dtype=np.uint32).reshape(-1, 2)
    ref_b, _, _ = po.batched_build(w, off)
    assert np.array_equal(brows, ref_b)
    soff = np.array([0, 1000, 2000, 3000], dtype=np.int64)
    assert np.array_equal(np.fromfile(prefix + "_batch_samples.bin", dtype=np.uint32),
                          po.batched_sample(brows, off, soff, seed, 0))
