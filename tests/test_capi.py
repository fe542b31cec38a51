"""The C ABI library loads and exports every entry point include/wrs.h declares; the
calls that need no GPU (sizes, status strings, argument checks) behave as documented."""
import ctypes
import os
import re

import pytest

import wrs

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "wrs.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wrs_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for required in ["wrs_alias_build_f32", "wrs_alias_sample", "wrs_rejection_build_f32", "wrs_rejection_sample",
                     "wrs_batched_build_f32", "wrs_batched_sample", "wrs_sum_f32", "wrs_status_string"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    L = wrs.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_library_exports_nothing_undeclared():
    # symbols come from the C ABI only (the library builds with -fvisibility=hidden)
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", wrs.LIB_PATH], capture_output=True, text=True).stdout
    exported = sorted(set(re.findall(r" T (wrs_[a-z0-9_]+)$", out, flags=re.M)))
    assert exported == declared_functions()


def test_status_strings():
    assert wrs.status_string(wrs.WRS_SUCCESS) == "success"
    for s in range(1, 10):
        assert wrs.status_string(s) not in ("", "unknown status")
    assert wrs.status_string(1234) == "unknown status"


def test_version():
    assert wrs.lib().wrs_version() == 2


def test_scratch_sizes_are_host_only_and_monotone():
    a = wrs.alias_build_scratch_bytes(1000)
    b = wrs.alias_build_scratch_bytes(1 << 20)
    c = wrs.alias_build_scratch_bytes(1 << 26)
    assert 0 < a <= b <= c
    assert wrs.alias_build_scratch_bytes(0) == 0
    bad = wrs.build_opts(tile_items=3000)
    assert wrs.alias_build_scratch_bytes(1000, bad) == 0
    assert wrs.rejection_build_scratch_bytes(1 << 20) > 0
    assert wrs.lib().wrs_sum_scratch_bytes(10) > 0


def test_argument_checks_before_any_device_work():
    L = wrs.lib()
    # null weights / table / scratch, n out of range: rejected without touching the GPU
    assert L.wrs_alias_build_f32(None, 10, None, None, None, None, 0, None) == wrs.WRS_ERR_INVALID_ARGUMENT
    assert L.wrs_alias_build_f32(16, 0, None, 16, None, 16, 1 << 20, None) == wrs.WRS_ERR_INVALID_ARGUMENT
    assert L.wrs_alias_build_f32(16, 1 << 40, None, 16, None, 16, 1 << 20, None) == wrs.WRS_ERR_INVALID_ARGUMENT
    # scratch too small
    assert L.wrs_alias_build_f32(16, 1000, None, 16, None, 16, 8, None) == wrs.WRS_ERR_SCRATCH_TOO_SMALL
    # unknown method / tile size
    opts = wrs.BuildOpts(7, 0, 0, 0)
    assert L.wrs_alias_build_f32(16, 1000, ctypes.byref(opts), 16, None, 16, 1 << 30, None) == \
        wrs.WRS_ERR_INVALID_ARGUMENT
    assert L.wrs_alias_sample(None, 10, 10, 0, 0, None, 16, None, None) == wrs.WRS_ERR_INVALID_ARGUMENT
    assert L.wrs_rejection_build_f32(None, 10, None, 0, None, None, None, None, 0, 0, None) == \
        wrs.WRS_ERR_INVALID_ARGUMENT
    assert L.wrs_rejection_sample(None, None, None, 10, 10, 0, 0, 0, None, None, 0, None) == \
        wrs.WRS_ERR_INVALID_ARGUMENT
    assert L.wrs_scratch_status(None, None) == wrs.WRS_ERR_INVALID_ARGUMENT


def test_header_compiles_as_c_and_cxx():
    # the boundary header must parse for C and C++ callers (FFI binders include it as is)
    import shutil
    import subprocess
    hdr = HEADER
    for cc, lang in (("gcc", "c"), ("g++", "c++")):
        if shutil.which(cc) is None:
            continue
        r = subprocess.run([cc, "-fsyntax-only", "-Wall", "-x", lang, hdr], capture_output=True, text=True)
        assert r.returncode == 0, f"{cc}: {r.stderr}"


def test_reference_named_sampler_variants():
    """SamplerGpuSectionedShared / SamplerRejectionGiveUp: the reference's other sampler names,
    as the sectioned sampler with staged 3000-row sections and rejection with at most 8 tries."""
    class Table:  # stands in for a built table: the constructors only keep the reference
        N, device = 10, "cpu"

    s = wrs.SamplerGpuSectionedShared(Table())
    assert s.name() == "SamplerGpuSectionedShared" and s.itemsPerSection == 3000 and s.counter == 0
    for bad in (0, 3001, 12290):
        with pytest.raises(wrs.WrsError) as e:
            wrs.SamplerGpuSectionedShared(Table(), bad)
        assert e.value.status == wrs.WRS_ERR_INVALID_ARGUMENT
    g = wrs.SamplerRejectionGiveUp(Table())
    assert g.name() == "SamplerRejectionGiveUp" and g.max_tries == 8


def test_batched_scratch_queries_plan_on_the_host():
    """The batched and mixed scratch queries run the host plan alone: valid CSR offsets give a
    size, offsets that do not start at 0 or that decrease give 0 (the builds then refuse)."""
    import numpy as np
    ok = np.array([0, 3, 3, 10, 5000, 5001], dtype=np.int64)
    a = wrs.batched_build_scratch_bytes(ok)
    assert a > 0
    # the default query covers every launch shape the autotuner may pick
    for small in (32, 64, 128, 256, 512):
        for tile in (1024, 2048, 4096):
            s = wrs.batched_build_scratch_bytes(ok, wrs.build_opts(tile_items=tile, small_table_items=small))
            assert 0 < s <= a
    assert wrs.batched_build_scratch_bytes(np.array([1, 3, 10], dtype=np.int64)) == 0
    assert wrs.batched_build_scratch_bytes(np.array([0, 5, 3], dtype=np.int64)) == 0
    kinds = np.array([wrs.WRS_TABLE_ALIAS, wrs.WRS_TABLE_REJECTION, wrs.WRS_TABLE_SKIP, wrs.WRS_TABLE_ALIAS,
                      wrs.WRS_TABLE_REJECTION], dtype=np.uint8)
    m_any = wrs.batched_mixed_build_scratch_bytes(ok)
    m_kinds = wrs.batched_mixed_build_scratch_bytes(ok, kinds)
    assert 0 < m_kinds <= m_any
    assert wrs.batched_mixed_build_scratch_bytes(np.array([0, 5, 3], dtype=np.int64)) == 0


def test_missing_library_fails_loudly():
    """Without the built CUDA library every entry point raises: there is no CPU fallback."""
    import subprocess
    import sys
    pkg = os.path.dirname(wrs.__file__)
    code = ("import sys; sys.path.insert(0, %r); import wrs; wrs.LIB_PATH = '/nonexistent/libwrs.so'\n"
            "try:\n    wrs.alias_build_scratch_bytes(1000)\nexcept RuntimeError as e:\n    print('raised', e)\n"
            "else:\n    print('no error')\n") % pkg
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("raised") and "libwrs.so not built" in r.stdout


def test_wait_limit_setters_check_their_arguments():
    assert wrs.set_device_wait_limit(0) == wrs.WRS_SUCCESS
    assert wrs.set_device_wait_limit(61 * 10 ** 9) == wrs.WRS_ERR_INVALID_ARGUMENT
    assert wrs.debug_hold_lookback(-2) == wrs.WRS_ERR_INVALID_ARGUMENT
    assert wrs.debug_hold_lookback(3) == wrs.WRS_SUCCESS
    assert wrs.debug_hold_lookback(-1) == wrs.WRS_SUCCESS


def test_precision_options_are_checked_on_the_host():
    n = 1 << 20
    assert wrs.alias_build_scratch_bytes(n, wrs.build_opts(precision=wrs.WRS_PRECISION_FP64)) > 24 * n
    assert wrs.alias_build_scratch_bytes(n, wrs.build_opts(precision=wrs.WRS_PRECISION_FP32)) > 16 * n
    assert wrs.alias_build_scratch_bytes(n, wrs.build_opts(precision=3)) == 0
    assert wrs.alias_build_scratch_bytes(
        n, wrs.build_opts(method=wrs.WRS_METHOD_PSA_PLUS, precision=wrs.WRS_PRECISION_FP64)) == 0
