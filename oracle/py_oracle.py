"""py_oracle — ctypes access to the CPU oracle (liboracle.so) and the compiled reference
(_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU-baseline
arm of bench.py, never by the library.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")
REF_DBG_SO = os.path.join(HERE, "_ref", "libref_dbg.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libref_gpu.so")

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32
_D = ctypes.c_double
_I = ctypes.c_int

_oracle = None
_ref = {}


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def oracle() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        sig = {
            "or_exact_sum_f32": (_D, [_P, _I64]),
            "or_philox4x32_10": (None, [_P, _P, _P]),
            "or_sweep_build": (_I, [_P, _I64, _P, _P, _P]),
            "or_sweep_build_f32": (_I, [_P, _I64, _P, _P, _P]),
            "or_check_ref_table_w": (_I, [_P, _I64, _P, _P, _D, _D, _P]),
            "or_split_build": (_I, [_P, _I64, _I64, _P, _P, _P, _I]),
            "or_check_table": (_I, [_P, _I64, _P, _P, _P]),
            "or_check_ref_table": (_I, [_P, _I64, _P, _P, _D, _P]),
            "or_exact_build": (_I, [_P, _I64, _D, _P]),
            "or_sample_plain": (None, [_P, _I64, _U64, _U64, _U64, _P]),
            "or_plain_replay_uniforms": (None, [_I64, _U64, _U64, _U64, _P, _P, _P]),
            "or_prec_build": (_I, [_P, _I64, _I, _P, _P]),
            "or_binomial": (_U64, [_U64, _D, _U32, _U32, _U64, _U32]),
            "or_section_counts": (None, [_I64, _U32, _U64, _U64, _U64, _P]),
            "or_sample_sectioned": (None, [_P, _I64, _U64, _U32, _U64, _U64, _P, _P]),
            "or_rejection_build": (_U64, [_P, _I64, _D, _P, _U64, _P]),
            "or_rejection_sample": (_I, [_P, _U64, _P, _U64, _U64, _U64, _U32, _P]),
            "or_sample_plain_timed": (_D, [_P, _I64, _U64, _U64, _I, _P]),
            "or_batched_build": (_I, [_P, _P, _I64, _P, _P]),
            "or_psa_plus_build": (_I, [_P, _I64, _D, _I64, _P]),
            "or_batched_sample": (None, [_P, _P, _I64, _P, _U64, _U64, _P]),
            "or_batched_mixed_build": (_I, [_P, _P, _I64, _P, _P, _P, _P, _P, _P]),
            "or_batched_mixed_sample": (_I, [_P, _P, _P, _P, _P, _I64, _P, _P, _U64, _U64, _U32, _P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _oracle = L
    return _oracle


def ref_available(debug: bool = False) -> bool:
    return os.path.exists(REF_DBG_SO if debug else REF_SO)


def ref(debug: bool = False) -> ctypes.CDLL:
    key = "dbg" if debug else "rel"
    if key not in _ref:
        L = ctypes.CDLL(REF_DBG_SO if debug else REF_SO)
        sig = {
            "ref_split_build": (_I, [_P, _I, _I, _P, _P, _P, _P]),
            "ref_sweep_build": (_I, [_P, _I, _P, _P, _P, _P]),
            "ref_stack_build": (_I, [_P, _I, _P, _P, _P, _P]),
            "ref_verify": (_I, [_P, _I, _P, _P, _D]),
            "ref_np_table": (_I, [_I, _I, _P, _P, _P, _P]),
            "ref_generate": (_I, [_I, _I, _P]),
            "ref_split_build_parallel": (_I, [_P, _I, _I, _I, _P, _P, _P, _P]),
            "ref_sampler_cpu": (_D, [_P, _P, _I, _D, ctypes.c_longlong, _P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _ref[key] = L
    return _ref[key]


def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


def ref_gpu() -> ctypes.CDLL:
    """The reference's own GPU code (doSample, the rejection build and acceptance), compiled
    from its sources for sm_100a (test infrastructure; needs a GPU to call)."""
    if "gpu" not in _ref:
        L = ctypes.CDLL(REF_GPU_SO)
        sig = {
            "ref_gpu_do_sample_aos": (_I, [_P, _P, _I, _D, _P, _P, _I]),
            "ref_gpu_do_sample_soa": (_I, [_P, _P, _I, _D, _P, _P, _I]),
            "ref_gpu_rejection_build": (_I, [_P, _I, _D, _P, ctypes.c_longlong, _P]),
            "ref_gpu_rejection_fraction": (_I, [_P, _I, _D, _P]),
            "ref_gpu_sample_timed": (_I, [_P, _P, _I, _D, _I, _I, ctypes.c_longlong, ctypes.c_ulonglong, _P, _P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _ref["gpu"] = L
    return _ref["gpu"]


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


# ---------------------------------------------------------------- oracle wrappers

def exact_sum(w: np.ndarray) -> float:
    w = np.ascontiguousarray(w, dtype=np.float32)
    return oracle().or_exact_sum_f32(_p(w), w.size)


def philox(ctr, key) -> np.ndarray:
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    oracle().or_philox4x32_10(_p(c), _p(k), _p(o))
    return o


def sweep_build(w64: np.ndarray):
    w64 = np.ascontiguousarray(w64, dtype=np.float64)
    n = w64.size
    wt = np.zeros(n, dtype=np.float64)
    al = np.zeros(n, dtype=np.int32)
    W = ctypes.c_double()
    oracle().or_sweep_build(_p(w64), n, _p(wt), _p(al), ctypes.byref(W))
    return wt, al, W.value


def sweep_build_f32(w: np.ndarray):
    """The sweep with every quantity in FP32; returns (row weights, aliases, W_N of the build)."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    n = w.size
    wt = np.zeros(n, dtype=np.float64)
    al = np.zeros(n, dtype=np.int32)
    W = ctypes.c_double()
    oracle().or_sweep_build_f32(_p(w), n, _p(wt), _p(al), ctypes.byref(W))
    W_N = float(np.float32(W.value) / np.float32(n))
    return wt, al, W_N


def check_ref_table_w(w: np.ndarray, weight: np.ndarray, alias: np.ndarray, W_N_table: float,
                      W_exact: float) -> dict:
    """A reference-format table on its own scale W_N_table against n w_i / W_exact."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    weight = np.ascontiguousarray(weight, dtype=np.float64)
    alias = np.ascontiguousarray(alias, dtype=np.int32)
    st = np.zeros(5, dtype=np.float64)
    oracle().or_check_ref_table_w(_p(w), w.size, _p(weight), _p(alias), W_N_table, W_exact, _p(st))
    return {"max_rel": st[0], "p9999_rel": st[1], "worst": int(st[2]), "zero_mass": int(st[3]),
            "bad_rows": int(st[4])}


def split_build(w64: np.ndarray, p: int, threads: int = 1):
    w64 = np.ascontiguousarray(w64, dtype=np.float64)
    n = w64.size
    wt = np.zeros(n, dtype=np.float64)
    al = np.zeros(n, dtype=np.int32)
    W = ctypes.c_double()
    rc = oracle().or_split_build(_p(w64), n, p, _p(wt), _p(al), ctypes.byref(W), threads)
    return wt, al, W.value, rc


def check_table(w: np.ndarray, rows: np.ndarray) -> dict:
    """rows: uint32 array of shape (n, 2) = (prob bits, alias)."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    st = np.zeros(5, dtype=np.float64)
    W = ctypes.c_double()
    oracle().or_check_table(_p(w), w.size, _p(rows), _p(st), ctypes.byref(W))
    return {"max_rel": st[0], "p9999_rel": st[1], "worst": int(st[2]), "zero_mass": int(st[3]),
            "bad_rows": int(st[4]), "W": W.value}


def check_ref_table(w64: np.ndarray, weight: np.ndarray, alias: np.ndarray, W: float) -> dict:
    w64 = np.ascontiguousarray(w64, dtype=np.float64)
    weight = np.ascontiguousarray(weight, dtype=np.float64)
    alias = np.ascontiguousarray(alias, dtype=np.int32)
    st = np.zeros(5, dtype=np.float64)
    oracle().or_check_ref_table(_p(w64), w64.size, _p(weight), _p(alias), W, _p(st))
    return {"max_rel": st[0], "p9999_rel": st[1], "worst": int(st[2]), "zero_mass": int(st[3]),
            "bad_rows": int(st[4])}


def exact_build(w: np.ndarray, W: float | None = None) -> np.ndarray:
    w = np.ascontiguousarray(w, dtype=np.float32)
    if W is None:
        W = exact_sum(w)
    rows = np.zeros((w.size, 2), dtype=np.uint32)
    oracle().or_exact_build(_p(w), w.size, W, _p(rows))
    return rows


def sample_plain(rows: np.ndarray, m: int, seed: int, cbase: int = 0) -> np.ndarray:
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    out = np.zeros(m, dtype=np.uint32)
    oracle().or_sample_plain(_p(rows), rows.shape[0], m, seed, cbase, _p(out))
    return out


def prec_build(w: np.ndarray, fp64: bool):
    """The library's all-FP64 / all-FP32 comparison build (rows, W); rows None for invalid
    weights or a zero total."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    rows = np.zeros((w.size, 2), dtype=np.uint32)
    W = np.zeros(1, dtype=np.float64)
    rc = oracle().or_prec_build(_p(w), w.size, 1 if fp64 else 0, _p(rows), _p(W))
    return (None if rc else rows), float(W[0])


def plain_replay_uniforms(n: int, m: int, seed: int, cbase: int = 0):
    """u = (row + coin) / n for output positions 0..m-1 of the plain contract, with the
    (row, coin) pairs themselves."""
    u = np.zeros(m, dtype=np.float64)
    rows = np.zeros(m, dtype=np.uint32)
    coins = np.zeros(m, dtype=np.float32)
    oracle().or_plain_replay_uniforms(n, m, seed & (2**64 - 1), cbase & (2**64 - 1), _p(u), _p(rows), _p(coins))
    return u, rows, coins


def psa_plus_build(w: np.ndarray, W: float | None = None, tile: int = 2048) -> np.ndarray:
    """Rows of the PSA+ build (tile-local pre-pack, then the exact merge of the leftovers)."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    if W is None:
        W = exact_sum(w)
    rows = np.zeros((w.size, 2), dtype=np.uint32)
    oracle().or_psa_plus_build(_p(w), w.size, W, tile, _p(rows))
    return rows


def batched_build(w: np.ndarray, off: np.ndarray):
    """Rows of every CSR table (or_exact_build per table), the per-table totals, and the
    number of tables left unbuilt (zero or invalid total)."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    off = np.ascontiguousarray(off, dtype=np.int64)
    rows = np.zeros((max(1, w.size), 2), dtype=np.uint32)
    W = np.zeros(off.size - 1, dtype=np.float64)
    bad = oracle().or_batched_build(_p(w), _p(off), off.size - 1, _p(rows), _p(W))
    return rows[:w.size], W, bad


def batched_sample(rows: np.ndarray, off: np.ndarray, soff: np.ndarray, seed: int, cbase: int = 0) -> np.ndarray:
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    off = np.ascontiguousarray(off, dtype=np.int64)
    soff = np.ascontiguousarray(soff, dtype=np.int64)
    out = np.zeros(max(1, int(soff[-1])), dtype=np.uint32)
    oracle().or_batched_sample(_p(rows), _p(off), off.size - 1, _p(soff), seed & (2**64 - 1), cbase, _p(out))
    return out[:int(soff[-1])]


def binomial(n: int, p: float, seed: int, cbase: int, node: int) -> int:
    return int(oracle().or_binomial(n, p, seed & 0xffffffff, seed >> 32, cbase, node))


def section_counts(n: int, S: int, m: int, seed: int, cbase: int = 0) -> np.ndarray:
    K = (n + S - 1) // S
    c = np.zeros(K, dtype=np.uint64)
    oracle().or_section_counts(n, S, m, seed, cbase, _p(c))
    return c


def sample_sectioned(rows: np.ndarray, m: int, S: int, seed: int, cbase: int = 0):
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    n = rows.shape[0]
    K = (n + S - 1) // S
    out = np.zeros(m, dtype=np.uint32)
    c = np.zeros(K, dtype=np.uint64)
    oracle().or_sample_sectioned(_p(rows), n, m, S, seed, cbase, _p(out), _p(c))
    return out, c


def rejection_build(w: np.ndarray, W: float | None = None):
    w = np.ascontiguousarray(w, dtype=np.float32)
    if W is None:
        W = exact_sum(w)
    cap = 2 * w.size + 2
    A = np.zeros(cap, dtype=np.uint32)
    frac = np.zeros(w.size, dtype=np.float32)
    asz = oracle().or_rejection_build(_p(w), w.size, W, _p(A), cap, _p(frac))
    return A[:asz], frac


def rejection_sample(A: np.ndarray, frac: np.ndarray, m: int, seed: int, cbase: int = 0, max_tries: int = 0):
    A = np.ascontiguousarray(A, dtype=np.uint32)
    frac = np.ascontiguousarray(frac, dtype=np.float32)
    out = np.zeros(m, dtype=np.uint32)
    failed = oracle().or_rejection_sample(_p(A), A.size, _p(frac), m, seed, cbase, max_tries, _p(out))
    return out, failed


def sample_plain_timed(rows: np.ndarray, m: int, seed: int, threads: int) -> float:
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    out = np.zeros(m, dtype=np.uint32)
    return oracle().or_sample_plain_timed(_p(rows), rows.shape[0], m, seed, threads, _p(out))


# ---------------------------------------------------------------- compiled reference

def ref_split_build(w64: np.ndarray, p: int, debug: bool = False):
    w64 = np.ascontiguousarray(w64, dtype=np.float64)
    n = w64.size
    wt = np.zeros(n, dtype=np.float64)
    al = np.zeros(n, dtype=np.int32)
    W = ctypes.c_double()
    sec = ctypes.c_double()
    ref(debug).ref_split_build(_p(w64), n, p, _p(wt), _p(al), ctypes.byref(W), ctypes.byref(sec))
    return wt, al, W.value, sec.value


def ref_sweep_build(w64: np.ndarray):
    w64 = np.ascontiguousarray(w64, dtype=np.float64)
    n = w64.size
    wt = np.zeros(n, dtype=np.float64)
    al = np.zeros(n, dtype=np.int32)
    W = ctypes.c_double()
    sec = ctypes.c_double()
    ref().ref_sweep_build(_p(w64), n, _p(wt), _p(al), ctypes.byref(W), ctypes.byref(sec))
    return wt, al, W.value, sec.value


def ref_stack_build(w64: np.ndarray):
    w64 = np.ascontiguousarray(w64, dtype=np.float64)
    n = w64.size
    wt = np.zeros(n, dtype=np.float64)
    al = np.zeros(n, dtype=np.int32)
    W = ctypes.c_double()
    sec = ctypes.c_double()
    ref().ref_stack_build(_p(w64), n, _p(wt), _p(al), ctypes.byref(W), ctypes.byref(sec))
    return wt, al, W.value, sec.value


def ref_split_build_parallel(w64: np.ndarray, p: int, threads: int):
    w64 = np.ascontiguousarray(w64, dtype=np.float64)
    n = w64.size
    wt = np.zeros(n, dtype=np.float64)
    al = np.zeros(n, dtype=np.int32)
    W = ctypes.c_double()
    sec = ctypes.c_double()
    ref().ref_split_build_parallel(_p(w64), n, p, threads, _p(wt), _p(al), ctypes.byref(W), ctypes.byref(sec))
    return wt, al, W.value, sec.value


def ref_verify(w64, weight, alias, W) -> bool:
    w64 = np.ascontiguousarray(w64, dtype=np.float64)
    weight = np.ascontiguousarray(weight, dtype=np.float64)
    alias = np.ascontiguousarray(alias, dtype=np.int32)
    return bool(ref(True).ref_verify(_p(w64), w64.size, _p(weight), _p(alias), W))


def ref_np_table(n: int, best: bool):
    w = np.zeros(n, dtype=np.float64)
    wt = np.zeros(n, dtype=np.float64)
    al = np.zeros(n, dtype=np.int32)
    W = ctypes.c_double()
    ref().ref_np_table(n, 1 if best else 0, _p(w), _p(wt), _p(al), ctypes.byref(W))
    return w, wt, al, W.value


def ref_generate(n: int, distribution: int) -> np.ndarray:
    w = np.zeros(n, dtype=np.float64)
    ref().ref_generate(n, distribution, _p(w))
    return w


def ref_sampler_cpu(weight, alias, W: float, num_samples: int, want_out: bool = False):
    weight = np.ascontiguousarray(weight, dtype=np.float64)
    alias = np.ascontiguousarray(alias, dtype=np.int32)
    out = np.zeros(num_samples, dtype=np.int32) if want_out else None
    sec = ref().ref_sampler_cpu(_p(weight), _p(alias), weight.size, W, num_samples, _p(out) if want_out else None)
    return sec, out


def batched_mixed_build(w: np.ndarray, off: np.ndarray, kinds: np.ndarray):
    """Mixed batch: returns (rows (n, 2) u32, A (2n) u32, frac (n) f32, a_size u64, W, bad)."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    off = np.ascontiguousarray(off, dtype=np.int64)
    kinds = np.ascontiguousarray(kinds, dtype=np.uint8)
    n = int(off[-1])
    rows = np.zeros((max(n, 1), 2), dtype=np.uint32)
    A = np.zeros(max(2 * n, 1), dtype=np.uint32)
    frac = np.zeros(max(n, 1), dtype=np.float32)
    a_size = np.zeros(kinds.size, dtype=np.uint64)
    W = np.zeros(kinds.size, dtype=np.float64)
    bad = oracle().or_batched_mixed_build(_p(w), _p(off), kinds.size, _p(kinds), _p(rows), _p(A), _p(frac),
                                          _p(a_size), _p(W))
    return rows[:n], A[:2 * n], frac[:n], a_size, W, bad


def batched_mixed_sample(rows, A, frac, a_size, off, kinds, soff, seed: int, cbase: int = 0, max_tries: int = 0,
                         out: np.ndarray | None = None):
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    A = np.ascontiguousarray(A, dtype=np.uint32)
    frac = np.ascontiguousarray(frac, dtype=np.float32)
    a_size = np.ascontiguousarray(a_size, dtype=np.uint64)
    off = np.ascontiguousarray(off, dtype=np.int64)
    kinds = np.ascontiguousarray(kinds, dtype=np.uint8)
    soff = np.ascontiguousarray(soff, dtype=np.int64)
    if out is None:
        out = np.zeros(max(int(soff[-1]), 1), dtype=np.uint32)
    failed = oracle().or_batched_mixed_sample(_p(rows), _p(A), _p(frac), _p(a_size), _p(off), kinds.size, _p(kinds),
                                              _p(soff), seed, cbase, max_tries, _p(out))
    return out[:int(soff[-1])], failed

