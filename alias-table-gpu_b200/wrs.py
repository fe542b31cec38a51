"""wrs — Python binding of the B200 weighted-random-sampling library (libwrs.so).

Two layers:

* thin ctypes wrappers over the C ABI declared in include/wrs.h (device pointers, sizes,
  streams), used with torch CUDA tensors for device memory;
* classes that keep the reference's build(weights) -> sample(n) surface
  (construction/SamplingAlgorithm.cuh:30-48, sampling/Sampler.cuh:10-31):
  ``AliasTableSplitGpu`` / ``RejectionSamplingGpu`` (preBuild, build, postBuild, fullBuild,
  name, weights, W, N) and ``SamplerGpuBasic`` / ``SamplerGpuSectioned`` / ``SamplerRejection``
  (name, benchmarkSampling, getSamplingDistribution, sample).

The CUDA path is the only path: importing this module without libwrs.so, or calling it
without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwrs.so")

WRS_SUCCESS = 0
WRS_ERR_INVALID_ARGUMENT = 1
WRS_ERR_INVALID_WEIGHT = 2
WRS_ERR_ZERO_TOTAL = 3
WRS_ERR_SCRATCH_TOO_SMALL = 4
WRS_ERR_CUDA = 5
WRS_ERR_DEVICE_TIMEOUT = 6
WRS_ERR_TOO_MANY_TRIES = 7
WRS_ERR_UNSUPPORTED = 8
WRS_ERR_CAPACITY = 9

WRS_METHOD_SPLIT = 0
WRS_METHOD_PSA_PLUS = 1
WRS_PRECISION_MIXED = 0
WRS_PRECISION_FP64 = 1
WRS_PRECISION_FP32 = 2
WRS_FLAG_SYNC = 1
WRS_SAMPLE_PLAIN = 0
WRS_SAMPLE_SECTIONED = 1
WRS_SAMPLE_HISTOGRAM = 2
WRS_SAMPLE_DISCARD = 3


class BuildOpts(ctypes.Structure):
    _fields_ = [("method", ctypes.c_uint32), ("tile_items", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("small_table_items", ctypes.c_uint32),
                ("precision", ctypes.c_uint32)]


class SampleOpts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_uint32), ("section_items", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("threads", ctypes.c_uint32)]


class WrsError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})" if what else status_string(status))


_lib = None
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32
_SZ = ctypes.c_size_t

_SIGNATURES = {
    "wrs_sum_scratch_bytes": (_SZ, [_I64]),
    "wrs_sum_f32": (ctypes.c_int, [_P, _I64, _P, _P, _SZ, _P]),
    "wrs_alias_build_scratch_bytes": (_SZ, [_I64, _P]),
    "wrs_alias_build_f32": (ctypes.c_int, [_P, _I64, _P, _P, _P, _P, _SZ, _P]),
    "wrs_alias_build_f32_static_scratch": (ctypes.c_int, [_P, _I64, _P, _P, _P, _P]),
    "wrs_alias_sample": (ctypes.c_int, [_P, _I64, _U64, _U64, _U64, _P, _P, _P, _P]),
    "wrs_alias_sample_to_host": (ctypes.c_int, [_P, _I64, _U64, _U64, _U64, _U64, _P, _P, _P]),
    "wrs_random_gather_probe": (ctypes.c_int, [_P, _I64, _U64, _U64, _P, _P]),
    "wrs_rejection_build_scratch_bytes": (_SZ, [_I64]),
    "wrs_rejection_build_f32": (ctypes.c_int, [_P, _I64, _P, _U64, _P, _P, _P, _P, _SZ, _U32, _P]),
    "wrs_rejection_sample": (ctypes.c_int, [_P, _P, _P, _I64, _U64, _U64, _U64, _U32, _P, _P, _U32, _P]),
    "wrs_rejection_pack": (ctypes.c_int, [_P, _P, _P, _I64, _U64, _P, _P]),
    "wrs_rejection_sample_packed": (ctypes.c_int, [_P, _U64, _P, _I64, _U64, _U64, _U64, _U32, _P, _P, _U32, _P]),
    "wrs_batched_build_scratch_bytes": (_SZ, [_P, _I64, _P]),
    "wrs_batched_build_f32": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P, _P, _SZ, _P]),
    "wrs_batched_sample": (ctypes.c_int, [_P, _P, _I64, _P, _U64, _U64, _U64, _P, _P]),
    "wrs_batched_build_sample_scratch_bytes": (_SZ, [_P, _I64, _P]),
    "wrs_batched_per_table": (ctypes.c_int, [_P, _P, _P, _P, _I64, _P, _P, _U64, _U64, _P, _P, _SZ, _P]),
    "wrs_batched_autotune_build_sample": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _U64, _P, _P, _SZ, _P, _P]),
    "wrs_batched_build_sample": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P, _P, _U64, _U64, _U64, _P, _P, _SZ,
                                                _P]),
    "wrs_batched_autotune": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _SZ, _P, _P]),
    "wrs_batched_mixed_build_scratch_bytes": (_SZ, [_P, _P, _I64, _P]),
    "wrs_batched_mixed_build_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "wrs_batched_mixed_sample": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _I64, _P, _U64, _U64, _U64, _U32, _P, _P,
                                                _P]),
    "wrs_batched_autotune_kinds": (ctypes.c_int, [_P, _P, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _SZ,
                                                  _P, _P, _P, _P]),
    "wrs_scratch_status": (ctypes.c_int, [_P, _P]),
    "wrs_table_file_write": (ctypes.c_int, [ctypes.c_char_p, _P, _I64, ctypes.c_double, _P]),
    "wrs_batched_table_file_write": (ctypes.c_int, [ctypes.c_char_p, _P, _P, _I64, _P]),
    "wrs_table_file_info": (ctypes.c_int, [ctypes.c_char_p, _P, _P, _P]),
    "wrs_table_file_read": (ctypes.c_int, [ctypes.c_char_p, _P, _I64, _P, _I64, _P]),
    "wrs_shard_tables": (ctypes.c_int, [_P, _I64, ctypes.c_int32, _I64, _P]),
    "wrs_autotune_build": (ctypes.c_int, [_P, _I64, _P, _P, _SZ, _P, _P]),
    "wrs_autotune_sections": (ctypes.c_int, [_P, _I64, _U64, _P, _P, _P]),
    "wrs_autotune_lookup": (ctypes.c_int, [_I64, _P, _P]),
    "wrs_autotune_cache_save": (ctypes.c_int, [ctypes.c_char_p]),
    "wrs_autotune_cache_load": (ctypes.c_int, [ctypes.c_char_p]),
    "wrs_static_scratch_status": (ctypes.c_int, [_P]),
    "wrs_set_device_wait_limit": (ctypes.c_int, [_U64]),
    "wrs_debug_hold_lookback": (ctypes.c_int, [_I64]),
    "wrs_export_reference_table": (ctypes.c_int, [_P, _I64, ctypes.c_double, _P, _P, _P]),
    "wrs_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "wrs_check_device": (ctypes.c_int, []),
    "wrs_version": (ctypes.c_int, []),
}


def lib() -> ctypes.CDLL:
    """Loads libwrs.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libwrs.so not built at {LIB_PATH}; run `make -C {_HERE}`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(status: int) -> str:
    return lib().wrs_status_string(int(status)).decode()


def _check(status: int, what: str):
    if status != WRS_SUCCESS:
        raise WrsError(status, what)


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream(stream) -> Optional[int]:
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


# ---------------------------------------------------------------- C ABI wrappers

def build_opts(method: int = WRS_METHOD_SPLIT, tile_items: int = 0, sync: bool = False,
               small_table_items: int = 0, precision: int = 0) -> BuildOpts:
    return BuildOpts(method, tile_items, WRS_FLAG_SYNC if sync else 0, small_table_items, precision)


def alias_build_scratch_bytes(n: int, opts: Optional[BuildOpts] = None) -> int:
    return int(lib().wrs_alias_build_scratch_bytes(n, ctypes.byref(opts) if opts else None))


def alias_build(w, table, scratch, opts: Optional[BuildOpts] = None, W_out=None, stream=None) -> int:
    """Builds into `table` (torch int64/uint32 tensor of n rows, 8 bytes each) from FP32 `w`."""
    n = w.numel()
    st = lib().wrs_alias_build_f32(_ptr(w), n, ctypes.byref(opts) if opts else None, _ptr(table), _ptr(W_out),
                                   _ptr(scratch), scratch.numel() * scratch.element_size(), _stream(stream))
    return st


def alias_build_static_scratch(w, table, opts: Optional[BuildOpts] = None, W_out=None, stream=None) -> int:
    """Builds without any caller scratch (n <= 2^18): for callers that cannot allocate device
    memory; the scratch is a fixed array inside the library, shared by all calls on a device."""
    return lib().wrs_alias_build_f32_static_scratch(_ptr(w), w.numel(), ctypes.byref(opts) if opts else None,
                                                    _ptr(table), _ptr(W_out), _stream(stream))


def table_file_write(path: str, table, W: float, stream=None) -> int:
    return lib().wrs_table_file_write(path.encode(), _ptr(table), table.numel(), W, _stream(stream))


def batched_table_file_write(path: str, table, h_offsets, stream=None) -> int:
    import numpy as np
    off = np.ascontiguousarray(h_offsets, dtype=np.int64)
    return lib().wrs_batched_table_file_write(path.encode(), _ptr(table), off.ctypes.data, off.size - 1,
                                              _stream(stream))


def table_file_info(path: str):
    """(status, n, num_tables, W) of a table file."""
    n, t, W = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_double(0.0)
    st = lib().wrs_table_file_info(path.encode(), ctypes.byref(n), ctypes.byref(t), ctypes.byref(W))
    return st, n.value, t.value, W.value


def table_file_read(path: str, table, num_tables: int = 1, stream=None):
    """(status, offsets) after reading a table file's rows into `table`."""
    import numpy as np
    off = np.zeros(num_tables + 1, dtype=np.int64)
    st = lib().wrs_table_file_read(path.encode(), _ptr(table), table.numel(), off.ctypes.data, num_tables,
                                   _stream(stream))
    return st, off


def shard_tables(h_offsets, num_shards: int, table_cost: int = 16):
    """(status, bounds): contiguous table ranges [bounds[s], bounds[s+1]) per shard."""
    import numpy as np
    off = np.ascontiguousarray(h_offsets, dtype=np.int64)
    bounds = np.zeros(num_shards + 1, dtype=np.int64)
    st = lib().wrs_shard_tables(off.ctypes.data, off.size - 1, num_shards, table_cost, bounds.ctypes.data)
    return st, bounds


def autotune_build(w, table, scratch, opts: Optional[BuildOpts] = None, stream=None):
    """(status, opts) with opts.tile_items the fastest tile size for these weights."""
    opts = opts if opts is not None else build_opts()
    st = lib().wrs_autotune_build(_ptr(w), w.numel(), _ptr(table), _ptr(scratch),
                                  scratch.numel() * scratch.element_size(), ctypes.byref(opts), _stream(stream))
    return st, opts


def autotune_sections(table, n: int, num_samples: int, out, stream=None):
    """(status, section_items): the fastest section size for sectioned sampling of this table."""
    S = ctypes.c_uint32(0)
    st = lib().wrs_autotune_sections(_ptr(table), n, num_samples, _ptr(out), ctypes.byref(S), _stream(stream))
    return st, S.value


def autotune_lookup(n: int):
    """(status, tile_items, section_items) recorded for this GPU and ceil(log2 n)."""
    t, S = ctypes.c_uint32(0), ctypes.c_uint32(0)
    st = lib().wrs_autotune_lookup(n, ctypes.byref(t), ctypes.byref(S))
    return st, t.value, S.value


def autotune_cache_save(path: str) -> int:
    return lib().wrs_autotune_cache_save(path.encode())


def autotune_cache_load(path: str) -> int:
    return lib().wrs_autotune_cache_load(path.encode())


def set_device_wait_limit(limit_ns: int) -> int:
    """Limit of every bounded device wait of later launches (0 = the default, 2 s)."""
    return lib().wrs_set_device_wait_limit(limit_ns)


def debug_hold_lookback(block: int) -> int:
    """Failure-detection tests: look-back block `block` of later builds publishes nothing
    (-1 = off), so its successors' waits run out."""
    return lib().wrs_debug_hold_lookback(block)


def static_scratch_status(stream=None) -> int:
    """Device status of the last allocation-free build on the current device (synchronises
    `stream`); valid until the next such build on that device."""
    return lib().wrs_static_scratch_status(_stream(stream))


def alias_sample(table, n: int, num_samples: int, seed: int, out, counter_base: int = 0,
                 mode: int = WRS_SAMPLE_PLAIN, section_items: int = 0, section_counts=None,
                 sync: bool = False, stream=None) -> int:
    opts = SampleOpts(mode, section_items, WRS_FLAG_SYNC if sync else 0, 0)
    return lib().wrs_alias_sample(_ptr(table), n, num_samples, seed & (2**64 - 1), counter_base & (2**64 - 1),
                                  ctypes.byref(opts), _ptr(out), _ptr(section_counts), _stream(stream))


def random_gather_probe(table, n: int, num_gathers: int, seed: int, sink, stream=None) -> int:
    """num_gathers random 8-byte row gathers of the table, XOR-folded into sink[0] (a diagnostic
    of the random-access rate)."""
    return lib().wrs_random_gather_probe(_ptr(table), n, num_gathers, seed & (2**64 - 1), _ptr(sink),
                                         _stream(stream))


def alias_sample_to_host(table, n: int, num_samples: int, seed: int, out, host_out, counter_base: int = 0,
                         chunk_samples: int = 0, stream=None) -> int:
    """Plain samples into `host_out` (a pinned CPU tensor), produced chunk by chunk in `out`
    on the device while the copies of finished chunks run on the library's copy stream."""
    return lib().wrs_alias_sample_to_host(_ptr(table), n, num_samples, seed & (2**64 - 1), counter_base & (2**64 - 1),
                                          chunk_samples, _ptr(out), host_out.data_ptr(), _stream(stream))


def rejection_build_scratch_bytes(n: int) -> int:
    return int(lib().wrs_rejection_build_scratch_bytes(n))


def rejection_build(w, A, frac, a_size, scratch, W_out=None, sync: bool = False, stream=None) -> int:
    return lib().wrs_rejection_build_f32(_ptr(w), w.numel(), _ptr(A), A.numel(), _ptr(frac), _ptr(a_size),
                                         _ptr(W_out), _ptr(scratch), scratch.numel() * scratch.element_size(),
                                         WRS_FLAG_SYNC if sync else 0, _stream(stream))


def rejection_sample(A, a_size, frac, n: int, num_samples: int, seed: int, out, counter_base: int = 0,
                     max_tries: int = 0, status=None, sync: bool = False, stream=None) -> int:
    return lib().wrs_rejection_sample(_ptr(A), _ptr(a_size), _ptr(frac), n, num_samples, seed & (2**64 - 1),
                                      counter_base & (2**64 - 1), max_tries, _ptr(out), _ptr(status),
                                      WRS_FLAG_SYNC if sync else 0, _stream(stream))


def rejection_pack(A, a_size, frac, n: int, slots, stream=None) -> int:
    """Packs the slot array and the first slots' fractions into 8-byte slots (int64 tensor of at
    least |A| entries)."""
    return lib().wrs_rejection_pack(_ptr(A), _ptr(a_size), _ptr(frac), n, slots.numel(), _ptr(slots), _stream(stream))


def rejection_sample_packed(slots, a_size, n: int, num_samples: int, seed: int, out, counter_base: int = 0,
                            max_tries: int = 0, status=None, sync: bool = False, stream=None) -> int:
    return lib().wrs_rejection_sample_packed(_ptr(slots), slots.numel(), _ptr(a_size), n, num_samples, seed & (2**64 - 1),
                                             counter_base & (2**64 - 1), max_tries, _ptr(out), _ptr(status),
                                             WRS_FLAG_SYNC if sync else 0, _stream(stream))


def scratch_status(scratch, stream=None) -> int:
    return lib().wrs_scratch_status(_ptr(scratch), _stream(stream))


def _host_i64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


def batched_build_scratch_bytes(h_offsets, opts: Optional[BuildOpts] = None) -> int:
    """Scratch of a batched build (opts None: enough for every launch shape)."""
    h = _host_i64(h_offsets)
    return lib().wrs_batched_build_scratch_bytes(h.ctypes.data, h.shape[0] - 1, ctypes.byref(opts) if opts else None)


def batched_build(w, d_offsets, h_offsets, table, scratch, opts: Optional[BuildOpts] = None, W_out=None,
                  stream=None) -> int:
    """Builds every CSR table of `w` (table t owns w[off[t]:off[t+1]]) into `table` (same rows)."""
    h = _host_i64(h_offsets)
    return lib().wrs_batched_build_f32(_ptr(w), _ptr(d_offsets), h.ctypes.data, h.shape[0] - 1,
                                       ctypes.byref(opts) if opts else None, _ptr(table), _ptr(W_out),
                                       _ptr(scratch), scratch.numel() * scratch.element_size(), _stream(stream))


def batched_sample(table, d_offsets, num_tables: int, d_sample_offsets, total: int, seed: int, out,
                   counter_base: int = 0, stream=None) -> int:
    return lib().wrs_batched_sample(_ptr(table), _ptr(d_offsets), num_tables, _ptr(d_sample_offsets), total,
                                    seed & (2**64 - 1), counter_base & (2**64 - 1), _ptr(out), _stream(stream))


def batched_build_sample_scratch_bytes(h_offsets, opts: Optional[BuildOpts] = None) -> int:
    """Scratch of wrs_batched_build_sample (opts None: enough for every launch shape)."""
    h = _host_i64(h_offsets)
    return lib().wrs_batched_build_sample_scratch_bytes(h.ctypes.data, h.shape[0] - 1,
                                                        ctypes.byref(opts) if opts else None)


def batched_build_sample(w, d_offsets, h_offsets, table, d_sample_offsets, total: int, seed: int, out, scratch,
                         opts: Optional[BuildOpts] = None, counter_base: int = 0, W_out=None, stream=None) -> int:
    """batched_build followed by batched_sample in one call: each size class's samples are drawn
    as soon as it is built, while the larger tables are still being built."""
    h = _host_i64(h_offsets)
    return lib().wrs_batched_build_sample(_ptr(w), _ptr(d_offsets), h.ctypes.data, h.shape[0] - 1,
                                          ctypes.byref(opts) if opts else None, _ptr(table), _ptr(W_out),
                                          _ptr(d_sample_offsets), total, seed & (2**64 - 1),
                                          counter_base & (2**64 - 1), _ptr(out), _ptr(scratch),
                                          scratch.numel() * scratch.element_size(), _stream(stream))


def batched_per_table(w, h_offsets, h_sample_offsets, tables, table, seed: int, out, scratch,
                      opts: Optional[BuildOpts] = None, counter_base: int = 0, stream=None) -> int:
    """The one-table-per-launch form of a batch (a native loop of single-table build and
    sample calls over the table ids `tables`), for comparison with the batched calls."""
    h = _host_i64(h_offsets)
    hs = _host_i64(h_sample_offsets)
    ids = _host_i64(tables)
    return lib().wrs_batched_per_table(_ptr(w), h.ctypes.data, hs.ctypes.data, ids.ctypes.data, ids.size,
                                       ctypes.byref(opts) if opts else None, _ptr(table), seed & (2**64 - 1),
                                       counter_base & (2**64 - 1), _ptr(out), _ptr(scratch),
                                       scratch.numel() * scratch.element_size(), _stream(stream))


def batched_autotune_build_sample(w, d_offsets, h_offsets, table, d_sample_offsets, total: int, out, scratch,
                                  opts: BuildOpts, stream=None) -> int:
    """Times every launch shape of batched_build_sample on this batch and stores the fastest in `opts`."""
    h = _host_i64(h_offsets)
    return lib().wrs_batched_autotune_build_sample(_ptr(w), _ptr(d_offsets), h.ctypes.data, h.shape[0] - 1,
                                                   _ptr(table), _ptr(d_sample_offsets), total, _ptr(out),
                                                   _ptr(scratch), scratch.numel() * scratch.element_size(),
                                                   ctypes.byref(opts), _stream(stream))


def batched_autotune(w, d_offsets, h_offsets, table, scratch, opts: BuildOpts, stream=None) -> int:
    """Times every batched launch shape on this batch and stores the fastest in `opts`."""
    h = _host_i64(h_offsets)
    return lib().wrs_batched_autotune(_ptr(w), _ptr(d_offsets), h.ctypes.data, h.shape[0] - 1, _ptr(table),
                                      _ptr(scratch), scratch.numel() * scratch.element_size(), ctypes.byref(opts),
                                      _stream(stream))


WRS_TABLE_ALIAS = 0
WRS_TABLE_REJECTION = 1
WRS_TABLE_SKIP = 2


def _host_u8(a) -> Optional[np.ndarray]:
    return None if a is None else np.ascontiguousarray(np.asarray(a, dtype=np.uint8))


def batched_mixed_build_scratch_bytes(h_offsets, h_kinds=None, opts: Optional[BuildOpts] = None) -> int:
    """Scratch of a mixed build (h_kinds None: enough for any kinds)."""
    h = _host_i64(h_offsets)
    k = _host_u8(h_kinds)
    return lib().wrs_batched_mixed_build_scratch_bytes(h.ctypes.data, None if k is None else k.ctypes.data,
                                                       h.shape[0] - 1, ctypes.byref(opts) if opts else None)


def batched_mixed_build(w, d_offsets, h_offsets, d_kinds, h_kinds, table, A, frac, a_size, scratch,
                        opts: Optional[BuildOpts] = None, W_out=None, stream=None) -> int:
    """Builds each table by its kind: alias rows into `table`, rejection slots into `A`
    (table t at A[2 off[t]:]), acceptances into `frac`, |A_t| into `a_size`."""
    h = _host_i64(h_offsets)
    k = _host_u8(h_kinds)
    return lib().wrs_batched_mixed_build_f32(_ptr(w), _ptr(d_offsets), h.ctypes.data, _ptr(d_kinds),
                                             None if k is None else k.ctypes.data, h.shape[0] - 1,
                                             ctypes.byref(opts) if opts else None, _ptr(table), _ptr(A), _ptr(frac),
                                             _ptr(a_size), _ptr(W_out), _ptr(scratch),
                                             scratch.numel() * scratch.element_size(), _stream(stream))


def batched_mixed_sample(table, A, frac, a_size, d_offsets, d_kinds, num_tables: int, d_sample_offsets, total: int,
                         seed: int, out, counter_base: int = 0, max_tries: int = 0, status=None, stream=None) -> int:
    return lib().wrs_batched_mixed_sample(_ptr(table), _ptr(A), _ptr(frac), _ptr(a_size), _ptr(d_offsets),
                                          _ptr(d_kinds), num_tables, _ptr(d_sample_offsets), total,
                                          seed & (2**64 - 1), counter_base & (2**64 - 1), max_tries, _ptr(out),
                                          _ptr(status), _stream(stream))


def batched_autotune_kinds(w, d_offsets, h_offsets, d_sample_offsets, h_sample_offsets, table, A, frac, a_size,
                           d_kinds_tmp, out, scratch, opts: Optional[BuildOpts] = None, stream=None):
    """Alias or rejection per size class (ceil(log2 n)), timed on this batch. Returns
    (status, kinds per table, kinds per class, ms per class as (alias, rejection) pairs)."""
    h = _host_i64(h_offsets)
    hs = _host_i64(h_sample_offsets)
    kinds = np.zeros(h.shape[0] - 1, dtype=np.uint8)
    cls = np.zeros(33, dtype=np.uint8)
    ms = np.zeros((33, 2), dtype=np.float32)
    st = lib().wrs_batched_autotune_kinds(_ptr(w), _ptr(d_offsets), h.ctypes.data, h.shape[0] - 1,
                                          _ptr(d_sample_offsets), hs.ctypes.data, ctypes.byref(opts) if opts else None,
                                          _ptr(table), _ptr(A), _ptr(frac), _ptr(a_size), _ptr(d_kinds_tmp), _ptr(out),
                                          _ptr(scratch), scratch.numel() * scratch.element_size(),
                                          kinds.ctypes.data, cls.ctypes.data, ms.ctypes.data, _stream(stream))
    return st, kinds, cls, ms


def export_reference_table(table, W: float, weight, alias, stream=None) -> int:
    """The table in the reference's format: FP64 absolute weights (prob * W/n) and int aliases."""
    return lib().wrs_export_reference_table(_ptr(table), table.numel(), W, _ptr(weight), _ptr(alias),
                                            _stream(stream))


def sum_f32(w, total, scratch, stream=None) -> int:
    return lib().wrs_sum_f32(_ptr(w), w.numel(), _ptr(total), _ptr(scratch),
                             scratch.numel() * scratch.element_size(), _stream(stream))


# ---------------------------------------------------------------- reference-shaped surface

def _device_bytes(nbytes: int, device):
    import torch
    return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=device)


class SamplingAlgorithm:
    """build(weights) surface of construction/SamplingAlgorithm.cuh:30-48.

    ``weights`` is a host array of N FP32 weights; ``W`` and ``N`` as in the reference.
    """

    def __init__(self, weights, device: str = "cuda"):
        self.weights = np.ascontiguousarray(np.asarray(weights, dtype=np.float32))
        self.N = int(self.weights.shape[0])
        self.W = 0.0
        self.device = device

    def name(self) -> str:
        raise NotImplementedError

    def preBuild(self):
        raise NotImplementedError

    def build(self):
        raise NotImplementedError

    def postBuild(self) -> bool:
        raise NotImplementedError

    def fullBuild(self) -> bool:
        self.preBuild()
        self.build()
        return self.postBuild()


class AliasTableSplitGpu(SamplingAlgorithm):
    """AliasTableSplitGpu (construction/aliasTable/buildMethod/AliasTableSplitGpu.cu).

    After postBuild(), ``aliasTable`` holds the host table as (prob float32, alias uint32)
    arrays; ``table`` is the device table (int64 tensor, one packed row per item).
    """

    def __init__(self, weights, method: int = WRS_METHOD_SPLIT, tile_items: int = 0, device: str = "cuda"):
        super().__init__(weights, device)
        self.method = method
        self.opts = build_opts(method, tile_items)
        self.table = None
        self.aliasTable = None

    def name(self) -> str:
        return "AliasTableSplitGpu" + ("PsaPlus" if self.method == WRS_METHOD_PSA_PLUS else "")

    def preBuild(self):
        import torch
        self.weightsGpu = torch.from_numpy(self.weights).to(self.device)
        self.table = torch.empty(self.N, dtype=torch.int64, device=self.device)
        self.scratch = _device_bytes(alias_build_scratch_bytes(self.N, self.opts), self.device)
        self.W_dev = torch.zeros(1, dtype=torch.float64, device=self.device)

    def build(self):
        _check(alias_build(self.weightsGpu, self.table, self.scratch, self.opts, self.W_dev), "alias build")

    def postBuild(self) -> bool:
        st = scratch_status(self.scratch)
        _check(st, "alias build (device)")
        self.W = float(self.W_dev.item())
        rows = self.table.cpu().numpy().view(np.uint32).reshape(-1, 2)
        self.aliasTable = (rows[:, 0].view(np.float32).copy(), rows[:, 1].copy())
        return True


class RejectionSamplingGpu(SamplingAlgorithm):
    """RejectionSampling (construction/rejectionSampling/RejectionSampling.cu)."""

    def __init__(self, weights, device: str = "cuda"):
        super().__init__(weights, device)

    def name(self) -> str:
        return "RejectionSamplingGpu"

    def preBuild(self):
        import torch
        self.weightsGpu = torch.from_numpy(self.weights).to(self.device)
        self.A = torch.empty(2 * self.N + 1, dtype=torch.int32, device=self.device)
        self.frac = torch.empty(self.N, dtype=torch.float32, device=self.device)
        self.A_size = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.scratch = _device_bytes(rejection_build_scratch_bytes(self.N), self.device)
        self.W_dev = torch.zeros(1, dtype=torch.float64, device=self.device)

    def build(self):
        _check(rejection_build(self.weightsGpu, self.A, self.frac, self.A_size, self.scratch, self.W_dev),
               "rejection build")

    def postBuild(self) -> bool:
        import torch
        _check(scratch_status(self.scratch), "rejection build (device)")
        self.W = float(self.W_dev.item())
        # the slots packed with the first slots' fractions: one gather per try when sampling
        self.slots = torch.empty(max(1, int(self.A_size.item())), dtype=torch.int64, device=self.device)
        _check(rejection_pack(self.A, self.A_size, self.frac, self.N, self.slots), "rejection pack")
        return True


class Sampler:
    """sampling/Sampler.cuh:10-31: name(), benchmarkSampling(n) in Gsamples/s,
    getSamplingDistribution(n) -> per-item counts; plus sample(n) -> device tensor."""

    def __init__(self, algorithm: SamplingAlgorithm, seed: int = 0x5EED):
        self.algorithm = algorithm
        self.seed = seed
        self.counter = 0

    def name(self) -> str:
        raise NotImplementedError

    def sample(self, numSamples: int, out=None):
        raise NotImplementedError

    def benchmarkSampling(self, numSamples: int) -> float:
        import torch
        out = torch.empty(numSamples, dtype=torch.int32, device=self.algorithm.device)
        self.sample(numSamples, out)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        self.sample(numSamples, out)
        stop.record()
        stop.synchronize()
        return numSamples / (start.elapsed_time(stop) * 1e6)

    def getSamplingDistribution(self, numSamples: int) -> np.ndarray:
        import torch
        out = self.sample(numSamples)
        return torch.bincount(out.long(), minlength=self.algorithm.N).cpu().numpy()


def alias_histogram(table, n: int, num_samples: int, seed: int, counts, counter_base: int = 0, stream=None) -> int:
    """Adds the plain samples' per-row counts to `counts` (n int32 on the device)."""
    return alias_sample(table, n, num_samples, seed, counts, counter_base, mode=WRS_SAMPLE_HISTOGRAM, stream=stream)


class SamplerGpuBasic(Sampler):
    def name(self) -> str:
        return "SamplerGpuBasic"

    def sample(self, numSamples: int, out=None):
        import torch
        a = self.algorithm
        if out is None:
            out = torch.empty(numSamples, dtype=torch.int32, device=a.device)
        _check(alias_sample(a.table, a.N, numSamples, self.seed, out, self.counter), "plain sample")
        self.counter += numSamples
        return out

    def getSamplingDistribution(self, numSamples: int) -> np.ndarray:
        """Per-item counts of numSamples plain samples, counted on the device (no sample list)."""
        import torch
        a = self.algorithm
        counts = torch.zeros(a.N, dtype=torch.int32, device=a.device)
        _check(alias_histogram(a.table, a.N, numSamples, self.seed, counts, self.counter), "plain histogram")
        self.counter += numSamples
        return counts.cpu().numpy().astype(np.int64)


class SamplerGpuSectioned(Sampler):
    def __init__(self, algorithm: SamplingAlgorithm, itemsPerSection: int = 0, seed: int = 0x5EED):
        super().__init__(algorithm, seed)
        self.itemsPerSection = itemsPerSection

    def name(self) -> str:
        return "SamplerGpuSectioned"

    def sample(self, numSamples: int, out=None):
        import torch
        a = self.algorithm
        if out is None:
            out = torch.empty(numSamples, dtype=torch.int32, device=a.device)
        _check(alias_sample(a.table, a.N, numSamples, self.seed, out, self.counter, mode=WRS_SAMPLE_SECTIONED,
                            section_items=self.itemsPerSection), "sectioned sample")
        self.counter += numSamples
        return out


class SamplerGpuSectionedShared(SamplerGpuSectioned):
    """SamplerGpuSectionedShared (sampling/aliasTable/SamplerGpuSectionedShared.cu:3-111): every
    section staged in shared memory. alias_sample stages sections of at most 12,288 rows (96 KiB),
    so this is the sectioned sampler with the reference's default of 3000 rows per section; a
    section too large to stage raises, as the reference asserts."""
    MAX_STAGED_ROWS = 12288

    def __init__(self, algorithm: SamplingAlgorithm, itemsPerSection: int = 3000, seed: int = 0x5EED):
        if not (2 <= itemsPerSection <= self.MAX_STAGED_ROWS) or itemsPerSection % 2:
            raise WrsError(WRS_ERR_INVALID_ARGUMENT, "SamplerGpuSectionedShared: itemsPerSection must be even, "
                                                     "in [2, 12288]")
        super().__init__(algorithm, itemsPerSection, seed)

    def name(self) -> str:
        return "SamplerGpuSectionedShared"


class SamplerRejection(Sampler):
    def __init__(self, algorithm: RejectionSamplingGpu, seed: int = 0x5EED, max_tries: int = 0):
        super().__init__(algorithm, seed)
        self.max_tries = max_tries

    def name(self) -> str:
        return "SamplerRejection"

    def sample(self, numSamples: int, out=None):
        import torch
        a = self.algorithm
        if out is None:
            out = torch.empty(numSamples, dtype=torch.int32, device=a.device)
        _check(rejection_sample_packed(a.slots, a.A_size, a.N, numSamples, self.seed, out, self.counter,
                                       self.max_tries), "rejection sample")
        self.counter += numSamples
        return out


class SamplerRejectionGiveUp(SamplerRejection):
    """SamplerRejectionGiveUp (sampling/rejectionSampling/SamplerRejectionGiveUp.cu:17-37, MAX_TRIES 8):
    at most 8 tries per sample; a sample that runs out of tries is written as 0xFFFFFFFF."""

    def __init__(self, algorithm: RejectionSamplingGpu, seed: int = 0x5EED):
        super().__init__(algorithm, seed, max_tries=8)

    def name(self) -> str:
        return "SamplerRejectionGiveUp"


class BatchedAliasTablesGpu:
    """Many alias tables built at once from CSR weights (the batched form of
    AliasTableSplitGpu; the reference builds such batches one object per table).

    ``offsets`` (int64, num_tables + 1) delimits the tables in ``weights``; after
    fullBuild() ``table`` holds every table's rows at its items' positions (table-local
    aliases) and ``W`` the per-table weight totals.
    """

    def __init__(self, weights, offsets, device: str = "cuda", opts: Optional[BuildOpts] = None):
        self.weights = np.ascontiguousarray(np.asarray(weights, dtype=np.float32))
        self.offsets = _host_i64(offsets)
        self.num_tables = int(self.offsets.shape[0] - 1)
        self.device = device
        self.opts = opts if opts is not None else build_opts()
        self.table = None

    def name(self) -> str:
        return "BatchedAliasTablesGpu"

    def preBuild(self):
        import torch
        self.weightsGpu = torch.from_numpy(self.weights).to(self.device)
        self.offsetsGpu = torch.from_numpy(self.offsets).to(self.device)
        self.table = torch.empty(max(1, self.weights.shape[0]), dtype=torch.int64, device=self.device)
        self.scratch = _device_bytes(batched_build_scratch_bytes(self.offsets), self.device)
        self.W_dev = torch.zeros(self.num_tables, dtype=torch.float64, device=self.device)

    def autotune(self):
        _check(batched_autotune(self.weightsGpu, self.offsetsGpu, self.offsets, self.table, self.scratch, self.opts),
               "batched autotune")

    def build(self):
        _check(batched_build(self.weightsGpu, self.offsetsGpu, self.offsets, self.table, self.scratch, self.opts,
                             self.W_dev), "batched build")

    def postBuild(self) -> bool:
        _check(scratch_status(self.scratch), "batched build (device)")
        self.W = self.W_dev.cpu().numpy()
        return True

    def fullBuild(self) -> bool:
        self.preBuild()
        self.build()
        return self.postBuild()


class SamplerBatched:
    """Per-table sample counts over a BatchedAliasTablesGpu: sample(counts) returns the
    table-local indices (table t's at [sample_offsets[t], sample_offsets[t+1])) and the
    sample offsets."""

    def __init__(self, tables: BatchedAliasTablesGpu, seed: int = 0x5EED):
        self.tables = tables
        self.seed = seed
        self.counter = 0

    def name(self) -> str:
        return "SamplerBatched"

    def sample(self, counts, out=None):
        import torch
        t = self.tables
        soff = np.zeros(t.num_tables + 1, dtype=np.int64)
        np.cumsum(np.asarray(counts, dtype=np.int64), out=soff[1:])
        total = int(soff[-1])
        d_soff = torch.from_numpy(soff).to(t.device)
        if out is None:
            out = torch.empty(max(1, total), dtype=torch.int32, device=t.device)
        _check(batched_sample(t.table, t.offsetsGpu, t.num_tables, d_soff, total, self.seed, out, self.counter),
               "batched sample")
        self.counter += total
        return out[:total], soff
