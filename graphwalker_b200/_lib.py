"""ctypes binding of the C ABI declared in include/graphwalker_b200.h.

The shared library is built in-tree (graphwalker_b200/lib/libgw_b200.so, see
graphwalker_b200/build.py).  There is no fallback: if the library is missing
the import fails loudly.
"""
from __future__ import annotations

import ctypes
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int32, c_size_t, c_uint32,
                    c_uint64, c_void_p)
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libgw_b200.so"
HEADER_PATH = Path(__file__).resolve().parent.parent / "include" / "graphwalker_b200.h"

GW_OK = 0
GW_E_INVALID, GW_E_CUDA, GW_E_NOMEM, GW_E_IO = 1, 2, 3, 4
GW_E_BOUNDS, GW_E_OVERFLOW, GW_E_STATE, GW_E_TIMEOUT = 5, 6, 7, 8

RULE_JUMP, RULE_STOP, RULE_PROB, RULE_RESTART, RULE_PPR = 0, 1, 2, 3, 4
SINK_NONE, SINK_VERTEX_COUNT, SINK_PATH_RECORD, SINK_CLOSURE_COUNT = 0, 1, 2, 3
MODE_RESIDENT, MODE_BLOCKED = 0, 1
RNG_PHILOX, RNG_NATIVE = 0, 1
RESIDENT_HBM, STREAM_PINNED = 0, 1
MAPPED_AUTO = (1 << 64) - 1  # gw_set_mapped_block_walks: per block, one walk per 128 CSR bytes


class WalkRec(Structure):
    _fields_ = [("cur", c_uint32), ("id", c_uint32), ("src", c_uint32), ("hop", c_uint32)]


class WalkParams(Structure):
    _fields_ = [("rule", c_uint32), ("sink", c_uint32), ("L", c_uint32), ("njump", c_uint32),
                ("jump_prob", c_double), ("seed", c_uint64), ("mode", c_uint32),
                ("path_stride", c_uint32), ("max_hops", c_uint32), ("prob", c_float),
                ("aggregate", c_uint32), ("max_supersteps", c_uint32), ("cache_hints", c_uint32),
                ("table_factor", c_uint32), ("block_lo", c_uint32), ("block_hi", c_uint32),
                ("rng", c_uint32), ("reserved", c_uint32)]


SERVE_BATCHED, SERVE_PLAIN = 0, 1
EDGE_RECORDS_OFF, EDGE_RECORDS_ON, EDGE_RECORDS_AUTO = 0, 1, 2
FAULT_NONE, FAULT_DEVICE_ALLOC, FAULT_PINNED_ALLOC, FAULT_FILE_READ = 0, 1, 2, 3


class ServeConfig(Structure):
    _fields_ = [("table_slots", c_uint64), ("max_walks_per_step", c_uint32), ("quantum", c_uint32),
                ("k", c_uint32), ("mode", c_uint32), ("reserved", c_uint32 * 4)]


class ServeTiming(Structure):
    _fields_ = [("arrival_ns", c_uint64), ("admit_ns", c_uint64), ("done_ns", c_uint64), ("restarts", c_uint32),
                ("reserved", c_uint32)]


class ServeStats(Structure):
    _fields_ = [("submitted", c_uint64), ("completed", c_uint64), ("supersteps", c_uint64), ("walks", c_uint64),
                ("restarts", c_uint64), ("pending", c_uint64), ("active", c_uint64)]


class ConvertStats(Structure):
    _fields_ = [("bytes", c_uint64), ("lines", c_uint64), ("edges", c_uint64), ("nvertices", c_uint32),
                ("nblocks", c_uint32), ("sorted", c_uint32), ("reserved0", c_uint32), ("ms_read", c_double),
                ("ms_device", c_double), ("ms_write", c_double), ("ms_total", c_double),
                ("reserved", c_uint64 * 4)]


class PprStats(Structure):
    _fields_ = [("walks", c_uint64), ("table_slots", c_uint64), ("launches", c_uint32), ("reserved", c_uint32),
                ("ms_clear", c_double), ("ms_walk", c_double), ("ms_topk", c_double), ("ms_total", c_double),
                ("visits", c_uint64)]


HINT_EXPLICIT = 0x80000000
HINT_COLUMNS_EVICT_FIRST, HINT_COUNTS_EVICT_LAST, HINT_RECORDS_EVICT_LAST = 1, 2, 4
HINT_STREAMS_EVICT_FIRST = 8


class RunStats(Structure):
    _fields_ = [("walks", c_uint64), ("supersteps", c_uint64), ("block_loads", c_uint64),
                ("bytes_h2d", c_uint64), ("ms_total", c_double), ("ms_walk", c_double),
                ("ms_partition", c_double), ("ms_copy_wait", c_double), ("mapped_supersteps", c_uint64),
                ("mapped_walks", c_uint64), ("pools_spilled", c_uint64), ("pools_refilled", c_uint64)]


class GraphDesc(Structure):
    _fields_ = [("base_filename", c_char_p), ("blocksize_kb", c_uint64), ("nmblocks", c_uint32),
                ("residency", c_uint32), ("device", c_int32)]


class GwError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gw status {code}: {msg}")
        self.code = code


_P = c_void_p
_SIGS = {
    "gw_version": (c_char_p, []),
    "gw_encode": (c_uint64, [c_uint32, c_uint32, c_uint32]),
    "gw_get_source": (c_uint32, [c_uint64]),
    "gw_get_current": (c_uint32, [c_uint64]),
    "gw_get_hop": (c_uint32, [c_uint64]),
    "gw_continue_threshold": (c_uint32, [c_double]),
    "gw_getblock": (c_uint32, [_P, c_uint32, c_uint32]),
    "gw_compute_blocks": (c_uint32, [_P, c_uint32, c_uint64, _P, c_uint32]),
    "gw_comp_block_size": (c_uint64, [c_uint64]),
    "gw_comp_nmblocks": (c_uint32, [c_uint64, c_uint64]),
    "gw_open": (c_int32, [POINTER(GraphDesc), POINTER(c_void_p)]),
    "gw_open_csr": (c_int32, [_P, _P, c_uint32, _P, c_uint32, c_uint32, c_int32, POINTER(c_void_p)]),
    "gw_open_rmat": (c_int32, [c_uint32, c_uint32, c_uint64, c_double, c_double, c_double, c_uint64,
                               c_int32, POINTER(c_void_p)]),
    "gw_close": (c_int32, [_P]),
    "gw_last_error": (c_char_p, [_P]),
    "gw_graph_info": (c_int32, [_P, POINTER(c_uint32), POINTER(c_uint64), POINTER(c_uint32)]),
    "gw_get_blocks": (c_int32, [_P, _P, c_uint32]),
    "gw_export_csr": (c_int32, [_P, _P, _P]),
    "gw_set_residency": (c_int32, [_P, c_uint32, c_uint32]),
    "gw_set_mapped_block_walks": (c_int32, [_P, c_uint64]),
    "gw_set_pool_budget": (c_int32, [_P, c_uint64]),
    "gw_walks_clear": (c_int32, [_P]),
    "gw_walks_add": (c_int32, [_P, c_uint32, _P, _P, c_size_t]),
    "gw_walks_count": (c_int32, [_P, _P, POINTER(c_uint64)]),
    "gw_run": (c_int32, [_P, POINTER(WalkParams)]),
    "gw_read_counts": (c_int32, [_P, _P, c_size_t]),
    "gw_read_paths": (c_int32, [_P, _P, _P, c_size_t]),
    "gw_read_closure": (c_int32, [_P, POINTER(c_uint64)]),
    "gw_read_stats": (c_int32, [_P, POINTER(RunStats)]),
    "gw_read_pool": (c_int32, [_P, c_uint32, _P, c_size_t, POINTER(c_uint64)]),
    "gw_run_pools": (c_int32, [_P, POINTER(WalkParams), _P, _P, _P, _P]),
    "gw_run_pools_submit": (c_int32, [_P, POINTER(WalkParams), _P, _P, _P, _P, POINTER(c_uint64)]),
    "gw_run_pools_wait": (c_int32, [_P, c_uint64]),
    "gw_walk_device": (c_int32, [_P, POINTER(WalkParams), _P, c_uint64, _P, _P, _P, _P, _P]),
    "gw_unpack_words_device": (c_int32, [_P, c_uint32, _P, _P, c_uint64, _P, _P]),
    "gw_pack_words_device": (c_int32, [_P, _P, c_uint64, _P, _P, _P]),
    "gw_sync": (c_int32, [_P, _P]),
    "gw_probe_gather": (c_int32, [_P, _P, c_uint64, c_uint64, ctypes.c_int, POINTER(c_double)]),
    "gw_probe_red": (c_int32, [_P, _P, c_uint64, c_uint64, ctypes.c_int, POINTER(c_double)]),
    "gw_superstep_static": (c_int32, [_P, POINTER(WalkParams), c_uint32, _P, c_uint64, _P, _P, _P, _P, _P]),
    "gw_ppr_run": (c_int32, [_P, POINTER(WalkParams), _P, _P, c_uint32, c_uint32, c_uint32, _P, _P,
                             POINTER(PprStats)]),
    "gw_ppr_autotune": (c_int32, [_P, POINTER(WalkParams), _P, _P, c_uint32, POINTER(c_uint32),
                                  POINTER(c_uint32)]),
    "gw_expected_visits": (c_int32, [_P, POINTER(WalkParams), c_uint32, _P]),
    "gw_serve_open": (c_int32, [_P, POINTER(WalkParams), POINTER(ServeConfig), POINTER(c_void_p)]),
    "gw_serve_submit": (c_int32, [_P, c_uint32, c_uint32, c_uint32, c_uint64, POINTER(c_uint64)]),
    "gw_serve_wait": (c_int32, [_P, c_uint64, ctypes.c_int64, _P, _P, POINTER(ServeTiming)]),
    "gw_serve_get_stats": (c_int32, [_P, POINTER(ServeStats)]),
    "gw_serve_clock_ns": (c_uint64, []),
    "gw_serve_close": (c_int32, [_P]),
    "gw_set_l2_fetch_granularity": (c_int32, [_P, c_uint32, POINTER(c_uint32)]),
    "gw_set_l2_persisting": (c_int32, [_P, c_uint64]),
    "gw_set_edge_records": (c_int32, [_P, c_uint32, POINTER(c_uint32)]),
    "gw_simrank_meet": (c_int32, [_P, _P, _P, c_uint32, c_uint32, _P, _P]),
    "gw_simrank_batch": (c_int32, [_P, POINTER(WalkParams), _P, _P, c_uint32, c_uint32, c_double, _P, _P]),
    "gw_convert_edgelist": (c_int32, [c_char_p, c_uint64, c_int32, POINTER(ConvertStats)]),
    "gw_inject_fault": (c_int32, [c_uint32, c_uint32]),
    "gw_walk_autotune": (c_int32, [_P, POINTER(WalkParams), _P, c_uint64, POINTER(c_uint32)]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Loads libgw_b200.so and declares every entry point; raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m graphwalker_b200.build` "
            "(the engine has no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, ctx=None) -> None:
    if status != GW_OK:
        msg = load().gw_last_error(ctx)
        raise GwError(status, msg.decode() if msg else "")


def exported_symbols() -> list[str]:
    return list(_SIGS)
