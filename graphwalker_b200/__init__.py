"""graphwalker_b200 -- a B200 (sm_100a) engine for GraphWalker's random-walk hot path.

The product is the CUDA library graphwalker_b200/lib/libgw_b200.so behind the
C ABI in include/graphwalker_b200.h; this package is its Python handle.
The first call into the engine loads the library and raises ImportError when
it is missing (build it with `python -m graphwalker_b200.build`); there is no
CPU fallback.
"""
from ._lib import (EDGE_RECORDS_AUTO, EDGE_RECORDS_OFF, EDGE_RECORDS_ON, FAULT_DEVICE_ALLOC, FAULT_FILE_READ,
                   FAULT_NONE, FAULT_PINNED_ALLOC, MAPPED_AUTO, MODE_BLOCKED, MODE_RESIDENT,
                   RESIDENT_HBM, RNG_NATIVE, RNG_PHILOX, RULE_JUMP, RULE_PPR, RULE_PROB,
                   RULE_RESTART, RULE_STOP, SINK_CLOSURE_COUNT, SINK_NONE, SINK_PATH_RECORD,
                   SINK_VERTEX_COUNT, STREAM_PINNED, GwError, WalkParams, WalkRec, load)
from .engine import (Graph, compute_blocks, convert_edgelist, encode, get_current, get_hop, get_source,
                     inject_fault, params, simrank_estimate)

__all__ = [
    "Graph", "GwError", "WalkParams", "WalkRec", "params", "encode", "get_source", "get_current",
    "get_hop", "compute_blocks", "load", "RULE_JUMP", "RULE_STOP", "RULE_PROB", "RULE_RESTART",
    "RULE_PPR", "SINK_NONE", "SINK_VERTEX_COUNT", "SINK_PATH_RECORD", "SINK_CLOSURE_COUNT",
    "MODE_RESIDENT", "MODE_BLOCKED", "RNG_PHILOX", "RNG_NATIVE", "RESIDENT_HBM", "STREAM_PINNED", "MAPPED_AUTO",
    "EDGE_RECORDS_OFF",
    "EDGE_RECORDS_ON", "EDGE_RECORDS_AUTO", "simrank_estimate", "convert_edgelist", "inject_fault",
    "FAULT_NONE", "FAULT_DEVICE_ALLOC", "FAULT_PINNED_ALLOC", "FAULT_FILE_READ",
]
