"""Host-side Python handle over the C ABI (used by the tests and bench.py).

`Graph` owns one engine context: a CSR resident in HBM (or held in pinned
host memory and streamed block by block), GraphWalker-style walk pools, and
the run/readback calls.  Host arrays are numpy; device arrays are any object
with a `data_ptr()` (torch tensors) or raw integer pointers.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_double, c_uint32, c_uint64, c_void_p

import numpy as np

from . import _lib
from ._lib import (MODE_BLOCKED, MODE_RESIDENT, RESIDENT_HBM, RULE_JUMP, SINK_VERTEX_COUNT,
                   STREAM_PINNED, GraphDesc, RunStats, WalkParams, check, load)


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
        return a.ctypes.data
    raise TypeError(f"cannot take a pointer of {type(a)}")


def convert_edgelist(path: str, blocksize_kb: int = 0, device: int = 0) -> _lib.ConvertStats:
    """Text edge list -> the reference's preprocessed files, on the device
    (gw_convert_edgelist; convert_if_notexists, conversions.hpp:181-404)."""
    st = _lib.ConvertStats()
    check(load().gw_convert_edgelist(str(path).encode(), blocksize_kb, device, byref(st)))
    return st


def inject_fault(kind: int, after: int = 0) -> None:
    """Makes the after-th next host-side operation of `kind` fail once
    (gw_inject_fault; FAULT_NONE disarms)."""
    check(load().gw_inject_fault(kind, after))


def simrank_estimate(meet, R: int, decay: float = 0.8) -> float:
    """SimRank estimate from first-meeting counts: sum_l meet[l] * decay^l / R^2
    (the quantity SimRank::computeResult sums, apps/simrank.cpp:71-84)."""
    return float(sum(int(m) * decay ** l for l, m in enumerate(meet)) / (float(R) * float(R)))


def params(rule: int = RULE_JUMP, sink: int = SINK_VERTEX_COUNT, L: int = 10, *, njump: int = 0,
           jump_prob: float = 0.15, seed: int = 42, mode: int = MODE_RESIDENT, path_stride: int = 0,
           max_hops: int = 0, prob: float = 0.2, aggregate: bool = False,
           max_supersteps: int = 0, cache_hints: int | None = None, block_lo: int = 0,
           block_hi: int = 0, rng: int = _lib.RNG_PHILOX) -> WalkParams:
    """gw_walk_params with the reference's defaults (0.15 else-branch, prob 0.2).
    cache_hints: None = engine default, else GW_HINT_* bits used as given.
    block_lo/block_hi: blocked mode runs only those blocks (block_hi 0 = all).
    rng: RNG_PHILOX (the deterministic mode) or RNG_NATIVE (one Philox block
    per two hops)."""
    p = WalkParams()
    p.rule, p.sink, p.L, p.njump = rule, sink, L, njump
    p.jump_prob, p.seed, p.mode = jump_prob, seed & 0xFFFFFFFFFFFFFFFF, mode
    p.path_stride, p.max_hops, p.prob, p.aggregate = path_stride, max_hops, prob, int(aggregate)
    p.max_supersteps = max_supersteps
    p.block_lo, p.block_hi = block_lo, block_hi
    p.rng = rng
    p.cache_hints = 0 if cache_hints is None else (_lib.HINT_EXPLICIT | cache_hints)
    return p


# ---- the reference's 64-bit walk word (src/walks/walk.hpp:69-84), vectorised ----
def encode(source, current, hop) -> np.ndarray:
    s = np.asarray(source, dtype=np.uint64) & np.uint64(0xFFFFFF)
    c = np.asarray(current, dtype=np.uint64) & np.uint64(0x3FFFFFF)
    h = np.asarray(hop, dtype=np.uint64) & np.uint64(0x3FFF)
    return (s << np.uint64(40)) | (c << np.uint64(14)) | h


def get_source(w) -> np.ndarray:
    return ((np.asarray(w, dtype=np.uint64) >> np.uint64(40)) & np.uint64(0xFFFFFF)).astype(np.uint32)


def get_current(w) -> np.ndarray:
    return ((np.asarray(w, dtype=np.uint64) >> np.uint64(14)) & np.uint64(0x3FFFFFF)).astype(np.uint32)


def get_hop(w) -> np.ndarray:
    return (np.asarray(w, dtype=np.uint64) & np.uint64(0x3FFF)).astype(np.uint32)


def compute_blocks(rowptr: np.ndarray, blocksize_kb: int) -> np.ndarray:
    """compute_block of the reference (conversions.hpp:300-364) via the library."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
    nv = len(rowptr) - 1
    out = np.zeros(nv + 2, dtype=np.uint32)
    n = load().gw_compute_blocks(_ptr(rowptr), nv, blocksize_kb, _ptr(out), len(out))
    if n == 0:
        raise ValueError("compute_blocks: output too small")
    return out[:n].copy()


class Graph:
    """One engine context (graphwalker_engine + WalkManager on the device)."""

    def __init__(self, handle: int):
        self._h = c_void_p(handle)
        nv, ne, nb = c_uint32(), c_uint64(), c_uint32()
        check(load().gw_graph_info(self._h, byref(nv), byref(ne), byref(nb)), self._h)
        self.nv, self.ne, self.nblocks = nv.value, ne.value, nb.value
        blocks = np.zeros(self.nblocks + 1, dtype=np.uint32)
        check(load().gw_get_blocks(self._h, _ptr(blocks), len(blocks)), self._h)
        self.blocks = blocks

    # ---- constructors ----
    @classmethod
    def open(cls, base: str, blocksize_kb: int, residency: int = RESIDENT_HBM, nmblocks: int = 0,
             device: int = 0) -> "Graph":
        d = GraphDesc(base.encode(), blocksize_kb, nmblocks, residency, device)
        h = c_void_p()
        check(load().gw_open(byref(d), byref(h)))
        return cls(h.value)

    @classmethod
    def from_csr(cls, rowptr: np.ndarray, colidx: np.ndarray, blocks: np.ndarray,
                 residency: int = RESIDENT_HBM, device: int = 0) -> "Graph":
        rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
        colidx = np.ascontiguousarray(colidx, dtype=np.uint32)
        blocks = np.ascontiguousarray(blocks, dtype=np.uint32)
        h = c_void_p()
        check(load().gw_open_csr(_ptr(rowptr), _ptr(colidx) if len(colidx) else None,
                                 len(rowptr) - 1, _ptr(blocks), len(blocks) - 1, residency, device,
                                 byref(h)))
        return cls(h.value)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, seed: int = 1, a: float = 0.57,
             b: float = 0.19, c: float = 0.19, blocksize_kb: int = 4096, device: int = 0) -> "Graph":
        h = c_void_p()
        check(load().gw_open_rmat(scale, edge_factor, seed, a, b, c, blocksize_kb, device, byref(h)))
        return cls(h.value)

    def close(self) -> None:
        if self._h:
            load().gw_close(self._h)
            self._h = c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> c_void_p:
        return self._h

    def export_csr(self) -> tuple[np.ndarray, np.ndarray]:
        rowptr = np.zeros(self.nv + 1, dtype=np.uint64)
        colidx = np.zeros(max(self.ne, 1), dtype=np.uint32)
        check(load().gw_export_csr(self._h, _ptr(rowptr), _ptr(colidx)), self._h)
        return rowptr, colidx[: self.ne]

    def set_residency(self, residency: int, nmblocks: int = 0) -> None:
        """Moves the CSR between HBM and pinned host memory (streamed blocks)."""
        check(load().gw_set_residency(self._h, residency, nmblocks), self._h)

    def set_pool_budget(self, nbytes: int) -> None:
        """Device bytes the blocked engine's walk pools may hold (0 = no limit);
        past it, pools move to host memory and come back when their block runs."""
        check(load().gw_set_pool_budget(self._h, nbytes), self._h)

    def set_mapped_block_walks(self, max_walks: int) -> None:
        """Streamed blocks with at most max_walks pending walks (and in no
        device slot) are read in place from pinned host memory, not copied."""
        check(load().gw_set_mapped_block_walks(self._h, max_walks), self._h)

    # ---- pools (WalkManager) ----
    def walks_clear(self) -> None:
        check(load().gw_walks_clear(self._h), self._h)

    def walks_add(self, block: int, words: np.ndarray, ids: np.ndarray | None = None) -> None:
        words = np.ascontiguousarray(words, dtype=np.uint64)
        if ids is not None:
            ids = np.ascontiguousarray(ids, dtype=np.uint32)
            assert len(ids) == len(words)
        check(load().gw_walks_add(self._h, block, _ptr(words), _ptr(ids), len(words)), self._h)

    def add_walks_at(self, cur: np.ndarray, source: np.ndarray | None = None,
                     hop: np.ndarray | int = 0, ids: np.ndarray | None = None) -> None:
        """Places walks at global vertices `cur` into the pools of their blocks."""
        cur = np.asarray(cur, dtype=np.uint32)
        source = cur if source is None else np.asarray(source, dtype=np.uint32)
        hop = np.broadcast_to(np.asarray(hop, dtype=np.uint32), cur.shape)
        blk = np.searchsorted(self.blocks[1:], cur, side="right").astype(np.uint32)
        for b in np.unique(blk):
            m = blk == b
            words = encode(source[m], cur[m] - self.blocks[b], hop[m])
            self.walks_add(int(b), words, None if ids is None else np.asarray(ids, np.uint32)[m])

    def walks_count(self) -> tuple[np.ndarray, int]:
        per = np.zeros(self.nblocks, dtype=np.uint64)
        tot = c_uint64()
        check(load().gw_walks_count(self._h, _ptr(per), byref(tot)), self._h)
        return per, tot.value

    # ---- runs ----
    def run(self, p: WalkParams) -> RunStats:
        check(load().gw_run(self._h, byref(p)), self._h)
        return self.stats()

    def stats(self) -> RunStats:
        s = RunStats()
        check(load().gw_read_stats(self._h, byref(s)), self._h)
        return s

    def read_counts(self) -> np.ndarray:
        out = np.zeros(self.nv, dtype=np.uint32)
        check(load().gw_read_counts(self._h, _ptr(out), self.nv), self._h)
        return out

    def read_paths(self, nwalks: int, stride: int) -> tuple[np.ndarray, np.ndarray]:
        paths = np.zeros(nwalks * stride, dtype=np.uint32)
        lens = np.zeros(nwalks, dtype=np.uint32)
        check(load().gw_read_paths(self._h, _ptr(paths), _ptr(lens), nwalks), self._h)
        return paths.reshape(nwalks, stride), lens

    def read_pool(self, block: int) -> np.ndarray:
        """Pending walks of one block's device pool, as an (n, 4) array of
        (cur, id, src, hop) in pool order."""
        n = c_uint64()
        check(load().gw_read_pool(self._h, block, None, 0, byref(n)), self._h)
        out = np.zeros((max(n.value, 1), 4), dtype=np.uint32)
        check(load().gw_read_pool(self._h, block, _ptr(out), n.value, byref(n)), self._h)
        return out[: n.value]

    def read_closure(self) -> int:
        v = c_uint64()
        check(load().gw_read_closure(self._h, byref(v)), self._h)
        return v.value

    def run_pools(self, p: WalkParams, words: np.ndarray, pool_offsets: np.ndarray,
                  counts_out: np.ndarray, ids: np.ndarray | None = None) -> None:
        check(load().gw_run_pools(self._h, byref(p), _ptr(words), _ptr(pool_offsets), _ptr(ids),
                                  _ptr(counts_out)), self._h)

    def run_pools_submit(self, p: WalkParams, words: np.ndarray, pool_offsets: np.ndarray,
                         counts_out: np.ndarray, ids: np.ndarray | None = None) -> int:
        """Queues a run_pools (gw_run_pools_submit) and returns its ticket; the
        arrays must stay alive, and counts_out unread, until run_pools_wait."""
        t = c_uint64(0)
        check(load().gw_run_pools_submit(self._h, byref(p), _ptr(words), _ptr(pool_offsets), _ptr(ids),
                                         _ptr(counts_out), byref(t)), self._h)
        return int(t.value)

    def run_pools_wait(self, ticket: int) -> None:
        """Blocks until the run of `ticket` has its counts on the host."""
        check(load().gw_run_pools_wait(self._h, ticket), self._h)

    # ---- device-pointer entry points ----
    def walk_device(self, p: WalkParams, walks, n: int, counts=None, paths=None, plen=None,
                    closure=None, stream: int | None = None) -> None:
        check(load().gw_walk_device(self._h, byref(p), _ptr(walks), n, _ptr(counts), _ptr(paths),
                                    _ptr(plen), _ptr(closure), stream), self._h)

    def unpack_words_device(self, block: int, words, ids, n: int, out, stream: int | None = None) -> None:
        check(load().gw_unpack_words_device(self._h, block, _ptr(words), _ptr(ids), n, _ptr(out),
                                            stream), self._h)

    def pack_words_device(self, walks, n: int, words, wblocks=None, stream: int | None = None) -> None:
        check(load().gw_pack_words_device(self._h, _ptr(walks), n, _ptr(words), _ptr(wblocks),
                                          stream), self._h)

    def simrank_meet(self, paths_a, paths_b, R: int, L: int, stream: int | None = None) -> np.ndarray:
        """Per-position first-meeting pair counts of two device path arrays
        (R rows of L visits; gw_simrank_meet)."""
        meet = np.zeros(L, np.uint64)
        check(load().gw_simrank_meet(self._h, _ptr(paths_a), _ptr(paths_b), R, L, _ptr(meet), stream), self._h)
        return meet

    def simrank_batch(self, a, b, R: int, L: int, seed: int = 42, decay: float = 0.8):
        """SimRank estimates of the queries (a[q], b[q]) and their per-position
        first-meeting counts (gw_simrank_batch): scores float64[nq], meet uint64[nq, L]."""
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = np.ascontiguousarray(b, dtype=np.uint32)
        nq = len(a)
        scores = np.zeros(nq, np.float64)
        meet = np.zeros((nq, L), np.uint64)
        p = params(_lib.RULE_RESTART, _lib.SINK_PATH_RECORD, L, seed=seed)
        check(load().gw_simrank_batch(self._h, byref(p), _ptr(a), _ptr(b), nq, R, decay, _ptr(meet), _ptr(scores)),
              self._h)
        return scores, meet

    def walk_autotune(self, p: WalkParams, walks, n: int) -> int:
        """CTAs per SM chosen for this graph's later resident walk launches
        (gw_walk_autotune), timed on the given device walks."""
        out = c_uint32()
        check(load().gw_walk_autotune(self._h, byref(p), _ptr(walks), n, byref(out)), self._h)
        return out.value

    def sync(self, stream: int | None = None) -> None:
        check(load().gw_sync(self._h, stream), self._h)

    # ---- multi-source PPR queries ----
    def ppr(self, p: WalkParams, sources, budgets, k: int = 100, batched: bool = True):
        """Top-k (ids, counts) per query, shape (nq, k), and the run's PprStats."""
        sources = np.ascontiguousarray(sources, dtype=np.uint32)
        budgets = np.ascontiguousarray(budgets, dtype=np.uint32)
        nq = len(sources)
        ids = np.zeros(nq * k, dtype=np.uint32)
        counts = np.zeros(nq * k, dtype=np.uint32)
        st = _lib.PprStats()
        check(load().gw_ppr_run(self._h, byref(p), _ptr(sources), _ptr(budgets), nq, k, int(batched), _ptr(ids),
                                _ptr(counts), byref(st)), self._h)
        return ids.reshape(nq, k), counts.reshape(nq, k), st

    def expected_visits(self, p: WalkParams, source: int) -> np.ndarray:
        """FP64 expected visits per vertex of one walk from `source`."""
        out = np.zeros(self.nv, dtype=np.float64)
        check(load().gw_expected_visits(self._h, byref(p), source, _ptr(out)), self._h)
        return out

    def ppr_autotune(self, p: WalkParams, sources, budgets) -> tuple[int, int]:
        """(threads per SM, walks per cursor grab) chosen for this graph's later
        batched PPR and serving launches (gw_ppr_autotune)."""
        sources = np.ascontiguousarray(sources, dtype=np.uint32)
        budgets = np.ascontiguousarray(budgets, dtype=np.uint32)
        threads, chunk = c_uint32(), c_uint32()
        check(load().gw_ppr_autotune(self._h, byref(p), _ptr(sources), _ptr(budgets), len(sources), byref(threads),
                                     byref(chunk)), self._h)
        return threads.value, chunk.value

    def serve(self, p: WalkParams, k: int = 100, mode: int = _lib.SERVE_BATCHED, table_slots: int = 0,
              max_walks_per_step: int = 0, quantum: int = 0) -> "Server":
        return Server(self, p, k, mode, table_slots, max_walks_per_step, quantum)

    def set_l2_fetch_granularity(self, nbytes: int) -> int:
        """Sets the context's L2 fetch granularity (0 = leave); returns the old one."""
        old = c_uint32()
        check(load().gw_set_l2_fetch_granularity(self._h, nbytes, byref(old)), self._h)
        return old.value

    def set_l2_persisting(self, nbytes: int) -> None:
        check(load().gw_set_l2_persisting(self._h, nbytes), self._h)

    def set_edge_records(self, mode: int) -> bool:
        """EDGE_RECORDS_OFF / _ON / _AUTO (gw_set_edge_records); True when in use."""
        built = c_uint32()
        check(load().gw_set_edge_records(self._h, mode, byref(built)), self._h)
        return bool(built.value)

    def probe_gather(self, buf, n_words: int, loads: int, iters: int = 5) -> float:
        out = c_double()
        check(load().gw_probe_gather(self._h, _ptr(buf), n_words, loads, iters, byref(out)), self._h)
        return out.value

    def probe_red(self, counters, n_words: int, ops: int, iters: int = 5) -> float:
        """Random visit-counter updates per second (gw_probe_red)."""
        out = c_double()
        check(load().gw_probe_red(self._h, _ptr(counters), n_words, ops, iters, byref(out)), self._h)
        return out.value


class Server:
    """A continuous-batching PPR query server on one graph (gw_serve_*)."""

    def __init__(self, graph: Graph, p: WalkParams, k: int, mode: int, table_slots: int, max_walks_per_step: int,
                 quantum: int):
        self.graph, self.k = graph, k
        cfg = _lib.ServeConfig(table_slots, max_walks_per_step, quantum, k, mode)
        h = c_void_p()
        check(load().gw_serve_open(graph.handle, byref(p), byref(cfg), byref(h)), graph.handle)
        self._h = h

    @staticmethod
    def clock_ns() -> int:
        return load().gw_serve_clock_ns()

    def submit(self, source: int, budget: int, stream: int = 0, arrival_ns: int = 0) -> int:
        t = c_uint64()
        check(load().gw_serve_submit(self._h, source, budget, stream, arrival_ns, byref(t)), self.graph.handle)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(ids[k], counts[k], ServeTiming) of a ticket."""
        ids = np.zeros(self.k, dtype=np.uint32)
        counts = np.zeros(self.k, dtype=np.uint32)
        tm = _lib.ServeTiming()
        check(load().gw_serve_wait(self._h, ticket, timeout_ms, _ptr(ids), _ptr(counts), byref(tm)),
              self.graph.handle)
        return ids, counts, tm

    def stats(self) -> _lib.ServeStats:
        s = _lib.ServeStats()
        check(load().gw_serve_get_stats(self._h, byref(s)), self.graph.handle)
        return s

    def close(self) -> None:
        if self._h:
            load().gw_serve_close(self._h)
            self._h = c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
