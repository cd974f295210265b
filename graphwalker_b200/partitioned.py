"""Vertex-partitioned walks over several GPUs: the graph is split by blocks and
a walk travels to the GPU that owns the block it enters.

This is the multi-GPU form of the out-of-core workload, for a graph larger than
one GPU's HBM: rank r owns a contiguous range of the reference's blocks
(`owned_blocks`) and its blocked engine runs only those (gw_walk_params
block_lo / block_hi).  One round is:

1. run: every walk pending in an owned block advances while it stays inside
   the rank's blocks (the engine's supersteps).  A visit is counted where it
   happens, so each vertex is counted by its owner only;
2. collect: the walks that moved into another rank's block are read from those
   blocks' pools (gw_read_pool) and grouped by owner;
3. exchange: one all-to-all of the record counts, then one all-to-all-v of the
   records (cur, id, src, hop: 16 B each);
4. accept: the received walks are placed in the pools of their blocks.

The run ends after the first round in which no rank received a walk (one
all-reduce per round).  Walks keep their ids and hops, and every draw is keyed
on (walk id, hop), so the summed counts equal a single-GPU run's exactly,
whatever the partition.  Between rounds a walk travels as the reference's
64-bit walk word (walk.hpp:69-84), so its source is the word's 24-bit field.

The reference runs one process over all blocks (graphwalker.hpp:272-311); it
has no counterpart to this exchange.  The rank-level logic is engine-agnostic:
`Partition` drives any object with the Graph methods it calls (nv, nblocks,
add_walks_at, run, read_counts, read_pool, walks_clear).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .sharding import shard_range


def owned_blocks(nblocks: int, rank: int, world: int) -> tuple[int, int]:
    """Blocks [lo, hi) of `rank`: contiguous, equal counts (blocks hold equal bytes)."""
    return shard_range(nblocks, rank, world)


def block_owners(nblocks: int, world: int) -> np.ndarray:
    """Owning rank of every block."""
    owner = np.zeros(nblocks, np.int64)
    for r in range(world):
        lo, hi = owned_blocks(nblocks, r, world)
        owner[lo:hi] = r
    return owner


class Partition:
    """One rank's share of a partitioned run on its graph context."""

    def __init__(self, graph, params, rank: int, world: int):
        if params.sink != _lib.SINK_VERTEX_COUNT:
            raise ValueError("a partitioned run counts visits per vertex (SINK_VERTEX_COUNT)")
        if not 0 <= rank < world:
            raise ValueError(f"rank {rank} outside a world of {world}")
        self.g = graph
        self.rank, self.world = rank, world
        self.lo, self.hi = owned_blocks(graph.nblocks, rank, world)
        self.owner = block_owners(graph.nblocks, world)
        self.blocks = np.asarray(graph.blocks, np.uint32)
        p = type(params).from_buffer_copy(params)
        p.mode = _lib.MODE_BLOCKED
        p.block_lo, p.block_hi = self.lo, self.hi
        self.params = p
        self.counts = np.zeros(graph.nv, np.uint64)
        self.rounds = 0
        self.walks_sent = 0

    def owns(self, cur: np.ndarray) -> np.ndarray:
        """Which of the vertices `cur` lie in this rank's blocks."""
        cur = np.asarray(cur, np.uint32)
        return (cur >= self.blocks[self.lo]) & (cur < self.blocks[self.hi])

    def place(self, cur, source=None, hop=0, ids=None) -> int:
        """Places the walks that start in this rank's blocks (the caller may
        pass the whole walk set); returns how many were placed."""
        cur = np.asarray(cur, np.uint32)
        source = cur if source is None else np.asarray(source, np.uint32)
        hop = np.broadcast_to(np.asarray(hop, np.uint32), cur.shape)
        ids = np.arange(len(cur), dtype=np.uint32) if ids is None else np.asarray(ids, np.uint32)
        m = self.owns(cur)
        if m.any():
            self.g.add_walks_at(cur[m], source=source[m], hop=hop[m], ids=ids[m])
        return int(m.sum())

    def step(self) -> list[np.ndarray]:
        """Runs the owned blocks until no walk is left in them and returns the
        walks that left, one (n, 4) array of (cur, id, src, hop) per rank.  A
        rank that owns no block (more ranks than blocks) has nothing to run."""
        out: list[list[np.ndarray]] = [[] for _ in range(self.world)]
        self.rounds += 1
        if self.lo == self.hi:
            return [np.zeros((0, 4), np.uint32) for _ in range(self.world)]
        self.g.run(self.params)
        self.counts += self.g.read_counts().astype(np.uint64)
        for b in range(self.g.nblocks):
            if self.lo <= b < self.hi:
                continue
            recs = self.g.read_pool(b)
            if len(recs):
                out[int(self.owner[b])].append(recs)
        self.g.walks_clear()
        res = [np.concatenate(o) if o else np.zeros((0, 4), np.uint32) for o in out]
        self.walks_sent += sum(len(r) for r in res)
        return res

    def accept(self, recs: np.ndarray) -> None:
        """Places walks received from other ranks (all in this rank's blocks)."""
        recs = np.asarray(recs, np.uint32).reshape(-1, 4)
        if not len(recs):
            return
        if not self.owns(recs[:, 0]).all():
            raise ValueError(f"rank {self.rank} received a walk outside its blocks")
        self.g.add_walks_at(recs[:, 0], source=recs[:, 2], hop=recs[:, 3], ids=recs[:, 1])


def exchange_records(outgoing: list[np.ndarray], group=None, device=None) -> np.ndarray:
    """All-to-all-v of walk records: outgoing[r] goes to rank r; returns what
    this rank received.  Tensors live on `device` (a CUDA device for NCCL)."""
    import torch
    import torch.distributed as dist
    send_n = torch.tensor([len(o) for o in outgoing], dtype=torch.int64, device=device)
    recv_n = torch.empty_like(send_n)
    dist.all_to_all_single(recv_n, send_n, group=group)
    flat = np.ascontiguousarray(np.concatenate(outgoing), dtype=np.uint32).reshape(-1, 4)
    send = torch.from_numpy(flat.view(np.int32)).to(device)
    rn = [int(x) for x in recv_n.cpu().tolist()]
    recv = torch.empty((sum(rn), 4), dtype=torch.int32, device=device)
    dist.all_to_all_single(recv, send, output_split_sizes=rn,
                           input_split_sizes=[int(x) for x in send_n.cpu().tolist()], group=group)
    return recv.cpu().numpy().view(np.uint32)


def run_partitioned(graph, params, cur, source=None, hop=0, ids=None, *, rank: int, world: int, group=None,
                    device=None, reduce: bool = True) -> tuple[np.ndarray, dict]:
    """Runs a walk set over `world` ranks, this process being `rank` (the
    process group is already initialised).  Every rank passes the same walk
    set; each keeps the walks that start in its blocks.  Returns the visit
    counts (summed over ranks when `reduce`, else this rank's) and stats."""
    import torch
    import torch.distributed as dist
    part = Partition(graph, params, rank, world)
    part.place(cur, source, hop, ids)
    while True:
        incoming = exchange_records(part.step(), group=group, device=device)
        part.accept(incoming)
        moved = torch.tensor([len(incoming)], dtype=torch.int64, device=device)
        dist.all_reduce(moved, group=group)
        if int(moved.item()) == 0:
            break
    counts = part.counts
    if reduce:
        t = torch.from_numpy(counts.view(np.int64).copy()).to(device)
        dist.all_reduce(t, group=group)
        counts = t.cpu().numpy().view(np.uint64)
    stats = {"rounds": part.rounds, "walks_sent": part.walks_sent, "blocks": (part.lo, part.hi)}
    return counts, stats
