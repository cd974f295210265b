"""The graph-context calls that graphwalker_b200.partitioned.Partition makes
(add_walks_at, run, read_counts, read_pool, walks_clear), restated on the C
oracle's block step (gwo_block_step) so that the partitioned protocol runs on
the CPU.  Test infrastructure only: the product runs them on the device."""
import ctypes

import numpy as np


class OracleBlocks:
    def __init__(self, oracle, rowptr, colidx, blocks):
        self.o = oracle
        self.rp = np.ascontiguousarray(rowptr, np.uint64)
        self.ci = np.ascontiguousarray(colidx if len(colidx) else np.zeros(1, np.uint32), np.uint32)
        self.blocks = np.ascontiguousarray(blocks, np.uint32)
        self.nv = len(self.rp) - 1
        self.nblocks = len(self.blocks) - 1
        self.walks_clear()
        self.counts = np.zeros(self.nv, np.uint32)

    def walks_clear(self):
        self.pools = [np.zeros((0, 4), np.uint32) for _ in range(self.nblocks)]

    def add_walks_at(self, cur, source=None, hop=0, ids=None):
        cur = np.asarray(cur, np.uint32)
        source = cur if source is None else np.asarray(source, np.uint32)
        hop = np.broadcast_to(np.asarray(hop, np.uint32), cur.shape)
        ids = source if ids is None else np.asarray(ids, np.uint32)
        blk = np.searchsorted(self.blocks[1:], cur, side="right")
        recs = np.stack([cur, ids, source, hop], axis=1).astype(np.uint32)
        for b in np.unique(blk):
            self.pools[b] = np.concatenate([self.pools[b], recs[blk == b]])

    def run(self, p):
        """Every walk in blocks [p.block_lo, p.block_hi) (all when block_hi is 0)
        advances until it ends or leaves them."""
        lo, hi = (p.block_lo, p.block_hi) if p.block_hi else (0, self.nblocks)
        prm = self.o.make_params(p.rule, p.L, p.jump_prob, p.njump or self.nv, p.seed, p.max_hops or 65535, p.rng)
        self.counts = np.zeros(self.nv, np.uint32)
        P = self.o._p
        while True:
            todo = [b for b in range(lo, hi) if len(self.pools[b])]
            if not todo:
                return
            b = todo[0]
            pool = self.pools[b]
            self.pools[b] = np.zeros((0, 4), np.uint32)
            c, i, s, h = (np.ascontiguousarray(pool[:, k]) for k in range(4))
            dest = np.zeros(len(c), np.uint32)
            st = self.o.lib().gwo_block_step(P(self.rp), P(self.ci), self.nv, P(self.blocks), self.nblocks, b,
                                             P(c), P(i), P(s), P(h), len(c), ctypes.byref(prm), P(self.counts),
                                             P(dest))
            assert st == 0
            moved = np.stack([c, i, s, h], axis=1)
            for d in np.unique(dest):
                if d != 0xFFFFFFFF:
                    self.pools[d] = np.concatenate([self.pools[d], moved[dest == d]])

    def read_counts(self):
        return self.counts.copy()

    def read_pool(self, b):
        return self.pools[b].copy()
