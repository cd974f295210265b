"""Vertex-partitioned walks on the device: each rank's context runs only its
own blocks (gw_walk_params block_lo / block_hi), and walks that leave them are
read from the pools of the blocks they entered and handed to the owner.

One GPU holds every rank's context here, and the ranks are driven round by
round in one process (no kernel waits on another), with the records routed
directly; the exchange over a process group is the all-to-all that
tests/test_partitioned.py runs with gloo ranks.  The summed counts must equal
the oracle's counts of the same walks exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _graph(oracle):
    rp, ci = oracle.rmat_csr(13, 8, seed=5)
    return rp, ci, oracle.compute_blocks(rp, 16)


def _lock_step(parts):
    world = len(parts)
    while True:
        outs = [part.step() for part in parts]
        moved = 0
        for r, part in enumerate(parts):
            inc = np.concatenate([outs[s][r] for s in range(world)])
            part.accept(inc)
            moved += len(inc)
        if moved == 0:
            return


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("rule,L", [(0, 10), (1, 20), (3, 6)])
def test_partitioned_counts_equal_the_oracle(cuda_device, oracle, world, rule, L):
    import graphwalker_b200 as gw
    from graphwalker_b200 import partitioned
    rp, ci, blocks = _graph(oracle)
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    ids = (np.arange(nv, dtype=np.uint32) * 5 + 1).astype(np.uint32)
    ref = oracle.run_walks(rp, ci, cur, ids=ids, src=cur, rule=rule, L=L, seed=9)["counts"]
    graphs = [gw.Graph.from_csr(rp, ci, blocks) for _ in range(world)]
    try:
        p = gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=9)
        parts = [partitioned.Partition(g, p, r, world) for r, g in enumerate(graphs)]
        assert sum(part.place(cur, ids=ids) for part in parts) == nv
        _lock_step(parts)
        assert np.array_equal(sum(part.counts for part in parts), ref.astype(np.uint64))
        assert all(part.rounds >= 2 for part in parts) and sum(part.walks_sent for part in parts) > 0
    finally:
        for g in graphs:
            g.close()


def test_owned_block_range_leaves_other_pools(cuda_device, oracle):
    """A blocked run restricted to blocks [lo, hi) empties those pools, counts
    visits only at their vertices, and leaves the walks that moved elsewhere in
    their new blocks' pools; a range outside the graph is rejected."""
    import graphwalker_b200 as gw
    rp, ci, blocks = _graph(oracle)
    nv, nb = len(rp) - 1, len(blocks) - 1
    lo, hi = 1, nb // 2 + 1
    cur = np.arange(nv, dtype=np.uint32)
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        G.walks_clear()
        G.add_walks_at(cur)
        G.run(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=2, mode=gw.MODE_BLOCKED, block_lo=lo, block_hi=hi))
        counts = G.read_counts()
        per_block = [len(G.read_pool(b)) for b in range(nb)]
        assert all(per_block[b] == 0 for b in range(lo, hi))
        assert sum(per_block) > 0
        inside = (cur >= blocks[lo]) & (cur < blocks[hi])
        assert counts[inside].sum() > 0 and not counts[~inside].any()
        with pytest.raises(gw.GwError):
            G.run(gw.params(0, gw.SINK_VERTEX_COUNT, 10, mode=gw.MODE_BLOCKED, block_lo=2, block_hi=nb + 1))


def test_run_partitioned_with_one_rank(cuda_device, oracle):
    """run_partitioned over a one-rank gloo group: the exchange is empty and
    the run equals the oracle."""
    import socket

    import torch.distributed as dist

    import graphwalker_b200 as gw
    from graphwalker_b200 import partitioned
    rp, ci, blocks = _graph(oracle)
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        with gw.Graph.from_csr(rp, ci, blocks) as G:
            counts, st = partitioned.run_partitioned(G, gw.params(1, gw.SINK_VERTEX_COUNT, 20, seed=6), cur,
                                                     ids=cur, rank=0, world=1)
    finally:
        dist.destroy_process_group()
    ref = oracle.run_walks(rp, ci, cur, ids=cur, src=cur, rule=1, L=20, seed=6)["counts"]
    assert np.array_equal(counts, ref.astype(np.uint64))
    assert st["walks_sent"] == 0
