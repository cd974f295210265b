"""Vertex-partitioned walks (graphwalker_b200.partitioned) on the CPU: the
rank protocol with the C oracle's block step standing in for each rank's
device engine (tests/oracle_blocks.py).  Walks that enter another rank's
blocks are exchanged with the all-to-all the GPUs use (two gloo ranks here);
the summed counts equal one process's run of the same walks exactly."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT

CASES = [(0, 10), (1, 20), (3, 6)]  # (rule, L): jump, stop, restart (reads the source)


def _graph(oracle):
    rp, ci = oracle.rmat_csr(11, 8, seed=5)
    return rp, ci, oracle.compute_blocks(rp, 8)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    import sys
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle import py_oracle
    from oracle_blocks import OracleBlocks

    from graphwalker_b200 import partitioned
    from graphwalker_b200.engine import params
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rp, ci, blocks = _graph(py_oracle)
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    ids = (np.arange(nv, dtype=np.uint32) * 7 + 3).astype(np.uint32)
    for rule, L in CASES:
        g = OracleBlocks(py_oracle, rp, ci, blocks)
        counts, st = partitioned.run_partitioned(g, params(rule, L=L, seed=11), cur, ids=ids, rank=rank,
                                                 world=world)
        if rank == 0:
            np.save(os.path.join(out_dir, f"counts_{rule}.npy"), counts)
            np.save(os.path.join(out_dir, f"stats_{rule}.npy"), np.array([st["rounds"], st["walks_sent"]]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_equal_one_process(tmp_path, oracle):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rp, ci, _ = _graph(oracle)
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    ids = (np.arange(nv, dtype=np.uint32) * 7 + 3).astype(np.uint32)
    for rule, L in CASES:
        ref = oracle.run_walks(rp, ci, cur, ids=ids, src=cur, rule=rule, L=L, seed=11)["counts"]
        got = np.load(tmp_path / f"counts_{rule}.npy")
        assert np.array_equal(got, ref.astype(np.uint64)), rule
        rounds, sent = np.load(tmp_path / f"stats_{rule}.npy")
        assert rounds >= 2 and sent > 0  # walks did cross between the ranks


def test_partitions_in_lock_step(oracle):
    """Three partitions driven round by round in one process, records routed
    directly: the same protocol without a process group."""
    from oracle_blocks import OracleBlocks

    from graphwalker_b200 import partitioned
    from graphwalker_b200.engine import params
    rp, ci, blocks = _graph(oracle)
    nv = len(rp) - 1
    rng = np.random.default_rng(2)
    cur = rng.integers(0, nv, 3000).astype(np.uint32)
    ids = np.arange(3000, dtype=np.uint32)
    hop = rng.integers(0, 3, 3000).astype(np.uint32)
    world = 3
    p = params(1, L=20, seed=4)
    parts = [partitioned.Partition(OracleBlocks(oracle, rp, ci, blocks), p, r, world) for r in range(world)]
    assert sum(part.place(cur, hop=hop, ids=ids) for part in parts) == len(cur)
    while True:
        outs = [part.step() for part in parts]
        moved = 0
        for r, part in enumerate(parts):
            inc = np.concatenate([outs[s][r] for s in range(world)])
            part.accept(inc)
            moved += len(inc)
        if moved == 0:
            break
    got = sum(part.counts for part in parts)
    ref = oracle.run_walks(rp, ci, cur, ids=ids, src=cur, hop0=hop, rule=1, L=20, seed=4)["counts"]
    assert np.array_equal(got, ref.astype(np.uint64))
    # each vertex is counted by its owner only
    for part in parts:
        outside = ~part.owns(np.arange(nv, dtype=np.uint32))
        assert not part.counts[outside].any()


def test_more_ranks_than_blocks(oracle):
    """Eight partitions of a five-block graph: three ranks own no block, run
    nothing and receive nothing; the counts are still the oracle's."""
    from oracle_blocks import OracleBlocks

    from graphwalker_b200 import partitioned
    from graphwalker_b200.engine import params
    rp, ci = oracle.rmat_csr(10, 8, seed=3)
    blocks = oracle.compute_blocks(rp, 7)
    assert len(blocks) - 1 == 5
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    world = 8
    parts = [partitioned.Partition(OracleBlocks(oracle, rp, ci, blocks), params(0, L=10, seed=1), r, world)
             for r in range(world)]
    assert sum(part.place(cur, ids=cur) for part in parts) == nv
    while True:
        outs = [part.step() for part in parts]
        moved = 0
        for r, part in enumerate(parts):
            inc = np.concatenate([outs[s][r] for s in range(world)])
            part.accept(inc)
            moved += len(inc)
        if moved == 0:
            break
    ref = oracle.run_walks(rp, ci, cur, ids=cur, src=cur, rule=0, L=10, seed=1)["counts"]
    assert np.array_equal(sum(part.counts for part in parts), ref.astype(np.uint64))
    assert sum(part.lo == part.hi for part in parts) == 3


def test_partition_rejects_other_sinks_and_ranks(oracle):
    import pytest

    from oracle_blocks import OracleBlocks

    from graphwalker_b200 import partitioned
    from graphwalker_b200.engine import params
    rp, ci = oracle.rmat_csr(10, 8, seed=3)
    g = OracleBlocks(oracle, rp, ci, oracle.compute_blocks(rp, 12))
    with pytest.raises(ValueError):
        partitioned.Partition(g, params(0, sink=0, L=10), 0, 2)
    with pytest.raises(ValueError):
        partitioned.Partition(g, params(0, L=10), 2, 2)


def test_owned_blocks_cover_every_block():
    from graphwalker_b200 import partitioned
    for nb in (1, 5, 33, 257):
        for world in (1, 2, 3, 8):
            owner = partitioned.block_owners(nb, world)
            spans = [partitioned.owned_blocks(nb, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nb
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            for r, (lo, hi) in enumerate(spans):
                assert (owner[lo:hi] == r).all()
