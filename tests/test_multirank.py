"""The multi-GPU path's host logic with two gloo ranks on the CPU: each rank
runs its shard of the walks (the C oracle stands in for the device) and the
visit counts are summed with the same all-reduce the bench uses."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    import sys
    sys.path.insert(0, str(ROOT))
    from graphwalker_b200 import sharding
    from oracle import py_oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rp, ci = py_oracle.rmat_csr(11, 8, seed=5)
    nv = len(rp) - 1
    # weak scaling: one walk per vertex per rank, ids offset by rank
    off = sharding.walk_id_offset(rank, nv)
    cur = np.arange(nv, dtype=np.uint32)
    r = py_oracle.run_walks(rp, ci, cur, ids=(cur + off).astype(np.uint32), rule=0, L=10, seed=3)
    counts = torch.from_numpy(r["counts"].view(np.int32).copy())
    sharding.reduce_counts(counts)
    # strong scaling: one walk set split into contiguous ranges
    lo, hi = sharding.shard_range(5000, rank, world)
    cur2 = (np.arange(lo, hi) % nv).astype(np.uint32)
    r2 = py_oracle.run_walks(rp, ci, cur2, ids=np.arange(lo, hi, dtype=np.uint32), rule=1, L=10, seed=4)
    counts2 = torch.from_numpy(r2["counts"].view(np.int32).copy())
    sharding.reduce_counts(counts2)
    slowest = sharding.max_over_ranks(float(rank + 1))
    if rank == 0:
        np.save(os.path.join(out_dir, "weak.npy"), counts.numpy())
        np.save(os.path.join(out_dir, "strong.npy"), counts2.numpy())
        np.save(os.path.join(out_dir, "slowest.npy"), np.array([slowest]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_sum_to_the_single_process_result(tmp_path, oracle):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rp, ci = oracle.rmat_csr(11, 8, seed=5)
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    ref = np.zeros(nv, np.uint64)
    for rank in range(world):
        ref += oracle.run_walks(rp, ci, cur, ids=(cur + rank * nv).astype(np.uint32), rule=0, L=10, seed=3)["counts"]
    assert np.array_equal(np.load(tmp_path / "weak.npy").view(np.uint32), ref.astype(np.uint32))
    cur2 = (np.arange(5000) % nv).astype(np.uint32)
    ref2 = oracle.run_walks(rp, ci, cur2, ids=np.arange(5000, dtype=np.uint32), rule=1, L=10, seed=4)["counts"]
    assert np.array_equal(np.load(tmp_path / "strong.npy").view(np.uint32), ref2)
    assert float(np.load(tmp_path / "slowest.npy")[0]) == 2.0


def test_shard_ranges_cover_exactly():
    from graphwalker_b200 import sharding
    for total in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            spans = [sharding.shard_range(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
