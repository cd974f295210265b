"""Parity of the CUDA walk engine with the reference and the oracle.

Bit-exact for every comparison here: visit counts, per-walk trajectories,
closure counts, final pools and scheduler decisions are integers.
"""
import numpy as np
import pytest

from conftest import golden_runs, load_golden

pytestmark = pytest.mark.gpu

CASES = ["hand", "rmat10", "rmat13"]
# both graph layouts of the resident kernels: plain CSR (OFF) and edge records (ON)
LAYOUTS = [0, 1]


def _graph(g, residency=0, layout=None):
    import graphwalker_b200 as gw
    G = gw.Graph.from_csr(g["rowptr"], g["colidx"], g["blocks"], residency=residency)
    if layout is not None:
        assert G.set_edge_records(layout) == bool(layout)
    return G


def _add_golden_walks(G, g, tag):
    cur, src, hop = g[f"{tag}_cur"], g[f"{tag}_src"], g[f"{tag}_hop"]
    G.walks_clear()
    G.add_walks_at(cur, source=src, hop=hop, ids=src)
    return cur, src, hop


def _pool_order(G, cur):
    """Walk order of the device pools (pool by pool, as gw_run uploads them)."""
    blk = np.searchsorted(G.blocks[1:], cur, side="right")
    return np.argsort(blk, kind="stable")


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("aggregate", [False, True])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_counts_match_reference_golden(cuda_device, case, aggregate, layout):
    import graphwalker_b200 as gw
    g = load_golden(case)
    with _graph(g, layout=layout) as G:
        for tag in golden_runs(g):
            _add_golden_walks(G, g, tag)
            p = gw.params(int(g[f"{tag}_rule"]), gw.SINK_VERTEX_COUNT, int(g[f"{tag}_L"]),
                          seed=int(g["seed"]), aggregate=aggregate)
            G.run(p)
            assert np.array_equal(G.read_counts(), g[f"{tag}_counts"]), f"{case}/{tag}"


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("layout", LAYOUTS)
def test_paths_and_closure_match_reference_golden(cuda_device, case, layout):
    import graphwalker_b200 as gw
    g = load_golden(case)
    with _graph(g, layout=layout) as G:
        for tag in golden_runs(g):
            cur, src, hop = _add_golden_walks(G, g, tag)
            rule, L = int(g[f"{tag}_rule"]), int(g[f"{tag}_L"])
            gp = g[f"{tag}_paths"]
            stride = gp.shape[1] if tag != "simrank" else L
            G.run(gw.params(rule, gw.SINK_PATH_RECORD, L, seed=int(g["seed"]), path_stride=stride))
            paths, lens = G.read_paths(len(cur), stride)
            order = _pool_order(G, cur)
            for row, j in enumerate(order):
                k = min(int(lens[row]), stride)
                if tag == "simrank":
                    i = j % (len(cur) // 2)
                    ref = gp[src[j]][i * L: i * L + L]
                else:
                    ref = gp[src[j]]
                assert np.array_equal(paths[row][:k], ref[:k]), f"{case}/{tag} walk {j}"
                assert np.all(ref[k:stride] == 0xFFFFFFFF)
            G.run(gw.params(rule, gw.SINK_CLOSURE_COUNT, L, seed=int(g["seed"])))
            assert G.read_closure() == int(g[f"{tag}_closure"])


@pytest.mark.parametrize("rule,L", [(0, 10), (1, 10), (2, 10), (3, 7), (4, 20)])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_rmat16_all_rules_match_oracle(cuda_device, oracle, rule, L, layout):
    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(16, 16, seed=2)
    blocks = oracle.compute_blocks(rp, 512)
    nv = len(rp) - 1
    rng = np.random.default_rng(rule)
    cur = rng.integers(0, nv, 200_000).astype(np.uint32)
    ids = np.arange(len(cur), dtype=np.uint32)
    src = cur.copy()
    ref = oracle.run_walks(rp, ci, cur, ids=ids, src=src, rule=rule, L=L, seed=99, stride=32, closure=True)
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        assert G.set_edge_records(layout) == bool(layout)
        G.add_walks_at(cur, source=src, ids=ids)
        G.run(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=99))
        assert np.array_equal(G.read_counts(), ref["counts"])
        G.run(gw.params(rule, gw.SINK_CLOSURE_COUNT, L, seed=99))
        assert G.read_closure() == ref["closure"]
        if rule != 2:
            G.run(gw.params(rule, gw.SINK_PATH_RECORD, L, seed=99, path_stride=32))
            paths, lens = G.read_paths(len(cur), 32)
            order = _pool_order(G, cur)
            assert np.array_equal(lens, ref["plen"][order])
            assert np.array_equal(paths, ref["paths"][order])


def test_ppr_single_source_matches_oracle(cuda_device, oracle):
    """Single-source PPR: many walks from one vertex, distinct walk ids."""
    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(14, 16, seed=1)
    blocks = oracle.compute_blocks(rp, 128)
    deg = np.diff(rp.astype(np.int64))
    s = int(np.argmax(deg))
    n = 100_000
    cur = np.full(n, s, np.uint32)
    ids = np.arange(n, dtype=np.uint32)
    ref = oracle.run_walks(rp, ci, cur, ids=ids, rule=4, L=20, seed=5)
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        for agg in (False, True):
            G.walks_clear()
            G.add_walks_at(cur, ids=ids)
            G.run(gw.params(gw.RULE_PPR, gw.SINK_VERTEX_COUNT, 20, seed=5, aggregate=agg))
            assert np.array_equal(G.read_counts(), ref["counts"])


@pytest.mark.parametrize("case", ["rmat10", "rmat13"])
@pytest.mark.parametrize("prob", [0.0, 0.2, 1.0])
def test_blocked_engine_matches_reference_loop(cuda_device, oracle, case, prob):
    import graphwalker_b200 as gw
    g = load_golden(case)
    for tag in ("jump", "stop"):
        rule, L = int(g[f"{tag}_rule"]), int(g[f"{tag}_L"])
        cur = g[f"{tag}_cur"]
        ref = oracle.block_engine(g["rowptr"], g["colidx"], g["blocks"], cur, rule=rule, L=L,
                                  seed=int(g["seed"]), prob=prob)
        assert np.array_equal(ref["counts"], g[f"{tag}_counts"])
        for residency in (gw.RESIDENT_HBM, gw.STREAM_PINNED):
            with _graph(g, residency) as G:
                G.set_mapped_block_walks(0)  # every block copied, as findSubGraph does
                _add_golden_walks(G, g, tag)
                st = G.run(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=int(g["seed"]),
                                     mode=gw.MODE_BLOCKED, prob=prob))
                assert np.array_equal(G.read_counts(), g[f"{tag}_counts"]), f"{case}/{tag}/{residency}"
                assert st.supersteps == ref["supersteps"]
                if residency == gw.STREAM_PINNED:
                    assert st.block_loads >= 1


@pytest.mark.parametrize("case", ["rmat10", "rmat13"])
@pytest.mark.parametrize("mapped", ["all", "small"])
def test_streamed_blocks_read_in_place_match_reference_loop(cuda_device, oracle, case, mapped):
    """Streamed blocks whose pools are small are read in place from pinned host
    memory instead of being copied into a slot: the same supersteps, the same
    counts, and (every block read in place) no block copies at all."""
    import graphwalker_b200 as gw
    g = load_golden(case)
    for tag in ("jump", "stop"):
        rule, L = int(g[f"{tag}_rule"]), int(g[f"{tag}_L"])
        ref = oracle.block_engine(g["rowptr"], g["colidx"], g["blocks"], g[f"{tag}_cur"], rule=rule, L=L,
                                  seed=int(g["seed"]), prob=0.2)
        limit = (1 << 63) if mapped == "all" else max(1, len(g[f"{tag}_cur"]) // (4 * (len(g["blocks"]) - 1)))
        with _graph(g, gw.STREAM_PINNED) as G:
            G.set_mapped_block_walks(limit)
            _add_golden_walks(G, g, tag)
            st = G.run(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=int(g["seed"]), mode=gw.MODE_BLOCKED,
                                 prob=0.2))
            assert np.array_equal(G.read_counts(), g[f"{tag}_counts"]), f"{case}/{tag}/{mapped}"
            assert st.supersteps == ref["supersteps"]
            assert st.mapped_supersteps >= 1
            if mapped == "all":
                assert st.block_loads == 0 and st.bytes_h2d == 0
                assert st.mapped_supersteps == st.supersteps and st.mapped_walks >= len(g[f"{tag}_cur"])
            else:
                assert st.mapped_supersteps < st.supersteps


@pytest.mark.parametrize("steps", [1, 3, 7])
def test_blocked_pools_are_stable_partitions(cuda_device, oracle, steps):
    """Pools after k supersteps equal the reference loop with stable pools."""
    import graphwalker_b200 as gw
    g = load_golden("rmat10")
    cur = g["jump_cur"]
    ref = oracle.block_engine(g["rowptr"], g["colidx"], g["blocks"], cur, rule=0, L=10,
                              seed=int(g["seed"]), prob=0.2, max_supersteps=steps)
    with _graph(g) as G:
        _add_golden_walks(G, g, "jump")
        st = G.run(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=int(g["seed"]), mode=gw.MODE_BLOCKED,
                             prob=0.2, max_supersteps=steps))
        assert st.supersteps == ref["supersteps"] == steps
        assert np.array_equal(G.read_counts(), ref["counts"])
        for b in range(G.nblocks):
            pool = G.read_pool(b)
            exp = np.stack(ref["pools"][b], axis=1) if len(ref["pools"][b][0]) else np.zeros((0, 4), np.uint32)
            assert np.array_equal(pool, exp), f"block {b}"


@pytest.mark.parametrize("steps", [3, 7, 0])
@pytest.mark.parametrize("residency", [0, 1], ids=["hbm", "streamed"])
def test_pool_budget_spills_pools_in_order(cuda_device, oracle, steps, residency):
    """A device budget far below the walk state: pools move to host memory and
    come back when their block runs.  Pools after k supersteps (their host part
    first) still equal the stable-pool restatement, and the full run's counts
    and superstep count equal the reference loop's."""
    import graphwalker_b200 as gw
    g = load_golden("rmat13")
    cur = g["jump_cur"]
    ref = oracle.block_engine(g["rowptr"], g["colidx"], g["blocks"], cur, rule=0, L=10,
                              seed=int(g["seed"]), prob=0.2, max_supersteps=steps)
    with _graph(g, residency) as G:
        G.set_pool_budget(48 * 1024)  # 3072 walk records; the run holds 8192 walks
        _add_golden_walks(G, g, "jump")
        st = G.run(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=int(g["seed"]), mode=gw.MODE_BLOCKED,
                             prob=0.2, max_supersteps=steps))
        assert st.supersteps == ref["supersteps"]
        assert np.array_equal(G.read_counts(), ref["counts"])
        assert st.pools_spilled > 0 and st.pools_refilled > 0
        for b in range(G.nblocks):
            pool = G.read_pool(b)
            exp = np.stack(ref["pools"][b], axis=1) if len(ref["pools"][b][0]) else np.zeros((0, 4), np.uint32)
            assert np.array_equal(pool, exp), f"block {b}"
        if steps == 0:
            assert np.array_equal(G.read_counts(), g["jump_counts"])


@pytest.mark.parametrize("rule", [0, 1, 3], ids=["jump", "stop", "restart"])
def test_streamed_in_place_and_spilled_native_rng(cuda_device, oracle, rule):
    """Both RNG modes through the streamed block loop with every block read in
    place and the walk pools over a small budget: counts equal the oracle's
    (which do not depend on the schedule)."""
    import graphwalker_b200 as gw
    g = load_golden("rmat13")
    rp, ci = g["rowptr"], g["colidx"]
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    L = 6
    with _graph(g, gw.STREAM_PINNED) as G:
        G.set_mapped_block_walks(1 << 40)
        G.set_pool_budget(32 * 1024)
        for rng in (0, 1):
            ref = oracle.run_walks(rp, ci, cur, rule=rule, L=L, seed=11, rng=rng)
            G.walks_clear()
            G.add_walks_at(cur)
            st = G.run(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=11, mode=gw.MODE_BLOCKED, rng=rng))
            assert np.array_equal(G.read_counts(), ref["counts"]), rng
            assert st.block_loads == 0 and st.pools_spilled > 0


def test_device_rmat_matches_oracle(cuda_device, oracle):
    import graphwalker_b200 as gw
    for scale, ef, seed in [(10, 16, 1), (13, 8, 3), (16, 16, 9)]:
        rp, ci = oracle.rmat_csr(scale, ef, seed=seed)
        with gw.Graph.rmat(scale, ef, seed=seed, blocksize_kb=64) as G:
            drp, dci = G.export_csr()
            assert np.array_equal(drp, rp) and np.array_equal(dci, ci)
            assert np.array_equal(G.blocks, oracle.compute_blocks(rp, 64))


def test_device_pointer_entry_points(cuda_device, oracle):
    import torch
    import graphwalker_b200 as gw
    g = load_golden("rmat10")
    nv = len(g["rowptr"]) - 1
    with _graph(g) as G:
        words = gw.encode(np.arange(nv), np.arange(nv), 0)  # all in block 0 when relative to 0
        b0 = int(G.blocks[1])
        dw = torch.from_numpy(words[:b0].view(np.int64)).cuda()
        recs = torch.empty((b0, 4), dtype=torch.int32, device="cuda")
        G.unpack_words_device(0, dw, None, b0, recs)
        counts = torch.zeros(nv, dtype=torch.int32, device="cuda")
        G.walk_device(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=int(g["seed"])), recs, b0, counts=counts)
        G.sync()
        ref = oracle.run_walks(g["rowptr"], g["colidx"], np.arange(b0, dtype=np.uint32), rule=0, L=10,
                               seed=int(g["seed"]))
        assert np.array_equal(counts.cpu().numpy().view(np.uint32), ref["counts"])
        back = torch.empty(b0, dtype=torch.int64, device="cuda")
        G.pack_words_device(recs, b0, back)
        torch.cuda.synchronize()
        assert np.array_equal(back.cpu().numpy().view(np.uint64), words[:b0])


def test_run_pools_host_call(cuda_device, oracle):
    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(15, 16, seed=4)
    blocks = oracle.compute_blocks(rp, 256)
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    blk = np.searchsorted(blocks[1:], cur, side="right")
    words = gw.encode(cur, cur - blocks[blk], 0)
    offs = np.r_[0, np.cumsum(np.bincount(blk, minlength=len(blocks) - 1))].astype(np.uint64)
    ref = oracle.run_walks(rp, ci, cur, rule=0, L=10, seed=3)
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        out = np.zeros(nv, np.uint32)
        G.run_pools(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=3), words, offs, out)
        assert np.array_equal(out, ref["counts"])


def test_run_pools_pipelined_equals_oracle(cuda_device, oracle):
    """gw_run_pools_submit / wait: two runs in flight, each with the counts of
    its own seed (and ids); a third submit is refused until the older run is
    waited on; a device error reaches the wait of its own run only."""
    import graphwalker_b200 as gw
    from graphwalker_b200._lib import GW_E_BOUNDS, GW_E_INVALID, GW_E_STATE, GwError
    rp, ci = oracle.rmat_csr(15, 16, seed=4)
    blocks = oracle.compute_blocks(rp, 256)
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    blk = np.searchsorted(blocks[1:], cur, side="right")
    words = gw.encode(cur, cur - blocks[blk], 0)
    offs = np.r_[0, np.cumsum(np.bincount(blk, minlength=len(blocks) - 1))].astype(np.uint64)
    ids = (cur * 7 + 11).astype(np.uint32)
    seeds = [3, 4, 5, 6, 7]
    refs = {s: oracle.run_walks(rp, ci, cur, ids=ids if s % 2 else None, rule=0, L=10, seed=s)["counts"]
            for s in seeds}
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        outs = {s: np.full(nv, 0xDEAD, np.uint32) for s in seeds}
        pending = []
        for s in seeds:
            if len(pending) == 2:
                with pytest.raises(GwError) as e:  # two in flight already
                    G.run_pools_submit(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=s), words, offs, outs[s])
                assert e.value.code == GW_E_STATE
                t, done = pending.pop(0)
                G.run_pools_wait(t)
                assert np.array_equal(outs[done], refs[done]), done
            t = G.run_pools_submit(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=s), words, offs, outs[s],
                                   ids=ids if s % 2 else None)
            pending.append((t, s))
        for t, done in pending:
            G.run_pools_wait(t)
            assert np.array_equal(outs[done], refs[done]), done
        with pytest.raises(GwError) as e:
            G.run_pools_wait(pending[-1][0])  # already waited
        assert e.value.code == GW_E_INVALID
        # a walk past the last vertex: its run's wait reports GW_E_BOUNDS, the
        # run in flight beside it is unaffected
        bad = words.copy()
        bad[-1] = gw.encode([0], [nv - int(blocks[-2]) + 5], [0])[0]
        out_bad, out_ok = np.zeros(nv, np.uint32), np.zeros(nv, np.uint32)
        tb = G.run_pools_submit(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=3), bad, offs, out_bad)
        tk = G.run_pools_submit(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=4), words, offs, out_ok)
        with pytest.raises(GwError) as e:
            G.run_pools_wait(tb)
        assert e.value.code == GW_E_BOUNDS
        G.run_pools_wait(tk)
        assert np.array_equal(out_ok, refs[4])


def test_errors_surface_as_status_codes(cuda_device, oracle):
    import graphwalker_b200 as gw
    from graphwalker_b200._lib import GW_E_BOUNDS, GW_E_INVALID, GW_E_OVERFLOW, GwError
    g = load_golden("hand")
    with _graph(g) as G:
        # a start vertex past the last block: the kernel's bounds check ends the
        # walk and reports GW_E_BOUNDS (no out-of-range load is issued)
        G.walks_add(int(G.nblocks - 1), gw.encode([0], [1000], [0]))
        with pytest.raises(GwError) as e:
            G.run(gw.params(0, gw.SINK_VERTEX_COUNT, 5))
        assert e.value.code == GW_E_BOUNDS
        G.walks_clear()
        G.add_walks_at(np.arange(12, dtype=np.uint32))
        with pytest.raises(GwError) as e:
            G.run(gw.params(0, gw.SINK_PATH_RECORD, 10, path_stride=3))
        assert e.value.code == GW_E_OVERFLOW
        with pytest.raises(GwError) as e:
            G.run(gw.params(3, gw.SINK_VERTEX_COUNT, 0))
        assert e.value.code == GW_E_INVALID
        # the context stays usable after device-reported errors
        G.run(gw.params(0, gw.SINK_VERTEX_COUNT, 10, seed=int(g["seed"])))
        assert G.read_counts().sum() == 12 * 10


@pytest.mark.parametrize("rule,L", [(0, 10), (3, 6)])
def test_checkpoint_and_resume_are_exact(cuda_device, oracle, rule, L):
    """A superstep-boundary checkpoint (pending pools + counts) resumed in a
    fresh context finishes with exactly the counts of an uninterrupted run:
    every draw is keyed on (walk id, hop), so where a walk stopped does not
    matter.  The reference's pools on disk are deleted at start and could not
    serve as one (walk.hpp:50-51)."""
    import graphwalker_b200 as gw
    g = load_golden("rmat13")
    seed = int(g["seed"])
    cur = g["jump_cur"]
    ids = np.arange(len(cur), dtype=np.uint32)
    full = oracle.run_walks(g["rowptr"], g["colidx"], cur, ids=ids, src=cur, rule=rule, L=L, seed=seed)["counts"]
    with _graph(g) as G:
        G.walks_clear()
        G.add_walks_at(cur, source=cur, ids=ids)
        G.run(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=seed, mode=gw.MODE_BLOCKED, max_supersteps=7))
        part = G.read_counts().astype(np.int64)
        pools = [G.read_pool(b) for b in range(G.nblocks)]
    left = np.concatenate([p for p in pools if len(p)]) if any(len(p) for p in pools) else np.zeros((0, 4), np.uint32)
    assert 0 < len(left) < len(cur)  # stopped mid-run
    with _graph(g) as G2:  # resume in a new context
        G2.walks_clear()
        if len(left):
            G2.add_walks_at(left[:, 0], source=left[:, 2], hop=left[:, 3], ids=left[:, 1])
        G2.run(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=seed))
        rest = G2.read_counts().astype(np.int64)
    assert np.array_equal(part + rest, full.astype(np.int64))


def test_walk_autotune_keeps_results(cuda_device, oracle):
    """The tuned launch shape of the resident kernel changes no count."""
    import torch

    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(16, 16, seed=2)
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    ref = oracle.run_walks(rp, ci, cur, ids=cur, src=cur, rule=0, L=10, seed=8)["counts"]
    with gw.Graph.from_csr(rp, ci, oracle.compute_blocks(rp, 512)) as G:
        v = torch.arange(nv, dtype=torch.int64, device="cuda")
        walks = torch.stack([v, v, v, torch.zeros_like(v)], dim=1).to(torch.int32).contiguous()
        p = gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, 10, seed=8)
        c = G.walk_autotune(p, walks, nv)
        assert 1 <= c <= 8
        counts = torch.zeros(nv, dtype=torch.int32, device="cuda")
        G.walk_device(p, walks, nv, counts=counts)
        G.sync()
        assert np.array_equal(counts.cpu().numpy().view(np.uint32), ref)
