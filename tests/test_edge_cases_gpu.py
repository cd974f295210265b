"""Edge cases of the walk kernels against the oracle.

Short walks (L = 0, 1, 2) are where the kernels' own shortcuts sit: the move
after a walk's last visit is skipped (nothing observes it), and a jump
target's record is fetched only when the target moves on.  Every rule, both
graph layouts, the resident, blocked and query kernels, walks that start at
odd hops, at the cap or past it, and empty calls.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RULES = [0, 1, 2, 3, 4]
RULE_IDS = ["jump", "stop", "prob", "restart", "ppr"]


@pytest.fixture(scope="module")
def graph(cuda_device, oracle):
    rp, ci = oracle.rmat_csr(11, 6, seed=9)
    return rp, ci, oracle.compute_blocks(rp, 8)


@pytest.mark.parametrize("rule", RULES, ids=RULE_IDS)
@pytest.mark.parametrize("L", [0, 1, 2, 3])
@pytest.mark.parametrize("layout", [0, 1], ids=["csr", "edge_records"])
def test_short_walks_equal_oracle(graph, oracle, rule, L, layout):
    import graphwalker_b200 as gw
    if rule == 3 and L == 0:
        pytest.skip("the restart rule needs L >= 1")
    rp, ci, blocks = graph
    nv = len(rp) - 1
    rng = np.random.default_rng(L * 10 + rule)
    cur = rng.integers(0, nv, 3000).astype(np.uint32)
    # starting hops below, at and past the cap (the uncapped rule keeps hop < max_hops)
    hop0 = rng.integers(0, max(1, L + 2), 3000).astype(np.uint32) if rule != 3 else np.zeros(3000, np.uint32)
    ids = np.arange(3000, dtype=np.uint32)
    for rng_mode in (0, 1):
        ref = oracle.run_walks(rp, ci, cur, ids=ids, src=cur, hop0=hop0, rule=rule, L=L, seed=77, rng=rng_mode)
        assert ref["status"] == 0
        with gw.Graph.from_csr(rp, ci, blocks) as G:
            assert G.set_edge_records(layout) == bool(layout)
            for mode in (gw.MODE_RESIDENT, gw.MODE_BLOCKED):
                G.walks_clear()
                G.add_walks_at(cur, hop=hop0, ids=ids)
                G.run(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=77, mode=mode, rng=rng_mode))
                assert np.array_equal(G.read_counts(), ref["counts"]), (mode, rng_mode)


@pytest.mark.parametrize("rule", [0, 1, 3, 4], ids=["jump", "stop", "restart", "ppr"])
@pytest.mark.parametrize("L", [1, 2])
def test_short_queries_equal_oracle(graph, oracle, rule, L):
    """msppr queries of one- and two-visit walks: top-k lists equal the oracle's."""
    import graphwalker_b200 as gw
    from graphwalker_b200 import accuracy
    rp, ci, blocks = graph
    deg = np.diff(rp.astype(np.int64))
    rng = np.random.default_rng(rule + 5 * L)
    sources = rng.choice(np.nonzero(deg)[0], 12).astype(np.uint32)
    budgets = rng.integers(1, 400, 12).astype(np.uint32)
    prefix = np.r_[0, np.cumsum(budgets.astype(np.int64))]
    k = 20
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        G.set_edge_records(1)
        ids, cnt, _ = G.ppr(gw.params(rule, gw.SINK_NONE, L, seed=3), sources, budgets, k=k, batched=True)
    for q in range(len(sources)):
        c = np.full(int(budgets[q]), sources[q], np.uint32)
        r = oracle.run_walks(rp, ci, c, ids=np.arange(prefix[q], prefix[q + 1], dtype=np.uint32), src=c, rule=rule,
                             L=L, seed=3)
        nz = np.flatnonzero(r["counts"])
        want = accuracy.count_topk(nz, r["counts"][nz], k)
        assert np.array_equal(ids[q][ids[q] != 0xFFFFFFFF], want), q
        assert np.array_equal(cnt[q][: len(want)], r["counts"][want]), q


def test_paths_and_closure_of_short_walks(graph, oracle):
    """Path records and closure counts of one- and two-visit walks (the
    visits a walk makes are recorded even though its last move is skipped)."""
    import graphwalker_b200 as gw
    rp, ci, blocks = graph
    nv = len(rp) - 1
    cur = np.arange(nv, dtype=np.uint32)
    for L in (1, 2):
        ref = oracle.run_walks(rp, ci, cur, rule=0, L=L, seed=5, stride=L, closure=True)
        with gw.Graph.from_csr(rp, ci, blocks) as G:
            G.set_edge_records(1)
            G.walks_clear()
            G.add_walks_at(cur)
            G.run(gw.params(0, gw.SINK_PATH_RECORD, L, seed=5, path_stride=L))
            paths, lens = G.read_paths(nv, L)
            blk = np.searchsorted(G.blocks[1:], cur, side="right")
            order = np.argsort(blk, kind="stable")  # pool order
            assert np.array_equal(paths, ref["paths"][order])
            assert np.array_equal(lens, ref["plen"][order])
            G.run(gw.params(0, gw.SINK_CLOSURE_COUNT, L, seed=5))
            assert G.read_closure() == ref["closure"]


def test_empty_calls(graph):
    """No walks, no queries: every entry point returns cleanly and writes
    zero counts."""
    import torch

    import graphwalker_b200 as gw
    rp, ci, blocks = graph
    nv = len(rp) - 1
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        p = gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, 10, seed=1)
        counts = torch.full((nv,), 7, dtype=torch.int32, device="cuda")
        walks = torch.zeros((1, 4), dtype=torch.int32, device="cuda")
        G.walk_device(p, walks, 0, counts=counts)
        G.sync()
        assert np.all(counts.cpu().numpy() == 7)  # n = 0 touches nothing
        words = np.zeros(1, np.uint64)
        offs = np.zeros(G.nblocks + 1, np.uint64)
        out = np.full(nv, 9, np.uint32)
        G.run_pools(p, words, offs, out)
        assert np.all(out == 0)  # the counts of no walks
        out[:] = 9
        G.run_pools_wait(G.run_pools_submit(p, words, offs, out))
        assert np.all(out == 0)
        ids, cnt, st = G.ppr(gw.params(gw.RULE_STOP, gw.SINK_NONE, 20), np.zeros(0, np.uint32),
                             np.zeros(0, np.uint32), k=10)
        assert ids.shape == (0, 10) and st.walks == 0
        G.walks_clear()
        st = G.run(gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, 10, mode=gw.MODE_BLOCKED))
        assert st.walks == 0 and not G.read_counts().any()
