"""Multi-source PPR queries (msppr): per-query sparse counts and exact top-k.

Parity is bit-exact against the oracle (per-walk trajectories, walk j of the
batch keyed by stream id j) and between the batched and the plain
one-query-at-a-time paths; accuracy is stated against the FP64 power series.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _topk_ref(counts: dict, k: int):
    """Top k (vertex, count) by count desc, vertex asc."""
    items = sorted(counts.items(), key=lambda kv: (-kv[1], kv[0]))[:k]
    ids = np.full(k, 0xFFFFFFFF, np.uint32)
    cnt = np.zeros(k, np.uint32)
    for r, (v, c) in enumerate(items):
        ids[r], cnt[r] = v, c
    return ids, cnt


def _oracle_queries(oracle, rp, ci, sources, budgets, rule, L, seed, k):
    prefix = np.r_[0, np.cumsum(budgets)].astype(np.int64)
    cur = np.repeat(np.asarray(sources, np.uint32), budgets)
    ids = np.arange(prefix[-1], dtype=np.uint32)
    stride = L if rule != 2 else 128
    r = oracle.run_walks(rp, ci, cur, ids=ids, src=cur, rule=rule, L=L, seed=seed, stride=stride, counts=False)
    assert r["status"] == 0
    out_ids = np.zeros((len(sources), k), np.uint32)
    out_cnt = np.zeros((len(sources), k), np.uint32)
    for q in range(len(sources)):
        counts = {}
        for w in range(prefix[q], prefix[q + 1]):
            for v in r["paths"][w][: r["plen"][w]]:
                counts[int(v)] = counts.get(int(v), 0) + 1
        out_ids[q], out_cnt[q] = _topk_ref(counts, k)
    return out_ids, out_cnt


@pytest.mark.parametrize("rule,L", [(1, 20), (4, 20), (3, 6), (0, 8)])
@pytest.mark.parametrize("layout", [0, 1])
def test_ppr_queries_match_oracle(cuda_device, oracle, rule, L, layout):
    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(13, 8, seed=21)
    deg = np.diff(rp.astype(np.int64))
    rng = np.random.default_rng(rule)
    sources = rng.choice(np.nonzero(deg)[0], 40).astype(np.uint32)
    sources[0] = np.nonzero(deg == 0)[0][0]  # a dangling source
    sources[1] = sources[2]                 # a repeated source
    budgets = rng.integers(1, 1500, 40).astype(np.uint32)
    budgets[3] = 0                          # an empty query
    k = 50
    ref_ids, ref_cnt = _oracle_queries(oracle, rp, ci, sources, budgets, rule, L, 13, k)
    with gw.Graph.from_csr(rp, ci, oracle.compute_blocks(rp, 64)) as G:
        assert G.set_edge_records(layout) == bool(layout)
        p = gw.params(rule, gw.SINK_NONE, L, seed=13)
        for batched in (True, False):
            ids, cnt, st = G.ppr(p, sources, budgets, k=k, batched=batched)
            assert np.array_equal(ids, ref_ids), f"batched={batched}"
            assert np.array_equal(cnt, ref_cnt), f"batched={batched}"
            assert st.walks == budgets.sum()


@pytest.mark.parametrize("tag_bits", [None, "2", "0"], ids=["tags", "3_tags", "untagged"])
def test_batches_reuse_tables_exactly(cuda_device, oracle, monkeypatch, tag_bits):
    """Consecutive batches in one context, with different table layouts
    (growing, shrinking): each batch writes under a new tag and sees none of
    the earlier batches' slots.  With 3 tags the tables are cleared every
    third batch; untagged, every batch.  Each result equals the oracle's."""
    import graphwalker_b200 as gw
    if tag_bits is None:
        monkeypatch.delenv("GW_PPR_TAG_BITS", raising=False)
    else:
        monkeypatch.setenv("GW_PPR_TAG_BITS", tag_bits)
    rp, ci = oracle.rmat_csr(12, 8, seed=5)
    deg = np.diff(rp.astype(np.int64))
    rng = np.random.default_rng(31)
    p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=8)
    with gw.Graph.from_csr(rp, ci, oracle.compute_blocks(rp, 64)) as G:
        for nq, top in [(20, 300), (30, 1200), (10, 50), (40, 900), (25, 2500), (5, 20), (30, 600), (15, 1500)]:
            sources = rng.choice(np.nonzero(deg)[0], nq).astype(np.uint32)
            budgets = rng.integers(1, top, nq).astype(np.uint32)
            ref_ids, ref_cnt = _oracle_queries(oracle, rp, ci, sources, budgets, 1, 20, 8, 30)
            ids, cnt, _ = G.ppr(p, sources, budgets, k=30)
            assert np.array_equal(ids, ref_ids) and np.array_equal(cnt, ref_cnt), (nq, top)


def test_split_tables_ranked_largest_first_match_oracle(cuda_device, oracle):
    """Tables of 2 to 8 top-k segments beside one-segment tables: the
    segments are ranked largest first and merged per query; each list equals
    the oracle's."""
    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(12, 8, seed=6)
    deg = np.diff(rp.astype(np.int64))
    rng = np.random.default_rng(4)
    budgets = np.array([5000, 20, 3000, 1, 70, 9000, 400, 2500], np.uint32)
    sources = rng.choice(np.nonzero(deg)[0], len(budgets)).astype(np.uint32)
    ref_ids, ref_cnt = _oracle_queries(oracle, rp, ci, sources, budgets, 1, 20, 3, 100)
    p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=3)
    with gw.Graph.from_csr(rp, ci, oracle.compute_blocks(rp, 64)) as G:
        for batched in (True, False):
            ids, cnt, st = G.ppr(p, sources, budgets, k=100, batched=batched)
            assert np.array_equal(ids, ref_ids) and np.array_equal(cnt, ref_cnt), f"batched={batched}"
        assert st.table_slots > 16384 * len(budgets)  # some tables span several segments


def test_ppr_batched_equals_plain_at_scale(cuda_device):
    import graphwalker_b200 as gw
    with gw.Graph.rmat(18, 16, seed=4, blocksize_kb=1024) as G:
        rp, _ = G.export_csr()
        deg = np.diff(rp.astype(np.int64))
        rng = np.random.default_rng(9)
        nq = 300
        sources = rng.choice(np.nonzero(deg)[0], nq).astype(np.uint32)
        budgets = np.round(10 ** rng.uniform(2, 4, nq)).astype(np.uint32)
        p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=77)
        ib, cb, sb = G.ppr(p, sources, budgets, k=100, batched=True)
        ip, cp, sp = G.ppr(p, sources, budgets, k=100, batched=False)
        assert np.array_equal(ib, ip) and np.array_equal(cb, cp)
        # the source is visited by every walk at hop 0
        assert np.all(cb[:, 0] >= budgets)
        for _ in range(3):  # repeated batches: the same lists every time
            ir, cr, _ = G.ppr(p, sources, budgets, k=100, batched=True)
            assert np.array_equal(ir, ip) and np.array_equal(cr, cp)
        threads, chunk = G.ppr_autotune(p, sources[:50], budgets[:50])
        assert threads in (512, 1024, 1536, 2048) and chunk in (64, 128, 256, 512)
        it, ct, _ = G.ppr(p, sources, budgets, k=100, batched=True)
        assert np.array_equal(it, ib) and np.array_equal(ct, cb)
        # the plain CSR layout gives the same lists as the edge records
        assert G.set_edge_records(gw.EDGE_RECORDS_OFF) is False
        io, co, _ = G.ppr(p, sources, budgets, k=100, batched=True)
        assert np.array_equal(io, ib) and np.array_equal(co, cb)


def test_ppr_full_tables_are_rerun_exactly(cuda_device, oracle):
    """Queries whose visit table fills up are re-run with larger tables and
    give exactly the result of a table that was large enough from the start."""
    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(14, 16, seed=2)
    deg = np.diff(rp.astype(np.int64))
    rng = np.random.default_rng(4)
    sources = rng.choice(np.nonzero(deg)[0], 20).astype(np.uint32)
    budgets = rng.integers(50, 3000, 20).astype(np.uint32)
    with gw.Graph.from_csr(rp, ci, oracle.compute_blocks(rp, 128)) as G:
        p = gw.params(gw.RULE_JUMP, gw.SINK_NONE, 20, seed=1)  # jumps visit many distinct vertices
        p.table_factor = 64
        ref_ids, ref_cnt, _ = G.ppr(p, sources, budgets, k=100)
        p.table_factor = 1  # max(256, budget) slots: most tables fill up
        for batched in (True, False):
            ids, cnt, st = G.ppr(p, sources, budgets, k=100, batched=batched)
            assert np.array_equal(ids, ref_ids) and np.array_equal(cnt, ref_cnt)
            assert st.launches > (3 if batched else 60)  # retries ran


def test_ppr_accuracy_against_fp64_power_series(cuda_device, oracle):
    """Top-100 of 100k walks vs the exact expected visits (FP64): every listed
    count lies within 5 standard deviations of its expectation and the list
    overlaps the exact top-100 by at least 90."""
    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(14, 16, seed=5)
    deg = np.diff(rp.astype(np.int64))
    rng = np.random.default_rng(3)
    sources = rng.choice(np.nonzero(deg > 4)[0], 3).astype(np.uint32)
    B, L = 100_000, 20
    with gw.Graph.from_csr(rp, ci, oracle.compute_blocks(rp, 128)) as G:
        p = gw.params(gw.RULE_STOP, gw.SINK_NONE, L, seed=99)
        ids, cnt, _ = G.ppr(p, sources, np.full(3, B, np.uint32), k=100)
    for q, s in enumerate(sources):
        mu = oracle.expected_visits(rp, ci, int(s), 1, L)  # expected visits per walk
        est = cnt[q].astype(np.float64) / B
        sd = np.sqrt(L * mu[ids[q]] / B)
        assert np.all(np.abs(est - mu[ids[q]]) <= 5 * sd + 1e-9)
        exact_top = set(np.argsort(-mu, kind="stable")[:100].tolist())
        assert len(exact_top & set(ids[q].tolist())) >= 90


@pytest.mark.parametrize("rule,L", [(0, 10), (1, 20), (3, 7), (4, 20), (2, 0)])
def test_expected_visits_kernel_matches_fp64_oracle(cuda_device, oracle, rule, L):
    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(12, 8, seed=17)
    deg = np.diff(rp.astype(np.int64))
    src = int(np.argmax(deg))
    with gw.Graph.from_csr(rp, ci, oracle.compute_blocks(rp, 32)) as G:
        got = G.expected_visits(gw.params(rule, gw.SINK_NONE, L), src)
    ref = oracle.expected_visits(rp, ci, src, rule, L)
    assert np.allclose(got, ref, rtol=1e-9, atol=1e-13)
